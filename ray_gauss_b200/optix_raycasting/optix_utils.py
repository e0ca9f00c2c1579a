"""Mirror of the reference's ``optix_raycasting/optix_utils.py`` host helpers on top of the B200
engine, so that a training script written against the reference keeps its call sites.

OptiX objects (context, modules, program groups, pipelines, shader-binding tables) have no
counterpart: ``create_context`` returns an :class:`~ray_gauss_b200.engine.Engine` (which the
drop-in ``RenderOptixSettings`` accepts as its ``context``) and the module/pipeline/SBT builders
return inert placeholders.  The geometric helpers compute what the reference computes:

  quaternion_to_rotation      optix_utils.py:34-46  (rows L1, L2, L3 of R for (w,x,y,z))
  compute_spheres_bbox        optix_utils.py:48-52
  compute_ellipsoids_bbox     optix_utils.py:54-66  (engine pre-pass; (N,6) device tensor)
  create_acceleration_structure / update_acceleration_structure  optix_utils.py:68-75 (LBVH)
  launch_pipeline_forward / launch_pipeline_backward             optix_utils.py:128-299
"""
from __future__ import annotations

import math

import torch

from ..engine import Engine, engine_for, make_gaussians, settings_struct

SIGMA_THRESHOLD = 0.1


def get_SIGMA_THRESHOLD(file_name=None):
    """The per-sample density threshold shared by all reference programs (gaussians_aabb.h:5)."""
    return SIGMA_THRESHOLD


def quaternion_to_rotation(quaternion):
    w, x, y, z = quaternion[:, 0], quaternion[:, 1], quaternion[:, 2], quaternion[:, 3]
    L1 = torch.stack([1 - 2 * (y ** 2 + z ** 2), 2 * (x * y - w * z), 2 * (x * z + w * y)], dim=1)
    L2 = torch.stack([2 * (x * y + w * z), 1 - 2 * (x ** 2 + z ** 2), 2 * (y * z - w * x)], dim=1)
    L3 = torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x ** 2 + y ** 2)], dim=1)
    return L1, L2, L3


def compute_spheres_bbox(centers, scales):
    return torch.cat([centers - 3 * scales, centers + 3 * scales], dim=1)


class _Placeholder:
    """Stands in for an OptiX object the engine does not need."""

    def __init__(self, what):
        self.what = what

    def __repr__(self):
        return f"<no OptiX object: {self.what}>"


class _GaussianSet:
    """Parameters handed to compute_ellipsoids_bbox, kept for the BVH helpers below."""

    def __init__(self, g):
        self.g = g


def create_context(log=None):
    return engine_for(torch.cuda.current_device())


def create_module(ctx, pipeline_opts=None, stage="forward"):
    if stage not in ("forward", "backward", "test", "gui"):
        raise ValueError("stage must be 'forward', 'backward', 'test' or 'gui'")
    return _Placeholder(f"module {stage}")


def create_program_groups(ctx, module):
    return (_Placeholder("raygen"), _Placeholder("miss"), _Placeholder("hitgroup"))


def create_pipeline(ctx, program_grps, pipeline_options=None, debug_level=None):
    return _Placeholder("pipeline")


def create_sbt(program_grps, positions, scales, quaternions):
    return _Placeholder("sbt")


_LAST = {}


def compute_ellipsoids_bbox(centers, scales, L1, L2, L3, densities, quaternions=None, engine: Engine | None = None):
    """(N,6) AABBs of the threshold ellipsoids.  The engine derives R from the quaternions itself;
    when only L1..L3 are given the quaternion is recovered from R (w >= 0 branch)."""
    eng = engine or engine_for(centers.device)
    if quaternions is None:
        quaternions = _rotation_to_quaternion(L1, L2, L3)
    n = centers.shape[0]
    dummy_sh = torch.zeros((n, 3, 1), device=centers.device)
    g = make_gaussians(centers, scales, quaternions, densities, dummy_sh)
    out = torch.empty((n, 6), dtype=torch.float32, device=centers.device)
    eng.ellipsoids_bbox(g, aabb_out=out)
    _LAST[id(eng)] = g
    return out


def _rotation_to_quaternion(L1, L2, L3):
    R = torch.stack([L1, L2, L3], dim=1).float()
    w = torch.sqrt(torch.clamp(1 + R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2], min=1e-12)) / 2
    x = (R[:, 2, 1] - R[:, 1, 2]) / (4 * w)
    y = (R[:, 0, 2] - R[:, 2, 0]) / (4 * w)
    z = (R[:, 1, 0] - R[:, 0, 1]) / (4 * w)
    return torch.stack([w, x, y, z], dim=1).contiguous()


def create_acceleration_structure(ctx, bboxes=None):
    """Build the LBVH over the Gaussians of the last compute_ellipsoids_bbox call on ``ctx``."""
    eng = ctx if isinstance(ctx, Engine) else engine_for(torch.cuda.current_device())
    eng.bvh_build()
    return eng


def update_acceleration_structure(gas, bboxes=None):
    eng = gas if isinstance(gas, Engine) else engine_for(torch.cuda.current_device())
    eng.bvh_refit()


def launch_pipeline_forward(pipeline, sbt, gas, bbox_min, bbox_max, camera, densities, color_features, positions,
                            scales, quaternions, max_prim_slice, iteration, jitter, rnd_sample, supersampling,
                            white_background, hit_prim_idx=None, color_sh=None):
    """Forward launch on per-Gaussian colours ``color_features`` (N,3) — the reference passes the
    output of its SH kernel here (render_optix.py:114-122).  Returns ray colours (R,3)."""
    eng = gas if isinstance(gas, Engine) else engine_for(positions.device)
    rgb = color_features.reshape(-1, 3).float()
    sh0 = ((rgb - 0.5) / 0.28209479177387814).reshape(-1, 3, 1).contiguous()
    g = make_gaussians(positions, scales, quaternions, densities, sh0)
    cams_t, recs, _ = eng.cameras([camera], tuple(supersampling))
    st = settings_struct(white_background, jitter, rnd_sample, max_prim_slice, iteration)
    out, _ = eng.render_forward(g, cams_t, 1, recs[0].width * recs[0].height, st, refit=True)
    return out


def launch_pipeline_backward(pipeline, sbt, gas, bbox_min, bbox_max, camera, densities, color_features, positions,
                             scales, quaternions, ray_colors, dloss_dray_colors, max_prim_slice, iteration, jitter,
                             rnd_sample, supersampling, hit_prim_idx=None):
    """Backward launch; returns (densities_grad, color_features_grad (N,3), positions_grad,
    scales_grad, quaternions_grad) as optix_utils.py:282-299 (position gradient without the
    view-direction term, which the reference adds after its SH backward)."""
    eng = gas if isinstance(gas, Engine) else engine_for(positions.device)
    rgb = color_features.reshape(-1, 3).float()
    sh0 = ((rgb - 0.5) / 0.28209479177387814).reshape(-1, 3, 1).contiguous()
    g = make_gaussians(positions, scales, quaternions, densities, sh0)
    cams_t, recs, _ = eng.cameras([camera], tuple(supersampling))
    st = settings_struct(True, jitter, rnd_sample, max_prim_slice, iteration)
    eng.ellipsoids_bbox(g)
    eng.bvh_build()
    eng.forward_sh(g, cams_t, 1)
    grads = eng.render_backward(g, cams_t, 1, st, ray_colors.contiguous().float(),
                                dloss_dray_colors.contiguous().float())
    # d(rgb) = C0 * d(sh0) for a degree-0 colour
    drgb = grads["color_features"].reshape(-1, 3) / 0.28209479177387814
    return grads["densities"], drgb, grads["positions"], grads["scales"], grads["quaternions"]


def launch_pipeline_test(pipeline, sbt, gas, bbox_min, bbox_max, camera, densities, color_features, positions,
                         scales, quaternions, max_prim_slice, rnd_sample, supersampling, white_background,
                         return_counts=False, mode="parity"):
    """Inference render (optix_utils.py:302-373 with the cuda_test programs) on per-Gaussian colours
    ``color_features`` (N,3): no jitter, no random sample offsets (``rnd_sample`` is accepted and
    ignored, as by those programs), slab queries not clipped at the scene-box exit.  Returns ray
    colours (R,3); with ``return_counts`` also the Gaussians per ray (R,) int32, which the reference
    computes but does not return."""
    eng = gas if isinstance(gas, Engine) else engine_for(positions.device)
    rgb = color_features.reshape(-1, 3).float()
    sh0 = ((rgb - 0.5) / 0.28209479177387814).reshape(-1, 3, 1).contiguous()
    g = make_gaussians(positions, scales, quaternions, densities, sh0)
    cams_t, recs, _ = eng.cameras([camera], tuple(supersampling))
    mode_id = {"parity": 0, "fast": 1}[mode]
    st = settings_struct(white_background, 0, 0, max_prim_slice, 0, mode_id)
    with torch.no_grad():
        out, cnt = eng.render_inference(g, cams_t, 1, recs[0].width * recs[0].height, st, refit=True,
                                        counts=return_counts)
    return (out, cnt) if return_counts else out
