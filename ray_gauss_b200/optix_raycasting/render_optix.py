"""Drop-in replacement of the reference renderer's torch-level call
(``optix_raycasting/render_optix.py`` of the reference project).

``RenderOptixFunction.apply(positions, scales, normalized_quaternions, densities, color_features,
sph_gauss_features, bandwidth_sharpness, lobe_axis, settings)`` returns ``ray_colors`` (R,3) float32
with R = H*W*ssx*ssy and ray index y*W + x, exactly as ``render_optix.py:92-132``; its backward
returns the nine gradients of ``render_optix.py:175-190`` (SG gradients ``None`` when there are no
spherical Gaussians, ``None`` for ``settings``).

``RenderOptixSettings`` keeps the reference constructor (``render_optix.py:67-87``).  The OptiX-only
fields (context, gas, program groups, pipelines, hit_prim_idx) are accepted and ignored, except
that ``context`` may carry an :class:`~ray_gauss_b200.engine.Engine` to use instead of the device's
default one.  ``update=True`` refits the LBVH of the previous build instead of rebuilding it (the
reference's ``update_acceleration_structure``).  Two optional keywords select the engine's sample
arithmetic (``mode``: "parity", the default, or "fast") and whether the reference's SH basis-9
y-derivative is reproduced (``sh_quirk``, default True).

Everything runs on torch's current CUDA stream without host synchronisation (the reference creates
a new CuPy stream per launch and synchronises it, ``optix_utils.py:200-202``).
"""
from __future__ import annotations

import torch

from .. import _lib
from ..engine import Engine, engine_for, make_gaussians, settings_struct

_MODES = {"parity": _lib.RG_MODE_PARITY, "fast": _lib.RG_MODE_FAST}


class RenderOptixSettings:
    def __init__(self, context, update, gas, program_grps_fwd, pipeline_fwd, program_grps_bwd, pipeline_bwd,
                 viewpoint_cam, max_prim_slice, num_sph_gauss, iteration, jitter, rnd_sample, supersampling,
                 white_background, hit_prim_idx, mode="parity", sh_quirk=True):
        self.context = context
        self.update = update
        self.gas = gas
        self.program_grps_fwd = program_grps_fwd
        self.pipeline_fwd = pipeline_fwd
        self.program_grps_bwd = program_grps_bwd
        self.pipeline_bwd = pipeline_bwd
        self.viewpoint_cam = viewpoint_cam
        self.max_prim_slice = max_prim_slice
        self.num_sph_gauss = num_sph_gauss
        self.iteration = iteration
        self.jitter = jitter
        self.rnd_sample = rnd_sample
        self.supersampling = supersampling
        self.white_background = white_background
        self.hit_prim_idx = hit_prim_idx
        self.mode = mode
        self.sh_quirk = sh_quirk


def _engine(settings, device) -> Engine:
    ctx = getattr(settings, "context", None)
    if isinstance(ctx, Engine):
        return ctx
    return engine_for(device)


def _settings_struct(settings):
    mode = settings.mode if hasattr(settings, "mode") else "parity"
    return settings_struct(white_background=settings.white_background, jitter=settings.jitter,
                           rnd_sample=settings.rnd_sample, max_prim_slice=settings.max_prim_slice,
                           iteration=settings.iteration, mode=_MODES[mode] if isinstance(mode, str) else int(mode),
                           sh_quirk=getattr(settings, "sh_quirk", True))


def _gaussians(positions, scales, quats, densities, color_features, sg, kappa, axis, nsg):
    if nsg == 0:
        sg = kappa = axis = None
    return make_gaussians(positions, scales, quats, densities, color_features, sg, kappa, axis)


class RenderOptixFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, scales, normalized_quaternions, densities, color_features, sph_gauss_features,
                bandwidth_sharpness, lobe_axis, settings):
        eng = _engine(settings, positions.device)
        nsg = int(settings.num_sph_gauss)
        g = _gaussians(positions, scales, normalized_quaternions, densities, color_features, sph_gauss_features,
                       bandwidth_sharpness, lobe_axis, nsg)
        ss = tuple(settings.supersampling)
        cams_t, recs, _ = eng.cameras([settings.viewpoint_cam], ss)
        n_rays = recs[0].width * recs[0].height
        st = _settings_struct(settings)
        ray_colors, _ = eng.render_forward(g, cams_t, 1, n_rays, st, refit=bool(settings.update))
        ctx.settings = settings
        ctx.engine = eng
        ctx.generation = eng.generation
        ctx.nsg = nsg
        ctx.save_for_backward(positions, scales, normalized_quaternions, densities, color_features,
                              sph_gauss_features, bandwidth_sharpness, lobe_axis, ray_colors.clone())
        return ray_colors

    @staticmethod
    def backward(ctx, dloss_dray_colors):
        settings, eng, nsg = ctx.settings, ctx.engine, ctx.nsg
        (positions, scales, quats, densities, color_features, sg, kappa, axis, ray_colors) = ctx.saved_tensors
        g = _gaussians(positions, scales, quats, densities, color_features, sg, kappa, axis, nsg)
        ss = tuple(settings.supersampling)
        cams_t, recs, _ = eng.cameras([settings.viewpoint_cam], ss)
        st = _settings_struct(settings)
        if eng.generation != ctx.generation:
            # another render ran on this engine since our forward: rebuild BVH and colours
            eng.ellipsoids_bbox(g)
            eng.bvh_build()
            eng.forward_sh(g, cams_t, 1)
        grads = eng.render_backward(g, cams_t, 1, st, ray_colors, dloss_dray_colors.contiguous().float())
        if nsg:
            dsg, dkap, dax = grads["sph_gauss_features"], grads["bandwidth_sharpness"], grads["lobe_axis"]
        else:
            dsg = dkap = dax = None
        return (grads["positions"], grads["scales"], grads["quaternions"], grads["densities"].reshape(densities.shape),
                grads["color_features"], dsg, dkap, dax, None)
