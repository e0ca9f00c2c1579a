"""Batched multi-view rendering: many cameras of uneven resolution in one persistent launch.

``BatchedRenderFunction.apply(positions, scales, quaternions, densities, color_features,
sph_gauss_features, bandwidth_sharpness, lobe_axis, views)`` renders every camera of ``views`` (a
:class:`BatchedViews`) in one forward launch and one backward launch.  The output packs the views'
rays in order (view v occupies ``views.offsets[v]:views.offsets[v+1]``, ray y*W+x within a view).
Parameters are read once per step for all views: one pre-pass, one BVH build (or refit), one
colour pass evaluating every view's SH/SG colour per Gaussian, one gradient assembly.

Storage: pass densities / colour features / SG amplitudes as ``torch.bfloat16`` to halve their
HBM traffic; geometry and all arithmetic and accumulation stay FP32 and gradients are FP32.
``mode="fast"`` (default here) uses the incremental per-slab sample evaluation and the moment-form
adjoint; ``mode="parity"`` the reference's per-sample arithmetic.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import _lib
from .engine import Engine, engine_for, make_gaussians, settings_struct


@dataclass
class BatchedViews:
    cameras: list
    white_background: bool = True
    supersampling: tuple = (1, 1)
    mode: str = "fast"
    max_prim_slice: int = 1024
    iteration: int = 0
    jitter: int = 0
    rnd_sample: int = 0
    update: bool = False
    sh_quirk: bool = True
    engine: Engine | None = None
    offsets: list = field(default_factory=list)

    def __post_init__(self):
        if not (1 <= len(self.cameras) <= _lib.MAX_VIEWS):
            raise ValueError(f"1..{_lib.MAX_VIEWS} views per launch")
        sx, sy = self.supersampling
        off = [0]
        for c in self.cameras:
            off.append(off[-1] + int(c.image_width) * sx * int(c.image_height) * sy)
        self.offsets = off

    @property
    def n_rays(self):
        return self.offsets[-1]

    def split(self, ray_colors):
        """Per-view (H, W, 3) images of a packed (R, 3) tensor."""
        sx, sy = self.supersampling
        out = []
        for v, c in enumerate(self.cameras):
            out.append(ray_colors[self.offsets[v]:self.offsets[v + 1]].reshape(int(c.image_height) * sy,
                                                                               int(c.image_width) * sx, 3))
        return out


def _st(views: BatchedViews):
    mode = {"parity": _lib.RG_MODE_PARITY, "fast": _lib.RG_MODE_FAST}[views.mode]
    return settings_struct(views.white_background, views.jitter, views.rnd_sample, views.max_prim_slice,
                           views.iteration, mode, views.sh_quirk)


class BatchedRenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, scales, quaternions, densities, color_features, sph_gauss_features,
                bandwidth_sharpness, lobe_axis, views: BatchedViews):
        eng = views.engine or engine_for(positions.device)
        nsg = 0 if sph_gauss_features is None or sph_gauss_features.numel() == 0 else sph_gauss_features.shape[2]
        g = make_gaussians(positions, scales, quaternions, densities, color_features,
                           sph_gauss_features if nsg else None, bandwidth_sharpness if nsg else None,
                           lobe_axis if nsg else None)
        cams_t, _, _ = eng.cameras(views.cameras, views.supersampling)
        ray_colors, _ = eng.render_forward(g, cams_t, len(views.cameras), views.n_rays, _st(views),
                                           refit=views.update)
        ctx.views, ctx.engine, ctx.generation, ctx.nsg = views, eng, eng.generation, nsg
        ctx.dtypes = (densities.dtype, color_features.dtype,
                      sph_gauss_features.dtype if sph_gauss_features is not None else None)
        ctx.save_for_backward(positions, scales, quaternions, densities, color_features, sph_gauss_features,
                              bandwidth_sharpness, lobe_axis, ray_colors.clone())
        return ray_colors

    @staticmethod
    def backward(ctx, dL):
        views, eng, nsg = ctx.views, ctx.engine, ctx.nsg
        (positions, scales, quats, densities, color_features, sg, kappa, axis, ray_colors) = ctx.saved_tensors
        g = make_gaussians(positions, scales, quats, densities, color_features, sg if nsg else None,
                           kappa if nsg else None, axis if nsg else None)
        cams_t, _, _ = eng.cameras(views.cameras, views.supersampling)
        n = len(views.cameras)
        if eng.generation != ctx.generation:
            eng.ellipsoids_bbox(g)
            eng.bvh_build()
            eng.forward_sh(g, cams_t, n)
        gr = eng.render_backward(g, cams_t, n, _st(views), ray_colors, dL.contiguous().float())
        dsg = gr.get("sph_gauss_features") if nsg else None
        dkap = gr.get("bandwidth_sharpness") if nsg else None
        dax = gr.get("lobe_axis") if nsg else None
        return (gr["positions"], gr["scales"], gr["quaternions"], gr["densities"].reshape(densities.shape),
                gr["color_features"], dsg, dkap, dax, None)


def render_views(params: dict, views: BatchedViews):
    """Convenience wrapper: params in the PointCloud.get_data layout (dict), returns packed ray colours."""
    return BatchedRenderFunction.apply(params["positions"], params["scales"], params["quaternions"],
                                       params["densities"], params["color_features"],
                                       params.get("sph_gauss_features"), params.get("bandwidth_sharpness"),
                                       params.get("lobe_axis"), views)


def render_views_inference(params: dict, views: BatchedViews, counts: bool = False):
    """Inference render of every view of ``views`` in one launch (the reference's cuda_test
    programs: no jitter or random sample offsets, slab queries not clipped at the scene-box exit).
    Returns packed ray colours and, with ``counts``, the Gaussians per ray (int32)."""
    eng = views.engine or engine_for(params["positions"].device)
    nsg = 0 if params.get("sph_gauss_features") is None else params["sph_gauss_features"].shape[2]
    g = make_gaussians(params["positions"], params["scales"], params["quaternions"], params["densities"],
                       params["color_features"], params.get("sph_gauss_features") if nsg else None,
                       params.get("bandwidth_sharpness") if nsg else None, params.get("lobe_axis") if nsg else None)
    cams_t, _, _ = eng.cameras(views.cameras, views.supersampling)
    with torch.no_grad():
        out, cnt = eng.render_inference(g, cams_t, len(views.cameras), views.n_rays, _st(views), refit=views.update,
                                        counts=counts)
    return (out, cnt) if counts else out
