"""Densify and prune (the reference's ``PointCloud.densify_and_prune``, classes/point_cloud.py:1068-1143)
on the engine's kernels: one classification + scan (``rg_densify_plan``, which reads the new size
back) and one gather that writes every trained tensor, both Adam moments, the statistics and
``filter_3D`` at the new size (``rg_densify_apply``).

The result is the reference's, row for row: surviving originals, then clones, then split copy 0 of
every split Gaussian, then copy 1; Adam moments move with kept rows and are zero for new rows
(classes/optimizer.py:54-83); ``xyz_gradient_accum_norm`` and ``num_accum`` restart at zero,
``num_accum_gnv`` keeps the old rows.  Split positions use standard normals drawn with
``torch.randn`` in the order of the reference's ``torch.normal(mean=0, std=exp(scales))``.

After it the LBVH must be rebuilt (render with ``update=False`` once; ``GraphedStep.rebuild``
re-captures with the new tensors).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check


def densify_and_prune(tail, filter_3D: torch.Tensor, grad_threshold: float, min_density: float, scene_extent: float,
                      n_split: int = 2, generator: torch.Generator | None = None,
                      normals: torch.Tensor | None = None) -> dict:
    """Densify and prune the Gaussians held by ``tail`` (a :class:`ray_gauss_b200.train_tail.FusedTrainTail`
    with the ``positions``, ``scales`` (log), ``quaternions`` and ``densities`` roles and its
    statistics).  The tail is rebound to the new tensors; returns
    ``{"params", "filter_3D", "n_clone", "n_split", "n_pruned", "n"}``.

    ``normals`` (optional, FP32 (n_split * selected, 3)) are the standard normals of the split
    samples, taken instead of drawing them with ``generator``: a caller that reproduces another
    run's random stream passes them (a wrong row count raises)."""
    roles = tail.roles
    for r in ("positions", "scales", "quaternions", "densities"):
        if r not in roles:
            raise ValueError(f"the tail needs the {r!r} role")
    if tail.stats is None:
        raise ValueError("the tail keeps no statistics")
    P = tail.params
    pos, ls, quat, dens = (P[roles[r]] for r in ("positions", "scales", "quaternions", "densities"))
    n = tail.n
    dev = pos.device
    if dev.type != "cuda":
        raise ValueError("densify_and_prune runs on CUDA tensors")
    lib = _lib.load()
    f3d = filter_3D.reshape(-1)
    if f3d.numel() != n or f3d.dtype != torch.float32 or not f3d.is_contiguous():
        raise ValueError("filter_3D: (N,) or (N, 1) FP32 contiguous")
    # the kernels launch on the current CUDA device: make it the tensors' device for the call
    with torch.cuda.device(dev):
        return _densify(tail, lib, P, roles, pos, ls, quat, dens, f3d, tuple(filter_3D.shape), n, dev,
                        grad_threshold, min_density, scene_extent, n_split, generator, normals)


def _densify(tail, lib, P, roles, pos, ls, quat, dens, f3d, f3d_shape, n, dev, grad_threshold, min_density,
             scene_extent, n_split, generator, normals):
    nbytes = ctypes.c_uint64()
    check(lib.rg_densify_workspace_bytes(n, n_split, ctypes.byref(nbytes)), None, "rg_densify_workspace_bytes")
    ws = torch.empty(int(nbytes.value), dtype=torch.uint8, device=dev)
    d = _lib.rg_densify()
    d.n = n
    d.grad_accum = tail.stats["xyz_gradient_accum_norm"].data_ptr()
    d.num_accum = tail.stats["num_accum"].data_ptr()
    d.log_scales, d.quaternions, d.densities = ls.data_ptr(), quat.data_ptr(), dens.data_ptr()
    # torch compares a float tensor with a Python number in float32; 0.01 * extent is a double product
    d.grad_threshold = float(np.float32(grad_threshold))
    d.scale_threshold = float(np.float32(0.01 * scene_extent))
    d.min_density = float(np.float32(min_density))
    # torch divides by a Python number as a multiplication by its float reciprocal
    d.split_scale_mul = float(np.float32(1.0) / np.float32(0.8 * n_split))
    d.n_split = n_split
    d.workspace = ws.data_ptr()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    check(lib.rg_densify_plan(ctypes.byref(d), stream), None, "rg_densify_plan")
    n_out, n_sel = int(d.n_out), int(d.n_split_sel)
    if normals is None:
        normals = torch.randn((n_split * n_sel, 3), device=dev, generator=generator) if n_sel else None
    else:
        if normals.shape != (n_split * n_sel, 3):
            raise ValueError(f"normals: expected ({n_split * n_sel}, 3) for {n_sel} split Gaussians, got "
                             f"{tuple(normals.shape)}")
        normals = normals.to(device=dev, dtype=torch.float32).contiguous() if n_sel else None

    new_p = {k: torch.empty((n_out,) + tuple(v.shape[1:]), dtype=v.dtype, device=dev) for k, v in P.items()}
    new_m = {k: torch.empty_like(new_p[k]) for k in P}
    new_v = {k: torch.empty_like(new_p[k]) for k in P}
    new_stats = {k: torch.empty(n_out, dtype=torch.float32, device=dev) for k in tail.stats}
    new_f3d = torch.empty((n_out,) + tuple(f3d_shape[1:]), dtype=torch.float32, device=dev)
    kind_of = {roles["positions"]: _lib.RG_DENSIFY_POSITIONS, roles["scales"]: _lib.RG_DENSIFY_LOG_SCALES,
               roles["densities"]: _lib.RG_DENSIFY_DENSITIES}
    items = []
    for k, v in P.items():
        w = int(v.numel() // max(1, n))
        if w == 0:
            continue
        items.append((v, new_p[k], w, kind_of.get(k, _lib.RG_DENSIFY_COPY)))
        items.append((tail.exp_avg[k], new_m[k], w, _lib.RG_DENSIFY_OLD_ONLY))
        items.append((tail.exp_avg_sq[k], new_v[k], w, _lib.RG_DENSIFY_OLD_ONLY))
    items.append((tail.stats["xyz_gradient_accum_norm"], new_stats["xyz_gradient_accum_norm"], 1, _lib.RG_DENSIFY_ZERO))
    items.append((tail.stats["num_accum"], new_stats["num_accum"], 1, _lib.RG_DENSIFY_ZERO))
    items.append((tail.stats["num_accum_gnv"], new_stats["num_accum_gnv"], 1, _lib.RG_DENSIFY_OLD_ONLY))
    items.append((f3d, new_f3d, 1, _lib.RG_DENSIFY_COPY))
    if len(items) > _lib.RG_DENSIFY_MAX_TENSORS:
        raise ValueError("too many tensors")
    arr = (_lib.rg_densify_tensor * max(1, len(items)))()
    for i, (src, dst, w, kind) in enumerate(items):
        if not src.is_contiguous() or src.dtype != torch.float32:
            raise ValueError("tensors must be FP32 and contiguous")
        arr[i].src, arr[i].dst, arr[i].width, arr[i].kind = src.data_ptr(), dst.data_ptr(), w, kind
    check(lib.rg_densify_apply(ctypes.byref(d), normals.data_ptr() if normals is not None else None, arr,
                               len(items), stream), None, "rg_densify_apply")
    # zero-width tensors (e.g. no SG lobes yet) have nothing to gather
    for k, v in P.items():
        if v.numel() == 0:
            new_m[k].zero_()
            new_v[k].zero_()
    for k in P:                               # leaves like the reference's concatenated tensors
        new_p[k].requires_grad_(P[k].requires_grad)
    tail.rebind(new_p, new_m, new_v, new_stats)
    # the density prune's count (the split originals are removed by the split itself)
    n_pruned = n + int(d.n_clone) + n_split * n_sel - n_sel - n_out
    return {"params": new_p, "filter_3D": new_f3d, "n_clone": int(d.n_clone), "n_split": n_sel,
            "n_pruned": n_pruned, "n": n_out}
