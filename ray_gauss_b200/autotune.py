"""Autotuner for the render kernels: picks the longest chunk (slabs per traversal), the warp hit-list
capacity and the resident CTAs per SM by timing forward+backward on the caller's own scene and
views with CUDA events, then leaves the winner set on the engine.

The search is small (a few dozen launches): chunk lengths {16, 32, 64, 128, 255} x list capacity
{64, 128} x CTAs/SM {occupancy limit, 2}; ties are broken towards the default.  Results are cached
per (engine, scene size, views, arithmetic) so repeated calls cost nothing.
"""
from __future__ import annotations

import itertools

import torch

from .batched import BatchedRenderFunction, BatchedViews

_KEYS = ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
         "bandwidth_sharpness", "lobe_axis")
_CACHE: dict = {}


def _time_step(params, views, target, repeats):
    P = {k: v.detach().requires_grad_(True) for k, v in params.items() if v is not None}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    best = float("inf")
    for r in range(repeats + 1):
        ev[0].record()
        out = BatchedRenderFunction.apply(*(P.get(k) for k in _KEYS), views)
        loss = torch.nn.functional.mse_loss(out, target)
        loss.backward()
        ev[1].record()
        torch.cuda.synchronize()
        if r > 0:
            best = min(best, ev[0].elapsed_time(ev[1]))
        for v in P.values():
            v.grad = None
    return best


def autotune(params: dict, views: BatchedViews, target: torch.Tensor | None = None, repeats: int = 1,
             chunks=(16, 32, 64, 128, 255), capacities=(64, 128), ctas=(0, 2), verbose=False):
    """Time the candidate tunings on (params, views); set and return the fastest."""
    eng = views.engine
    if eng is None:
        from .engine import engine_for
        eng = engine_for(params["positions"].device)
        views.engine = eng
    n = params["positions"].shape[0]
    key = (id(eng), n, tuple((c.image_width, c.image_height) for c in views.cameras), views.mode)
    if key in _CACHE:
        eng.set_tuning(**_CACHE[key])
        return dict(_CACHE[key])
    if target is None:
        target = torch.zeros((views.n_rays, 3), device=params["positions"].device)
    default = eng.get_tuning()
    results = []
    for chunk, cap, cta in itertools.product(chunks, capacities, ctas):
        eng.set_tuning(chunk_slabs=chunk, list_capacity=cap, blocks_per_sm=cta)
        ms = _time_step(params, views, target, repeats)
        results.append((ms, (chunk, cap, cta)))
        if verbose:
            print(f"autotune chunk={chunk} capacity={cap} ctas/SM={cta or 'max'}: {ms:.2f} ms")
    results.sort(key=lambda r: (r[0], r[1] != (default["chunk_slabs"], default["list_capacity"], 0)))
    chunk, cap, cta = results[0][1]
    best = dict(chunk_slabs=chunk, list_capacity=cap, blocks_per_sm=cta)
    eng.set_tuning(**best)
    _CACHE[key] = best
    return dict(best, ms=results[0][0])
