"""rg_render_forward_noalloc: the allocation-free forward render for callers that cannot call
cudaMalloc (allocation-free graph capture, fixed device-memory budgets, plugins that must not touch
the process allocator).  Its scratch is a static device array shared by all calls; this checks,
through the C ABI, that two calls in a row give the image of the allocating entry point
(rg_render_forward through the engine), that its device counters can be read back
(rg_noalloc_get_status) and that oversize requests are refused.

Collected last (file name) so a run that stops at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-4


def _scene(dev, n=6000, seed=2):
    from ray_gauss_b200 import synthetic as S
    p, _, white = S.workload("small_object", n=n, seed=seed)
    p["scales"] = p["scales"] * 2.0
    return {k: v.to(dev) for k, v in p.items()}, white


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_forward_matches_allocating_entry_point(cuda, mode):
    from ray_gauss_b200 import _lib, synthetic as S
    from ray_gauss_b200.engine import Engine, make_gaussians, settings_struct
    lib = _lib.load()
    P, white = _scene(cuda)
    cams = [S.sphere_camera(3.0, 64, 48, 40.0, seed=k, device=cuda) for k in range(2)]
    g = make_gaussians(P["positions"], P["scales"], P["quaternions"], P["densities"], P["color_features"])
    st = settings_struct(white, mode=mode)
    eng = Engine(cuda.index or 0)
    cams_t, recs, _ = eng.cameras(cams)
    n_rays = sum(r.width * r.height for r in recs)
    ref, ref_T = eng.render_forward(g, cams_t, len(cams), n_rays, st, final_T=True)
    torch.cuda.synchronize()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        out = torch.full((n_rays, 3), -1.0, device=cuda)
        out_T = torch.full((n_rays,), -1.0, device=cuda)
        rc = lib.rg_render_forward_noalloc(ctypes.byref(g.struct), ctypes.c_void_p(cams_t.data_ptr()), len(cams),
                                           ctypes.byref(st), ctypes.c_void_p(out.data_ptr()),
                                           ctypes.c_void_p(out_T.data_ptr()), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.abs(out.cpu().numpy() - ref.cpu().numpy()).max() <= IMG_TOL
        assert np.abs(out_T.cpu().numpy() - ref_T.cpu().numpy()).max() <= IMG_TOL


def test_noalloc_refuses_oversize_requests(cuda):
    from ray_gauss_b200 import _lib, synthetic as S
    from ray_gauss_b200.engine import make_gaussians, settings_struct, Engine
    lib = _lib.load()
    P, white = _scene(cuda, n=16385)
    g = make_gaussians(P["positions"], P["scales"], P["quaternions"], P["densities"], P["color_features"])
    st = settings_struct(white)
    cams_t, recs, _ = Engine(cuda.index or 0).cameras([S.sphere_camera(3.0, 8, 8, 40.0, device=cuda)])
    out = torch.empty((64, 3), device=cuda)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.rg_render_forward_noalloc(ctypes.byref(g.struct), ctypes.c_void_p(cams_t.data_ptr()), 1,
                                       ctypes.byref(st), ctypes.c_void_p(out.data_ptr()), None, stream)
    assert rc == 5  # RG_ERR_CAPACITY: more than 16384 Gaussians
    P, white = _scene(cuda, n=500)
    g = make_gaussians(P["positions"], P["scales"], P["quaternions"], P["densities"], P["color_features"])
    rc = lib.rg_render_forward_noalloc(ctypes.byref(g.struct), ctypes.c_void_p(cams_t.data_ptr()), 5,
                                       ctypes.byref(st), ctypes.c_void_p(out.data_ptr()), None, stream)
    assert rc == 5  # more than 4 views


def _noalloc_status(lib, stream):
    from ray_gauss_b200 import _lib
    st = _lib.rg_status()
    assert lib.rg_noalloc_get_status(ctypes.byref(st), stream) == 0
    return {k: int(getattr(st, k)) for k, _ in _lib.rg_status._fields_}


def test_noalloc_status_reports_each_call(cuda):
    """The counters of the latest call: a non-finite Gaussian is counted (and skipped), and the
    next call with finite inputs starts from zero."""
    from ray_gauss_b200 import _lib, synthetic as S
    from ray_gauss_b200.engine import Engine, make_gaussians, settings_struct
    lib = _lib.load()
    P, white = _scene(cuda, n=3000, seed=4)
    cams_t, recs, _ = Engine(cuda.index or 0).cameras([S.sphere_camera(3.0, 40, 32, 40.0, seed=1, device=cuda)])
    n_rays = recs[0].width * recs[0].height
    st = settings_struct(white, mode=1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.empty((n_rays, 3), device=cuda)
    bad = P["positions"].clone()
    bad[7, 2] = float("nan")
    for pos, n_bad in ((bad, 1), (P["positions"], 0)):
        g = make_gaussians(pos, P["scales"], P["quaternions"], P["densities"], P["color_features"])
        rc = lib.rg_render_forward_noalloc(ctypes.byref(g.struct), ctypes.c_void_p(cams_t.data_ptr()), 1,
                                           ctypes.byref(st), ctypes.c_void_p(out.data_ptr()), None, stream)
        assert rc == 0
        s = _noalloc_status(lib, stream)
        assert s["nonfinite_inputs"] == n_bad
        assert s["slabs"] > 0 and s["hit_pairs"] > 0
        assert s["watchdog_trips"] == 0 and s["stack_overflows"] == 0 and s["record_words"] == 0
        assert torch.isfinite(out).all()
