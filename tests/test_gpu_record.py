"""Hit-list record and replay: the forward stores each warp chunk's leaf list and the backward of
the same launch replays it instead of traversing the BVH again.  The replayed backward must give
the gradients of the traversing backward, fall back to traversal for tiles whose record did not
fit, and never replay a record made for other cameras or settings."""
import pytest
import torch

from helpers import rel_l2

pytestmark = pytest.mark.gpu

KEYS = ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
        "bandwidth_sharpness", "lobe_axis")
SIZES = ((64, 48), (40, 30), (33, 17))


def _setup(dev, mode, n=3000, seed=3):
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews
    from ray_gauss_b200.engine import Engine
    p, _, white = S.workload("small_object", n=n, seed=seed)
    p["scales"] = p["scales"] * 2.0
    P = {k: v.to(dev).contiguous() for k, v in p.items()}
    cams = [S.sphere_camera(3.0, w, h, 40.0, seed=k, device=dev) for k, (w, h) in enumerate(SIZES)]
    eng = Engine(dev.index or 0)
    views = BatchedViews(cams, engine=eng, mode=mode, white_background=white)
    return P, views, eng


def _grads(P, views, target):
    from ray_gauss_b200.batched import BatchedRenderFunction
    Q = {k: v.detach().clone().requires_grad_(True) for k, v in P.items()}
    out = BatchedRenderFunction.apply(*(Q[k] for k in KEYS), views)
    torch.nn.functional.mse_loss(out, target).backward()
    return out.detach(), {k: Q[k].grad for k in KEYS if Q[k].grad is not None}


def _target(dev, n_rays):
    return torch.rand((n_rays, 3), device=dev, generator=torch.Generator(device=dev).manual_seed(0))


@pytest.mark.parametrize("mode", ["parity", "fast"])
def test_replayed_backward_matches_traversing_backward(cuda, mode):
    P, views, eng = _setup(cuda, mode)
    target = _target(cuda, views.n_rays)
    eng.set_tuning(record_hits=-1)
    eng.status(reset=True)
    out0, g0 = _grads(P, views, target)
    st0 = eng.status(reset=True)
    assert st0["replayed_chunks"] == 0
    eng.set_tuning(record_hits=1)
    out1, g1 = _grads(P, views, target)
    st1 = eng.status(reset=True)
    assert st1["replayed_chunks"] > 0 and st1["record_overflows"] == 0 and st1["record_words"] > 0
    assert torch.equal(out0, out1)
    # the replaying backward runs no traversal (multi-pass chunks aside)
    assert st1["traversals"] < st0["traversals"]
    assert st1["hit_pairs"] == st0["hit_pairs"] and st1["slabs"] == st0["slabs"]
    for k, g in g0.items():
        assert rel_l2(g1[k].cpu().numpy(), g.cpu().numpy()) <= 1e-5, k


def _low_level(eng, P, views, settings, dL, record):
    """bbox -> build -> colour -> forward -> backward through the engine's C-ABI steps."""
    from ray_gauss_b200.engine import make_gaussians
    g = make_gaussians(*(P[k] for k in KEYS))
    cams_t, _, _ = eng.cameras(views.cameras)
    n = len(views.cameras)
    eng.set_tuning(record_hits=1 if record else -1)
    eng.ellipsoids_bbox(g)
    eng.bvh_build()
    eng.forward_sh(g, cams_t, n)
    out = torch.empty((views.n_rays, 3), dtype=torch.float32, device=dL.device)
    eng.launch_forward(cams_t, n, settings, out)
    grads = eng.render_backward(g, cams_t, n, settings, out, dL)
    return out, grads, g, cams_t


def test_record_overflow_falls_back_to_traversal(cuda):
    from ray_gauss_b200.batched import _st
    from ray_gauss_b200.engine import Engine
    P, views, _ = _setup(cuda, "fast")
    R = views.n_rays
    dL = torch.randn((R, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(1))
    st = _st(views)
    eng = Engine(cuda.index or 0)
    # a record sized for R/64 rays: later tiles are not recorded, the arena fills up mid-launch
    eng.reserve(P["positions"].shape[0], len(views.cameras), R // 64)
    eng.status(reset=True)
    out1, g1, _, _ = _low_level(eng, P, views, st, dL, record=True)
    s1 = eng.status(reset=True)
    assert s1["record_overflows"] > 0 and s1["replayed_chunks"] > 0
    out0, g0, _, _ = _low_level(eng, P, views, st, dL, record=False)
    s0 = eng.status(reset=True)
    assert s0["replayed_chunks"] == 0
    assert torch.equal(out0, out1)
    for k, g in g0.items():
        assert rel_l2(g1[k].cpu().numpy(), g.cpu().numpy()) <= 1e-5, k


def test_record_of_other_settings_is_not_replayed(cuda):
    from ray_gauss_b200.batched import _st
    from ray_gauss_b200.engine import make_gaussians
    P, views, eng = _setup(cuda, "fast")
    R = views.n_rays
    dL = torch.randn((R, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(2))
    eng.reserve(P["positions"].shape[0], len(views.cameras), R)
    st_a = _st(views)
    out_a, g_ref, g, cams_t = _low_level(eng, P, views, st_a, dL, record=False)
    eng.set_tuning(record_hits=1)
    views.white_background = not views.white_background
    st_b = _st(views)
    out_b = torch.empty_like(out_a)
    eng.launch_forward(cams_t, len(views.cameras), st_b, out_b)    # the record now belongs to st_b
    eng.status(reset=True)
    g_a = eng.render_backward(g, cams_t, len(views.cameras), st_a, out_a, dL)
    assert eng.status(reset=True)["replayed_chunks"] == 0
    for k, v in g_ref.items():
        assert rel_l2(g_a[k].cpu().numpy(), v.cpu().numpy()) <= 1e-5, k
