"""Fused training-step tail against the reference's tail in torch: one torch.optim.Adam per
tensor (eps 1e-15) driven by OptimizerManager's step logic with ExponentialLR
(classes/optimizer.py:4-21, 203-218), the statistics of classes/point_cloud.py:633-640 and the clamps
of scripts/train.py:166-181.  Tolerance: parameters and Adam moments within 2e-6 relative."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N = 5000
SHAPES = {"xyz": (3,), "rgb": (3,), "sh": (3, 15), "density": (), "scales": (3,), "quaternions": (4,),
          "sph_gauss_features": (3, 2), "bandwidth_sharpness": (2,), "lobe_axis": (2, 3)}
ROLES = {"positions": "xyz", "densities": "density", "scales": "scales", "quaternions": "quaternions",
         "lobe_axis": "lobe_axis"}


class _Manager:
    """The reference's OptimizerManager step logic around a torch Adam (classes/optimizer.py:13-21)."""

    def __init__(self, p, sched):
        self.opt = torch.optim.Adam([p], lr=sched.lr, eps=1e-15)
        self.sch = torch.optim.lr_scheduler.ExponentialLR(self.opt, gamma=sched.gamma) if sched.gamma != 1.0 else None
        self.sched, self.current = sched, 0

    def step(self):
        if self.current < self.sched.donotuse:
            self.current += 1
            return
        self.opt.step()
        if self.sch is not None and self.sched.delay <= self.current < self.sched.delay + self.sched.decay:
            self.sch.step()
        self.current += 1


def _reference_tail(params, mgrs, stats, min_scale, max_scale):
    with torch.no_grad():
        g = params["xyz"].grad
        nrm = torch.norm(g, dim=1)
        stats["xyz_gradient_accum_norm"] += nrm
        stats["num_accum"] += torch.where(nrm > 0, 1.0, 0.0)
        stats["num_accum_gnv"] += torch.where(nrm > 0, 1.0, 0.0)
    for m in mgrs.values():
        m.step()
    with torch.no_grad():
        params["density"][params["density"] < 0] = 0
        q = params["quaternions"]
        nq = torch.norm(q, dim=1)
        q[nq == 0] = torch.tensor([1.0, 0.0, 0.0, 0.0], device=q.device)
        q /= torch.norm(q, dim=1)[:, None]
        s = params["scales"]
        mask = s < min_scale.repeat(1, 3)
        s[mask] = min_scale.repeat(1, 3)[mask]
        s[s > max_scale] = max_scale


def test_fused_tail_matches_torch_adam_and_clamps(cuda):
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    gen = torch.Generator(device="cpu").manual_seed(3)
    init = {k: torch.randn((N,) + sh, generator=gen) * 0.5 for k, sh in SHAPES.items()}
    init["quaternions"][7] = 0.0                      # zero-norm quaternion -> (1,0,0,0)
    sched = {k: LrSchedule(1e-3 * (i + 1)) for i, k in enumerate(SHAPES)}
    sched["xyz"] = LrSchedule.exponential(1.6e-4, 1.6e-6, decay=3, delay=1)
    sched["sh"] = LrSchedule(2.5e-3, donotuse=2)
    mine = {k: v.clone().to(cuda).contiguous() for k, v in init.items()}
    ref = {k: v.clone().to(cuda).requires_grad_(True) for k, v in init.items()}
    tail = FusedTrainTail(mine, sched, roles=ROLES, normalize_quaternion=True, normalize_lobe_axis=False,
                          max_scale=0.5)
    mgrs = {k: _Manager(ref[k], sched[k]) for k in SHAPES}
    stats = {k: torch.zeros(N, device=cuda) for k in ("xyz_gradient_accum_norm", "num_accum", "num_accum_gnv")}
    min_scale = (torch.randn(N, 1, generator=gen) * 0.3 - 1.0).to(cuda)
    for it in range(6):
        grads = {k: torch.randn((N,) + sh, generator=gen).to(cuda) for k, sh in SHAPES.items()}
        grads["xyz"][: N // 3] = 0.0                  # invisible Gaussians: no statistic, moments decay
        if it == 3:
            grads["rgb"] = None                       # a tensor without a gradient this step
        for k in SHAPES:
            mine[k].grad = None if grads[k] is None else grads[k].clone()
            ref[k].grad = None if grads[k] is None else grads[k].clone()
        tail.step(min_scale=min_scale)
        _reference_tail(ref, mgrs, stats, min_scale, 0.5)
        torch.cuda.synchronize()
        for k in SHAPES:
            a, b = mine[k].detach().cpu().numpy(), ref[k].detach().cpu().numpy()
            assert np.allclose(a, b, rtol=2e-6, atol=2e-7), (it, k, np.abs(a - b).max())
            st = mgrs[k].opt.state.get(ref[k])
            if st:
                assert np.allclose(tail.exp_avg[k].cpu().numpy(), st["exp_avg"].cpu().numpy(), rtol=2e-6, atol=1e-9)
                assert np.allclose(tail.exp_avg_sq[k].cpu().numpy(), st["exp_avg_sq"].cpu().numpy(), rtol=2e-6,
                                   atol=1e-12)
            assert math.isclose(tail.lr[k], mgrs[k].opt.param_groups[0]["lr"], rel_tol=1e-12), (it, k)
        for k in stats:
            assert np.allclose(tail.stats[k].cpu().numpy(), stats[k].cpu().numpy(), rtol=1e-6, atol=1e-6), k
    assert float(mine["density"].min()) >= 0.0
    assert float(mine["scales"].max()) <= 0.5


def test_lobe_axes_and_unaligned_tensors(cuda):
    """Lobe-axis normalisation with a zero axis, and tensors whose storage is not 16-byte aligned
    (the kernel's scalar path) against the same torch reference."""
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    n = 777
    gen = torch.Generator(device="cpu").manual_seed(5)
    base = {"xyz": torch.randn(n, 3, generator=gen), "lobe_axis": torch.randn(n, 3, 3, generator=gen),
            "quaternions": torch.randn(n, 4, generator=gen), "scales": torch.randn(n, 3, generator=gen) - 1.0}
    base["lobe_axis"][11, 1] = 0.0
    dens = torch.randn(n + 1, generator=gen)
    sched = {k: LrSchedule(2e-3) for k in ("xyz", "lobe_axis", "quaternions", "scales", "density")}
    mine = {k: v.clone().to(cuda) for k, v in base.items()}
    dens_buf = dens.clone().to(cuda)
    mine["density"] = dens_buf[1:]                   # 4-byte offset: the unaligned path
    assert mine["density"].data_ptr() % 16 != 0
    ref = {k: v.clone().to(cuda).requires_grad_(True) for k, v in base.items()}
    ref["density"] = dens[1:].clone().to(cuda).requires_grad_(True)
    roles = {"positions": "xyz", "densities": "density", "scales": "scales", "quaternions": "quaternions",
             "lobe_axis": "lobe_axis"}
    tail = FusedTrainTail(mine, sched, roles=roles, normalize_lobe_axis=True, statistics=False)
    opts = {k: torch.optim.Adam([ref[k]], lr=2e-3, eps=1e-15) for k in ref}
    for it in range(3):
        for k in mine:
            g = torch.randn(mine[k].shape, generator=gen).to(cuda)
            mine[k].grad, ref[k].grad = g.clone(), g.clone()
        tail.step()
        for o in opts.values():
            o.step()
        with torch.no_grad():
            ref["density"][ref["density"] < 0] = 0
            q = ref["quaternions"]
            q /= torch.norm(q, dim=1)[:, None]
            ax = ref["lobe_axis"]
            ax[torch.norm(ax, dim=2) == 0] = torch.tensor([0.0, 0.0, 1.0], device=cuda)
            ax /= torch.norm(ax, dim=2)[:, :, None]
        torch.cuda.synchronize()
        for k in mine:
            a, b = mine[k].detach().cpu().numpy(), ref[k].detach().cpu().numpy()
            assert np.allclose(a, b, rtol=2e-6, atol=2e-7), (it, k, np.abs(a - b).max())
    assert float(dens_buf[0]) == float(dens[0])        # the element before the view is untouched


def test_graphed_step_with_tail_equals_eager_tail(cuda):
    """A whole training iteration in one graph: the reference's get_data activations on the raw
    tensors (log scales, rgb + SH, softplus bandwidths, normalised lobe axes), render, MSE, backward
    and the fused tail, its learning rates and bias corrections written before each replay.  It must
    update the raw tensors, moments and statistics exactly as the eager tail given the same gradients
    (the graph's own), with the log-scale clamp of scripts/train.py:176-179 active."""
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.graph import GraphedStep
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule, point_cloud_data, raw_from_render_inputs
    p, _, white = S.workload("small_object", n=3000, seed=5)
    gen = torch.Generator(device="cpu").manual_seed(9)
    n = p["positions"].shape[0]
    p["sph_gauss_features"] = 0.1 * torch.randn(n, 3, 2, generator=gen)        # two SG lobes per Gaussian
    p["bandwidth_sharpness"] = torch.rand(n, 2, generator=gen) * 4.0 + 0.5
    p["lobe_axis"] = torch.nn.functional.normalize(torch.randn(n, 2, 3, generator=gen), dim=2)
    raw = {k: v.to(cuda).contiguous() for k, v in raw_from_render_inputs(p).items()}
    X = point_cloud_data(raw)
    for k in ("positions", "quaternions", "densities", "color_features", "sph_gauss_features", "lobe_axis"):
        assert torch.allclose(X[k], p[k].to(cuda), rtol=1e-6, atol=1e-7), k
    for k in ("scales", "bandwidth_sharpness"):
        assert torch.allclose(X[k], p[k].to(cuda), rtol=1e-5), k
    cams = [S.sphere_camera(3.0, w, h, 40.0, seed=k, device=cuda) for k, (w, h) in enumerate(((48, 36), (33, 17)))]
    views = BatchedViews(cams, engine=Engine(cuda.index or 0), mode="fast", white_background=white)
    target = torch.rand((views.n_rays, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(0))
    trained = {k: v for k, v in raw.items() if v.numel()}
    sched = {k: LrSchedule(1e-3) for k in trained}
    sched["positions"] = LrSchedule.exponential(1.6e-4, 1.6e-6, decay=3, delay=1)
    sched["spherical_harmonics"] = LrSchedule(2.5e-3, donotuse=2)
    roles = {"positions": "positions", "densities": "densities", "scales": "scales", "quaternions": "quaternions"}
    log_s = raw["scales"]
    min_scale = torch.quantile(log_s.min(dim=1).values, 0.3).expand(log_s.shape[0]).contiguous()
    max_scale = float(torch.quantile(log_s.max(dim=1).values, 0.7))
    mirror = {k: v.clone() for k, v in trained.items()}
    tail_g = FusedTrainTail(trained, sched, roles=roles, max_scale=max_scale)
    tail_e = FusedTrainTail(mirror, sched, roles=roles, max_scale=max_scale)
    step = GraphedStep(raw, views, target, tail=tail_g, min_scale=min_scale,
                       activation=lambda r: point_cloud_data(r, normalized_quaternion=False))
    for k in trained:
        assert torch.equal(trained[k], mirror[k])       # capturing runs nothing
    for it in range(5):
        step.replay()
        tail_e.step(min_scale=min_scale, grads={k: step.grads[k] for k in trained})
        torch.cuda.synchronize()
        for k in trained:
            assert torch.isfinite(trained[k]).all(), (it, k)
            assert torch.equal(trained[k], mirror[k]), (it, k)
            assert torch.equal(tail_g.exp_avg[k], tail_e.exp_avg[k]), (it, k)
            assert torch.equal(tail_g.exp_avg_sq[k], tail_e.exp_avg_sq[k]), (it, k)
        for k in tail_g.stats:
            assert torch.equal(tail_g.stats[k], tail_e.stats[k]), (it, k)
        assert tail_g.current_lrs() == tail_e.current_lrs()
    assert float(tail_g.stats["num_accum"].max()) == 5.0
    s_now = trained["scales"].detach()
    assert float(s_now.min()) >= float(min_scale[0]) and float(s_now.max()) <= max_scale
    assert tail_g.adam_step["spherical_harmonics"] == 3 and tail_g.adam_step["positions"] == 5


def _cat_state(opt, ext, dim):
    """The reference's _cat_tensor (classes/optimizer.py:71-83) on a torch Adam."""
    group = opt.param_groups[0]
    p = group["params"][0]
    st = opt.state.get(p, None)
    with torch.no_grad():
        newp = torch.cat((p, ext), dim=dim).requires_grad_(True)
    if st is not None:
        st["exp_avg"] = torch.cat((st["exp_avg"], torch.zeros_like(ext)), dim=dim)
        st["exp_avg_sq"] = torch.cat((st["exp_avg_sq"], torch.zeros_like(ext)), dim=dim)
        del opt.state[p]
        opt.state[newp] = st
    group["params"][0] = newp
    return newp


def _replace_state(opt, new):
    """The reference's _replace (classes/optimizer.py:97-106)."""
    group = opt.param_groups[0]
    p = group["params"][0]
    st = opt.state.get(p, None)
    st["exp_avg"] = torch.zeros_like(new)
    st["exp_avg_sq"] = torch.zeros_like(new)
    del opt.state[p]
    group["params"][0] = new
    opt.state[new] = st
    return new


def test_unlocks_and_density_reset_follow_the_reference_state_surgery(cuda):
    """SH unlocked from zero width, two SG lobes unlocked (axes from the same generator), densities
    reset (classes/point_cloud.py:518-545, 1145-1149), interleaved with Adam steps: the fused tail
    against torch Adams whose state the reference's _cat_tensor / _replace rewrite."""
    from ray_gauss_b200.train_tail import (FusedTrainTail, LrSchedule, reset_density, unlock_spherical_gaussians,
                                           unlock_spherical_harmonics)
    n = 3000
    g = torch.Generator(device="cpu").manual_seed(8)
    init = {"positions": torch.randn(n, 3, generator=g), "rgb": torch.randn(n, 3, generator=g),
            "spherical_harmonics": torch.zeros(n, 3, 0), "densities": torch.rand(n, generator=g) * 6,
            "sph_gauss_features": torch.zeros(n, 3, 0), "bandwidth_sharpness": torch.zeros(n, 0),
            "lobe_axis": torch.zeros(n, 0, 3)}
    sched = {k: LrSchedule(1e-3 * (i + 1)) for i, k in enumerate(init)}
    mine = {k: v.clone().to(cuda).contiguous() for k, v in init.items()}
    tail = FusedTrainTail(mine, sched, roles={"positions": "positions", "densities": "densities",
                                              "lobe_axis": "lobe_axis"}, normalize_quaternion=False,
                          statistics=False)
    opts = {k: torch.optim.Adam([v.clone().to(cuda).requires_grad_(True)], lr=sched[k].lr, eps=1e-15)
            for k, v in init.items()}
    ref = lambda k: opts[k].param_groups[0]["params"][0]  # noqa: E731
    for it in range(6):
        if it == 2:
            unlock_spherical_harmonics(tail, 4)
            _cat_state(opts["spherical_harmonics"], torch.zeros(n, 3, 3, device=cuda), 2)
        if it == 3:
            unlock_spherical_gaussians(tail, 2, generator=torch.Generator(device=cuda).manual_seed(4))
            _cat_state(opts["sph_gauss_features"], torch.zeros(n, 3, 2, device=cuda), 2)
            _cat_state(opts["bandwidth_sharpness"], torch.zeros(n, 2, device=cuda), 1)
            axes = torch.randn((n, 2, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(4))
            _cat_state(opts["lobe_axis"], axes, 1)
        if it == 4:
            reset_density(tail)
            d = ref("densities").detach()
            _replace_state(opts["densities"], torch.min(d, torch.ones_like(d) * 4.0).contiguous().requires_grad_(True))
        grads = {}
        for k in init:
            shape = tuple(ref(k).shape)
            grads[k] = torch.randn(shape, generator=g).to(cuda) if ref(k).numel() else None
        for k in init:
            ref(k).grad = grads[k]
            tail.params[k].grad = None if grads[k] is None else grads[k].clone()
        tail.step()
        for o in opts.values():
            o.step()
        with torch.no_grad():
            ref("densities")[ref("densities") < 0] = 0
        torch.cuda.synchronize()
        for k in init:
            a, b = tail.params[k].detach(), ref(k).detach()
            assert a.shape == b.shape, (it, k)
            assert torch.allclose(a, b, rtol=2e-6, atol=2e-7), (it, k, (a - b).abs().max().item())
            st = opts[k].state.get(ref(k))
            if st and st["exp_avg"].numel():
                assert torch.allclose(tail.exp_avg_sq[k], st["exp_avg_sq"], rtol=2e-6, atol=1e-12), (it, k)
                assert tail.adam_step[k] == int(st["step"]), (it, k)
    assert tail.params["spherical_harmonics"].shape == (n, 3, 3) and tail.params["lobe_axis"].shape == (n, 2, 3)
    assert float(tail.params["densities"].max()) <= 4.0 + 1e-2
