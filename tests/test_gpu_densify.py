"""Densify and prune against the reference's own densify_and_prune and optimizer-state surgery
(classes/point_cloud.py:497-516, 1034-1143; classes/optimizer.py:54-83, 151-164): fixtures that
tests/golden/make_densify_golden.py generates by running those functions on the CPU, fed with the
same standard normals; and, at sizes a fixture cannot hold (1.1M Gaussians), against the same
functions restated in torch (_RefCloud; build_rotation of utils/general_utils.py:466-487).

Every tensor must match row for row: exactly, except the positions and log scales of split copies
(a 3x3 product and a division by a Python number whose operation order inside torch is not
specified, and the CPU's exponential against the GPU's) within 1e-6 relative + 1e-6 absolute."""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

NAMES = ("positions", "rgb", "spherical_harmonics", "densities", "scales", "quaternions", "sph_gauss_features",
         "bandwidth_sharpness", "lobe_axis")
ROLES = {"positions": "positions", "densities": "densities", "scales": "scales", "quaternions": "quaternions"}


def _cloud(n, dev, seed=0, nsg=2):
    g = torch.Generator(device="cpu").manual_seed(seed)
    raw = {"positions": torch.randn(n, 3, generator=g), "rgb": torch.rand(n, 3, generator=g),
           "spherical_harmonics": 0.1 * torch.randn(n, 3, 15, generator=g),
           "densities": torch.rand(n, generator=g) * 3.5 - 0.5,
           "scales": torch.rand(n, 3, generator=g) * 5.0 - 6.0,
           "quaternions": torch.randn(n, 4, generator=g),
           "sph_gauss_features": torch.randn(n, 3, nsg, generator=g),
           "bandwidth_sharpness": torch.randn(n, nsg, generator=g),
           "lobe_axis": torch.randn(n, nsg, 3, generator=g)}
    m = {k: torch.randn(v.shape, generator=g) * 1e-3 for k, v in raw.items()}
    v = {k: torch.rand(v.shape, generator=g) * 1e-6 for k, v in raw.items()}
    num = torch.randint(0, 5, (n,), generator=g).float()
    accum = torch.rand(n, generator=g) * 2e-4 * num           # num == 0 -> 0 / 0 -> grad 0
    stats = {"xyz_gradient_accum_norm": accum, "num_accum": num,
             "num_accum_gnv": torch.randint(0, 9, (n,), generator=g).float()}
    f3d = torch.rand(n, 1, generator=g) * 2.0 - 7.0
    to = lambda d: {k: x.to(dev).contiguous() for k, x in d.items()}  # noqa: E731
    return to(raw), to(m), to(v), to(stats), f3d.to(dev)


def _build_rotation(r):
    norm = torch.sqrt(r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1] + r[:, 2] * r[:, 2] + r[:, 3] * r[:, 3])
    q = r / norm[:, None]
    R = torch.zeros((q.size(0), 3, 3), device=r.device)
    r, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - r * z)
    R[:, 0, 2] = 2 * (x * z + r * y)
    R[:, 1, 0] = 2 * (x * y + r * z)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - r * x)
    R[:, 2, 0] = 2 * (x * z - r * y)
    R[:, 2, 1] = 2 * (y * z + r * x)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


class _RefCloud:
    """The reference's point cloud state during densify_and_prune: parameters, Adam moments,
    statistics and filter_3D, with its postfix (cat) and prune operations."""

    def __init__(self, raw, m, v, stats, f3d):
        self.p = {k: x.clone() for k, x in raw.items()}
        self.m = {k: x.clone() for k, x in m.items()}
        self.v = {k: x.clone() for k, x in v.items()}
        self.s = {k: x.clone() for k, x in stats.items()}
        self.f3d = f3d.clone()

    def postfix(self, new, new_f3d):                    # densification_postfix + _cat_tensor
        for k in NAMES:
            self.m[k] = torch.cat((self.m[k], torch.zeros_like(new[k])))
            self.v[k] = torch.cat((self.v[k], torch.zeros_like(new[k])))
            self.p[k] = torch.cat((self.p[k], new[k]))
        n = self.p["positions"].shape[0]
        self.s["xyz_gradient_accum_norm"] = torch.zeros(n, device=self.f3d.device)
        self.s["num_accum"] = torch.zeros(n, device=self.f3d.device)
        self.s["num_accum_gnv"] = torch.cat((self.s["num_accum_gnv"],
                                             torch.zeros(len(new["positions"]), device=self.f3d.device)))
        self.f3d = torch.cat((self.f3d, new_f3d))

    def prune(self, mask):                              # prune_points + _prune_optimizer
        keep = ~mask
        for d in (self.p, self.m, self.v, self.s):
            for k in d:
                d[k] = d[k][keep]
        self.f3d = self.f3d[keep]

    def densify_and_prune(self, max_grad, min_density, extent, n_split, gen):
        grads = self.s["xyz_gradient_accum_norm"] / self.s["num_accum"]
        grads[grads.isnan()] = 0.0
        # clone
        sel = torch.where(grads >= max_grad, True, False)
        sel = torch.logical_and(sel, torch.max(torch.exp(self.p["scales"]), dim=1).values <= 0.01 * extent)
        self.p["densities"][sel] = self.p["densities"][sel] / 2
        self.postfix({k: self.p[k][sel] for k in NAMES}, self.f3d[sel])
        n_clone = int(sel.sum())
        # split
        n_init = self.p["positions"].shape[0]
        padded = torch.zeros(n_init, device=grads.device)
        padded[: grads.shape[0]] = grads.squeeze()
        sel = torch.where(padded >= max_grad, True, False)
        sel = torch.logical_and(sel, torch.max(torch.exp(self.p["scales"]), dim=1).values > 0.01 * extent)
        stds = torch.exp(self.p["scales"])[sel].repeat(n_split, 1)
        samples = torch.normal(mean=torch.zeros((stds.size(0), 3), device=stds.device), std=stds, generator=gen)
        rots = _build_rotation(self.p["quaternions"][sel]).repeat(n_split, 1, 1)
        new = {"positions": torch.bmm(rots, samples.unsqueeze(-1)).squeeze(-1) +
               self.p["positions"][sel].repeat(n_split, 1),
               "scales": torch.log(torch.exp(self.p["scales"])[sel].repeat(n_split, 1) / (0.8 * n_split)),
               "densities": self.p["densities"][sel].repeat(n_split) / 2}
        for k in NAMES:
            if k not in new:
                x = self.p[k][sel]
                new[k] = x.repeat(n_split, *([1] * (x.dim() - 1)))
        self.postfix(new, self.f3d[sel].repeat(n_split, 1))
        n_sel = int(sel.sum())
        self.prune(torch.cat((sel, torch.zeros(n_split * n_sel, device=sel.device, dtype=bool))))
        # prune
        self.prune((self.p["densities"] <= min_density).squeeze())
        return n_clone, n_sel


def _run(n, dev, max_grad, min_density, extent, n_split=2, seed=0):
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    raw, m, v, stats, f3d = _cloud(n, dev, seed)
    ref = _RefCloud(raw, m, v, stats, f3d)
    n_clone, n_sel = ref.densify_and_prune(max_grad, min_density, extent, n_split,
                                           torch.Generator(device=dev).manual_seed(11))
    params = {k: raw[k].clone() for k in NAMES}
    tail = FusedTrainTail(params, {k: LrSchedule(1e-3) for k in NAMES}, roles=ROLES)
    tail.adam_step = {k: 7 for k in NAMES}
    for k in NAMES:
        tail.exp_avg[k].copy_(m[k])
        tail.exp_avg_sq[k].copy_(v[k])
    for k in stats:
        tail.stats[k].copy_(stats[k])
    out = densify_and_prune(tail, f3d.clone(), max_grad, min_density, extent, n_split=n_split,
                            generator=torch.Generator(device=dev).manual_seed(11))
    torch.cuda.synchronize()
    return ref, tail, out, n_clone, n_sel


def _compare(ref, tail, out, n_clone, n_sel, n_split):
    n_out = ref.p["positions"].shape[0]
    assert out["n"] == n_out and out["n_clone"] == n_clone and out["n_split"] == n_sel
    assert tail.n == n_out and all(tail.adam_step[k] == 7 for k in NAMES)
    split_rows = torch.zeros(n_out, dtype=torch.bool, device=ref.f3d.device)
    for k in NAMES:
        a, b = tail.params[k], ref.p[k]
        assert a.shape == b.shape, k
        if k in ("positions", "scales"):
            assert torch.allclose(a, b, rtol=1e-6, atol=1e-6), (k, (a - b).abs().max().item())
            exact = (a == b).all(dim=1) if a.numel() else torch.ones(0, dtype=torch.bool, device=a.device)
            split_rows |= ~exact
        else:
            assert torch.equal(a, b), k
        assert torch.equal(tail.exp_avg[k], ref.m[k]), k
        assert torch.equal(tail.exp_avg_sq[k], ref.v[k]), k
    for k in ref.s:
        assert torch.equal(tail.stats[k], ref.s[k]), k
    assert torch.equal(out["filter_3D"], ref.f3d)
    # only split copies may differ from the restatement in the last bits
    new_rows = (ref.m["positions"] == 0).all(dim=1)
    assert not bool((split_rows & ~new_rows).any())


@pytest.mark.parametrize("n", [20_000, 1_100_000])
def test_densify_and_prune_matches_reference(cuda, n):
    """Clones, splits and prunes all occur; 1.1M Gaussians span more than 1024 scan blocks."""
    ref, tail, out, n_clone, n_sel = _run(n, cuda, max_grad=1e-4, min_density=0.1, extent=1.0)
    assert n_clone > 0 and n_sel > 0 and out["n_pruned"] > 0
    _compare(ref, tail, out, n_clone, n_sel, 2)


def test_densify_three_way_split_and_nothing_selected(cuda):
    ref, tail, out, n_clone, n_sel = _run(5000, cuda, max_grad=1e-4, min_density=0.1, extent=1.0, n_split=3, seed=2)
    assert n_sel > 0
    _compare(ref, tail, out, n_clone, n_sel, 3)
    ref, tail, out, n_clone, n_sel = _run(3000, cuda, max_grad=1e9, min_density=-1e9, extent=1.0, seed=3)
    assert n_clone == 0 and n_sel == 0 and out["n"] == 3000
    _compare(ref, tail, out, n_clone, n_sel, 2)


def test_densify_prunes_everything(cuda):
    ref, tail, out, n_clone, n_sel = _run(2500, cuda, max_grad=1e-4, min_density=1e9, extent=1.0, seed=4)
    assert out["n"] == 0 and ref.p["positions"].shape[0] == 0
    assert all(v.shape[0] == 0 for v in tail.params.values())


def test_graphed_step_recaptured_after_densify(cuda):
    """Train a few captured iterations, densify (the tail's moments and counters carry over),
    rebuild the LBVH and re-capture, and keep training at the new size."""
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.graph import GraphedStep
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule, point_cloud_data, raw_from_render_inputs
    p, _, white = S.workload("small_object", n=4000, seed=6)
    raw = {k: x.to(cuda).contiguous() for k, x in raw_from_render_inputs(p).items()}
    cams = [S.sphere_camera(3.0, 40, 30, 40.0, seed=k, device=cuda) for k in range(2)]
    views = BatchedViews(cams, engine=Engine(cuda.index or 0), mode="fast", white_background=white)
    target = torch.rand((views.n_rays, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(0))
    trained = {k: x for k, x in raw.items() if x.numel()}
    tail = FusedTrainTail(trained, {k: LrSchedule(1e-3) for k in trained}, roles=ROLES)
    f3d = torch.full((raw["positions"].shape[0], 1), -9.0, device=cuda)
    act = lambda r: point_cloud_data(r, normalized_quaternion=False)  # noqa: E731
    step = GraphedStep(raw, views, target, tail=tail, min_scale=f3d, activation=act)
    for _ in range(3):
        step.replay()
    torch.cuda.synchronize()
    n0 = tail.n
    thr = float(torch.quantile(tail.stats["xyz_gradient_accum_norm"] / tail.stats["num_accum"].clamp(min=1), 0.8))
    res = densify_and_prune(tail, f3d, thr, 0.05, scene_extent=float(torch.exp(raw["scales"].detach()).max()) * 50.0)
    assert res["n_clone"] > 0 and tail.n == res["n"] != n0
    new_raw = dict(res["params"])
    for k in raw:
        if k not in new_raw:
            new_raw[k] = raw[k].new_zeros((res["n"],) + tuple(raw[k].shape[1:]))
    step.rebuild(new_raw, tail=tail, min_scale=res["filter_3D"])
    for _ in range(3):
        loss = step.replay()
    torch.cuda.synchronize()
    assert np.isfinite(float(loss)) and all(int(tail.adam_step[k]) == 6 for k in tail.names)
    assert all(torch.isfinite(x).all() for x in tail.params.values())
    assert float(tail.stats["num_accum"].max()) <= 3.0


def test_densify_with_zero_width_sg_tensors_in_the_tail(cuda):
    """SG tensors held at zero width (no lobe unlocked yet) pass through densification with their
    new row count, and the tail keeps stepping afterwards."""
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    raw, m, v, stats, f3d = _cloud(4000, cuda, seed=9, nsg=0)
    tail = FusedTrainTail({k: raw[k].clone() for k in NAMES}, {k: LrSchedule(1e-3) for k in NAMES}, roles=ROLES)
    for k in stats:
        tail.stats[k].copy_(stats[k])
    out = densify_and_prune(tail, f3d.clone(), 1e-4, 0.1, 1.0)
    torch.cuda.synchronize()
    n = out["n"]
    assert out["n_clone"] > 0 and out["n_split"] > 0
    assert tail.params["sph_gauss_features"].shape == (n, 3, 0) and tail.params["lobe_axis"].shape == (n, 0, 3)
    assert tail.exp_avg["bandwidth_sharpness"].shape == (n, 0)
    for k in NAMES:
        tail.params[k].grad = torch.ones_like(tail.params[k])
    tail.step(min_scale=out["filter_3D"])
    torch.cuda.synchronize()
    assert all(torch.isfinite(x).all() for x in tail.params.values())


@pytest.mark.parametrize("case", ["mixed", "sg8_extent"])
def test_densify_matches_the_reference_functions(cuda, case):
    """Inputs, normals and outputs of the reference's PointCloud.densify_and_prune with its Adam
    optimizers (three real steps taken before), including rows whose mean gradient is infinite."""
    from conftest import GOLDEN
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    z = np.load(os.path.join(GOLDEN, "densify", case + ".npz"))
    t = lambda a: torch.tensor(np.ascontiguousarray(a), device=cuda)  # noqa: E731
    tail = FusedTrainTail({k: t(z[f"in/{k}"]) for k in NAMES}, {k: LrSchedule(1e-3) for k in NAMES}, roles=ROLES)
    tail.adam_step = {k: int(z[f"in_step/{k}"]) for k in NAMES}
    for k in NAMES:
        tail.exp_avg[k].copy_(t(z[f"in_m/{k}"]))
        tail.exp_avg_sq[k].copy_(t(z[f"in_v/{k}"]))
    for k in tail.stats:
        tail.stats[k].copy_(t(z[f"in_stat/{k}"]))
    out = densify_and_prune(tail, t(z["in_filter_3D"]), float(z["max_grad"]), float(z["min_density"]),
                            float(z["extent"]), n_split=int(z["n_split"]), normals=t(z["normals"]))
    torch.cuda.synchronize()
    n_out = z["out/positions"].shape[0]
    assert out["n"] == n_out and out["n_split"] * int(z["n_split"]) == z["normals"].shape[0]
    for k in NAMES:
        a, b = tail.params[k], t(z[f"out/{k}"])
        assert a.shape == b.shape, k
        if k in ("positions", "scales"):
            assert torch.allclose(a, b, rtol=1e-6, atol=1e-6), (k, (a - b).abs().max().item())
        else:
            assert torch.equal(a, b), k
        assert torch.equal(tail.exp_avg[k], t(z[f"out_m/{k}"])), k
        assert torch.equal(tail.exp_avg_sq[k], t(z[f"out_v/{k}"])), k
        assert int(tail.adam_step[k]) == int(z[f"out_step/{k}"]), k
    for k in tail.stats:
        assert torch.equal(tail.stats[k], t(z[f"out_stat/{k}"])), k
    assert torch.equal(out["filter_3D"], t(z["out_filter_3D"]))


def test_densify_rejects_normals_of_the_wrong_size(cuda):
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    raw, m, v, stats, f3d = _cloud(3000, cuda, seed=5)
    tail = FusedTrainTail({k: raw[k].clone() for k in NAMES}, {k: LrSchedule(1e-3) for k in NAMES}, roles=ROLES)
    for k in stats:
        tail.stats[k].copy_(stats[k])
    with pytest.raises(ValueError, match="normals"):
        densify_and_prune(tail, f3d.clone(), 1e-4, 0.1, 1.0, normals=torch.zeros((1, 3), device=cuda))
