"""A training loop in the shape of the reference's scripts/train.py:25-181, run entirely on the
engine's components: the get_data activations, render, the reference's L1 + SSIM loss and backward
captured with the fused
Adam / statistics / clamp tail in one CUDA graph (schedules from the reference's optimisation config),
the 3D filter refreshed every 5 iterations, densify and prune, SG lobes unlocked from zero width, the
density reset, and a checkpoint saved, reloaded and restored into a fresh tail.  Every change of
tensor storage is followed by GraphedStep.rebuild (LBVH rebuild and re-capture)."""
from types import SimpleNamespace as NS

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _config():
    def sec(sched, init, final=None, decay=0):
        return NS(scheduler=sched, init_lr=init, final_lr=final if final is not None else init, decay_step=decay,
                  delay_step=0, donotuse_steps=0)
    # the learning rates of configs/base.yml (training.optimization), density rate lowered for a short run
    return NS(density=sec(True, 0.05, 0.0001, 30000), rgb=sec(False, 0.001), sh=sec(False, 0.00026),
              position=sec(True, 0.000017, 0.000001, 30000), scale=sec(False, 0.0115),
              quaternion=sec(False, 0.00022), sph_gauss_features=sec(False, 0.00036),
              bandwidth_sharpness=sec(False, 0.045), lobe_axis=sec(False, 0.003))


def test_training_loop_through_every_component(cuda, tmp_path):
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews
    from ray_gauss_b200.densify import densify_and_prune
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.filter3d import compute_3D_filter
    from ray_gauss_b200.graph import GraphedStep
    from ray_gauss_b200.io import load_checkpoint, load_tail_state, save_checkpoint, tail_state_dict
    from ray_gauss_b200.train_tail import (FusedTrainTail, point_cloud_data, raw_from_render_inputs, reset_density,
                                           schedules_from_config, unlock_spherical_gaussians)
    p, _, white = S.workload("small_object", n=4000, seed=11)
    raw = {k: v.to(cuda).contiguous() for k, v in raw_from_render_inputs(p).items()}
    assert raw["sph_gauss_features"].shape[2] == 0                  # no SG lobe before the unlock
    cams = [S.sphere_camera(3.0, 48, 36, 40.0, seed=k, device=cuda) for k in range(3)]
    views = BatchedViews(cams, engine=Engine(cuda.index or 0), mode="fast", white_background=white)
    target = torch.rand((views.n_rays, 3), device=cuda, generator=torch.Generator(device=cuda).manual_seed(2))
    tail = FusedTrainTail(raw, schedules_from_config(_config()),
                          roles={"positions": "positions", "densities": "densities", "scales": "scales",
                                 "quaternions": "quaternions", "lobe_axis": "lobe_axis"},
                          normalize_quaternion=True, normalize_lobe_axis=True, max_scale=0.0)
    filt = compute_3D_filter(tail.params["positions"].detach(), cams)
    act = lambda r: point_cloud_data(r, normalized_quaternion=False, normalized_lobe_axis=False)  # noqa: E731
    step = GraphedStep(dict(tail.params), views, target, loss="l1_ssim", tail=tail, min_scale=filt, activation=act)
    losses, n0 = [], tail.n
    for it in range(1, 31):
        losses.append(step.replay())
        if it % 5 == 0:                                               # scripts/train.py:163-164
            filt.copy_(compute_3D_filter(tail.params["positions"].detach(), cams))
        if it == 10:                                                  # scripts/train.py:143-146
            thr = float(torch.quantile(tail.stats["xyz_gradient_accum_norm"] /
                                       tail.stats["num_accum"].clamp(min=1), 0.7))
            extent = float(torch.exp(tail.params["scales"].detach()).max()) * 60.0
            res = densify_and_prune(tail, filt, thr, 0.05, extent)
            assert res["n"] != n0 and res["n_clone"] + res["n_split"] > 0
            filt = res["filter_3D"]
            step.rebuild(dict(tail.params), tail=tail, min_scale=filt)
        if it == 15:                                                  # scripts/train.py:156-160
            unlock_spherical_gaussians(tail, 2, generator=torch.Generator(device=cuda).manual_seed(3))
            step.rebuild(dict(tail.params), tail=tail, min_scale=filt)
        if it == 20:                                                  # classes/point_cloud.py:1145-1149
            reset_density(tail)
            step.rebuild(dict(tail.params), tail=tail, min_scale=filt)
    torch.cuda.synchronize()
    loss = np.array([float(x) for x in losses])
    assert np.isfinite(loss).all() and loss[-5:].mean() < loss[:5].mean()
    assert tail.params["lobe_axis"].shape == (tail.n, 2, 3) and tail.adam_step["lobe_axis"] == 15
    assert tail.adam_step["positions"] == 30 and float(tail.params["densities"].detach().min()) >= 0.0
    assert float(tail.params["scales"].detach().max()) <= 0.0
    # checkpoint (save_model / restore_model) and a fresh tail restored from it
    path = tmp_path / "chkpnt30.pth"
    save_checkpoint(path, tail.params, 16, 2, tail.stats, tail_state_dict(tail), 30)
    c = load_checkpoint(path, cuda)
    assert c["iteration"] == 30 and c["num_sph_gauss"] == 2
    fresh = FusedTrainTail({k: v.clone() for k, v in c["params"].items()}, schedules_from_config(_config()))
    load_tail_state(fresh, c["optimizer_state"])
    for k in tail.names:
        assert torch.equal(fresh.params[k], tail.params[k].detach()), k
        assert torch.equal(fresh.exp_avg_sq[k], tail.exp_avg_sq[k]), k
        assert fresh.adam_step[k] == tail.adam_step[k] and fresh.lr[k] == tail.lr[k], k
