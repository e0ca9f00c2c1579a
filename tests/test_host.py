"""Host-side logic on the CPU: argument validation, camera records, settings, the drop-in
signatures and the replica timing reduction of bench.py over a gloo process group."""
import inspect
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import ROOT


def test_render_optix_settings_keeps_reference_signature():
    from ray_gauss_b200.optix_raycasting.render_optix import RenderOptixSettings
    # optix_raycasting/render_optix.py:67-71 of the reference
    ref = ["context", "update", "gas", "program_grps_fwd", "pipeline_fwd", "program_grps_bwd", "pipeline_bwd",
           "viewpoint_cam", "max_prim_slice", "num_sph_gauss", "iteration", "jitter", "rnd_sample", "supersampling",
           "white_background", "hit_prim_idx"]
    names = list(inspect.signature(RenderOptixSettings.__init__).parameters)[1:]
    assert names[: len(ref)] == ref
    s = RenderOptixSettings(*range(16))
    assert s.mode == "parity" and s.sh_quirk is True and s.hit_prim_idx == 15


def test_render_optix_function_arity():
    from ray_gauss_b200.optix_raycasting.render_optix import RenderOptixFunction
    params = list(inspect.signature(RenderOptixFunction.forward).parameters)
    assert params == ["ctx", "positions", "scales", "normalized_quaternions", "densities", "color_features",
                      "sph_gauss_features", "bandwidth_sharpness", "lobe_axis", "settings"]


def test_make_gaussians_validates_on_host():
    from ray_gauss_b200.engine import make_gaussians
    n = 4
    ok = dict(positions=torch.zeros(n, 3), scales=torch.ones(n, 3), quaternions=torch.zeros(n, 4),
              densities=torch.ones(n), color_features=torch.zeros(n, 3, 16))
    with pytest.raises(ValueError, match="CUDA"):
        make_gaussians(**ok)
    bad = dict(ok, color_features=torch.zeros(n, 3, 5))
    with pytest.raises(ValueError, match="1, 4, 9 or 16"):
        make_gaussians(**bad)
    bad = dict(ok, quaternions=torch.zeros(n, 3))
    with pytest.raises(ValueError):
        make_gaussians(**bad)
    with pytest.raises(ValueError, match="at most"):
        make_gaussians(**ok, sph_gauss_features=torch.zeros(n, 3, 17), bandwidth_sharpness=torch.zeros(n, 17),
                       lobe_axis=torch.zeros(n, 17, 3))


def test_camera_record_matches_reference_launch_parameters():
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.engine import camera_record
    cam = S.look_at_camera([1.0, -2.5, 0.7], [0, 0, 0], 64, 48, fovy=math.radians(50))
    r = camera_record(cam, supersampling=(2, 1))
    wvt = cam.world_view_transform.numpy()
    np.testing.assert_allclose(list(r.u), wvt[:3, 0], rtol=1e-6)
    np.testing.assert_allclose(list(r.v), wvt[:3, 1], rtol=1e-6)
    np.testing.assert_allclose(list(r.w), wvt[:3, 2], rtol=1e-6)
    np.testing.assert_allclose(list(r.eye), cam.camera_center.numpy(), rtol=1e-6)
    assert (r.width, r.height) == (128, 48)
    assert abs(r.tan_half_fovy - math.tan(math.radians(25))) < 1e-6
    # camera axes: right-handed x right, y down, z forward, z towards the target
    U, V, W = np.array(r.u), np.array(r.v), np.array(r.w)
    np.testing.assert_allclose(np.cross(U, V), W, atol=1e-6)
    fwd = -np.array(r.eye) / np.linalg.norm(r.eye)
    np.testing.assert_allclose(W, fwd, atol=1e-6)


def test_settings_struct_fields():
    from ray_gauss_b200 import _lib
    from ray_gauss_b200.engine import settings_struct
    s = settings_struct(white_background=False, jitter=1, rnd_sample=2, max_prim_slice=77, iteration=2 ** 33 + 5,
                        mode=_lib.RG_MODE_FAST, sh_quirk=False)
    assert (s.white_background, s.jitter, s.rnd_sample, s.max_prim_slice, s.iteration, s.mode, s.sh_quirk) == \
        (0, 1, 2, 77, 5, 1, 0)


def test_batched_views_offsets_and_split():
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews
    cams = [S.sphere_camera(3.0, w, h, 40.0, seed=k) for k, (w, h) in enumerate([(5, 3), (2, 7), (4, 4)])]
    v = BatchedViews(cams, supersampling=(1, 2))
    assert v.offsets == [0, 30, 58, 90]
    imgs = v.split(torch.arange(90 * 3, dtype=torch.float32).reshape(90, 3))
    assert [tuple(i.shape) for i in imgs] == [(6, 5, 3), (14, 2, 3), (8, 4, 3)]
    with pytest.raises(ValueError):
        BatchedViews([])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 10.0 + 5.0 * rank
    out[rank] = bench.max_over_ranks(ms, torch.device("cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_replica, args=(world, _free_port(), out), nprocs=world, join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_train_tail_rejects_bad_arguments_without_a_launch(engine_lib):
    """rg_train_tail_step validates its descriptor on the host: these return RG_ERR_INVALID_ARG (1)
    before any device work."""
    import ctypes

    from ray_gauss_b200 import _lib
    lib = engine_lib
    d = _lib.rg_train_tail()
    d.n_tensors = _lib.RG_TAIL_MAX_TENSORS + 1
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 1
    d = _lib.rg_train_tail()
    d.n, d.n_tensors = 10, 1
    d.idx_positions, d.idx_densities, d.idx_scales, d.idx_quaternions, d.idx_lobe_axis = 0, -1, -1, -1, -1
    d.tensors[0].param, d.tensors[0].width = 0x1000, 4          # positions must be 3 wide
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 1
    d.tensors[0].width, d.tensors[0].active = 3, 1              # active without moments
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 1
    d.tensors[0].exp_avg, d.tensors[0].exp_avg_sq = 0x2000, 0x3000
    d.tensors[0].bias1, d.tensors[0].bias2_sqrt = 0.0, 1.0      # bias correction of step 0
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 1
    d.idx_positions, d.idx_quaternions, d.normalize_quaternions = -1, 0, 1
    d.tensors[0].width, d.tensors[0].active, d.tensors[0].param = 4, 0, 0x1004   # unaligned quaternions
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 1
    d.n = 0
    d.tensors[0].param = 0x1000
    assert lib.rg_train_tail_step(ctypes.byref(d), None) == 0   # nothing to do


@pytest.mark.filterwarnings("ignore:Detected call of")
def test_lr_schedule_follows_optimizer_manager_logic():
    """The host-side schedule of the fused tail against torch's Adam + ExponentialLR driven by the
    reference's manager logic (classes/optimizer.py:13-21), on CPU tensors."""
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    s = LrSchedule.exponential(1e-2, 1e-4, decay=4, delay=2, donotuse=1)
    assert abs(s.gamma ** 4 - 1e-2) < 1e-12
    tail = FusedTrainTail.__new__(FusedTrainTail)
    tail.names, tail.betas = ["a"], (0.9, 0.999)
    tail.schedules, tail.lr = {"a": s}, {"a": s.lr}
    tail.manager_step, tail.adam_step = {"a": 0}, {"a": 0}
    p = torch.zeros(1, requires_grad=True)
    opt = torch.optim.Adam([p], lr=s.lr)
    sch = torch.optim.lr_scheduler.ExponentialLR(opt, gamma=s.gamma)
    for it in range(9):
        has = it != 4
        (_, use, lr, b1c, b2c), = tail._plan(lambda k: has)
        if it < s.donotuse:
            assert not use
            continue
        assert use == has
        assert abs(lr - opt.param_groups[0]["lr"]) <= 1e-15
        if has:
            t = tail.adam_step["a"]
            assert abs(b1c - (1 - 0.9 ** t)) < 1e-15 and abs(b2c - (1 - 0.999 ** t) ** 0.5) < 1e-15
        if s.delay <= it < s.delay + s.decay:
            sch.step()


def test_point_cloud_data_inverts_raw_from_render_inputs():
    """get_data activations (classes/point_cloud.py:689-739) on CPU tensors: the raw tensors made
    from render inputs give those inputs back; a zero lobe axis renders as (0, 0, 1)."""
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.train_tail import point_cloud_data, raw_from_render_inputs
    p, _, _ = S.workload("small_object", n=200, seed=2)
    g = torch.Generator().manual_seed(0)
    p["sph_gauss_features"] = torch.randn(200, 3, 2, generator=g)
    p["bandwidth_sharpness"] = torch.rand(200, 2, generator=g) * 3 + 0.2
    p["lobe_axis"] = torch.nn.functional.normalize(torch.randn(200, 2, 3, generator=g), dim=2)
    raw = raw_from_render_inputs(p)
    X = point_cloud_data(raw)
    for k in X:
        assert torch.allclose(X[k], p[k], rtol=2e-5, atol=1e-6), k
    raw["lobe_axis"][5, 1] = 0.0
    assert torch.equal(point_cloud_data(raw)["lobe_axis"][5, 1], torch.tensor([0.0, 0.0, 1.0]))


def test_densify_validates_on_the_host(engine_lib):
    """The densify entry points reject bad descriptors before any device work (RG_ERR_INVALID_ARG
    = 1), size their workspace, and plan an empty cloud without touching a device."""
    import ctypes

    from ray_gauss_b200 import _lib
    lib = engine_lib
    nb = ctypes.c_uint64()
    assert lib.rg_densify_workspace_bytes(1000, 0, ctypes.byref(nb)) == 1
    assert lib.rg_densify_workspace_bytes(1000, 2, ctypes.byref(nb)) == 0 and nb.value > 1000 * 28
    d = _lib.rg_densify()
    d.n, d.n_split = 10, 2
    assert lib.rg_densify_plan(ctypes.byref(d), None) == 1                 # no inputs, no workspace
    d.n = 0
    assert lib.rg_densify_plan(ctypes.byref(d), None) == 0 and d.planned == 1 and d.n_out == 0
    t = (_lib.rg_densify_tensor * 1)()
    t[0].width, t[0].kind = 2, _lib.RG_DENSIFY_POSITIONS                   # positions are 3 wide
    assert lib.rg_densify_apply(ctypes.byref(d), None, t, 1, None) == 1
    t[0].width, t[0].kind = 1, 9                                           # unknown kind
    assert lib.rg_densify_apply(ctypes.byref(d), None, t, 1, None) == 1
    t[0].kind = _lib.RG_DENSIFY_DENSITIES
    assert lib.rg_densify_apply(ctypes.byref(d), None, t, 1, None) == 0    # nothing to write
    d.planned = 0
    assert lib.rg_densify_apply(ctypes.byref(d), None, t, 1, None) == 1    # apply before plan


def test_filter3d_camera_table_and_validation(engine_lib):
    """The 3D filter's camera rows hold the reference's per-camera values rounded to float
    (classes/point_cloud.py:1170-1196), and the entry point rejects missing buffers on the host."""
    import ctypes

    import numpy as np

    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.filter3d import camera_table, fov2focal
    cams = S.ring_cameras(3, seed=1)
    table, focal = camera_table(cams)
    assert table.shape == (3, 20) and table.dtype == np.float32
    c = cams[1]
    wvt = c.world_view_transform.numpy()
    assert np.array_equal(table[1, :9], wvt[:3, :3].reshape(-1)) and np.array_equal(table[1, 9:12], wvt[3, :3])
    assert table[1, 12] == np.float32(fov2focal(c.FoVx, c.image_width))
    assert table[1, 17] == np.float32(c.image_width * 1.15) and table[1, 18] == np.float32(-0.15 * c.image_height)
    assert focal == max(max(fov2focal(k.FoVx, k.image_width), fov2focal(k.FoVy, k.image_height)) for k in cams)
    lib = engine_lib
    assert lib.rg_compute_3d_filter(None, 10, None, 0, ctypes.c_float(1.0), None, None, None, None) == 1
    assert lib.rg_compute_3d_filter(None, 0, None, 0, ctypes.c_float(1.0), None, None, None, None) == 0


def test_knn_validates_on_the_host(engine_lib):
    import ctypes
    lib = engine_lib
    nb = ctypes.c_uint64()
    assert lib.rg_knn_workspace_bytes(1000, ctypes.byref(nb)) == 0 and nb.value > 1000 * 16
    assert lib.rg_knn_workspace_bytes(-1, ctypes.byref(nb)) == 1
    assert lib.rg_knn_mean_dist(None, 10, None, None, None) == 1
    assert lib.rg_knn_mean_dist(None, 0, None, None, None) == 0


def test_schedules_from_the_reference_config():
    """configs/base.yml's optimisation section (values restated here) through the manager logic of
    utils/optim_utils.py:4-82: exponential schedules where `scheduler` is set, constant otherwise."""
    from types import SimpleNamespace as NS

    from ray_gauss_b200.train_tail import schedules_from_config
    def sec(sched, init, final, decay, delay=0, donotuse=0, **kw):
        return NS(scheduler=sched, init_lr=init, final_lr=final, decay_step=decay, delay_step=delay,
                  donotuse_steps=donotuse, **kw)
    cfg = NS(density=sec(True, 0.5, 0.0001, 30000), rgb=sec(False, 0.001, 0.001, 0),
             sh=sec(False, 0.00026, 0.00026, 0, donotuse=5), position=sec(True, 0.000017, 0.000001, 30000, 100),
             scale=sec(False, 0.0115, 0.0115, 0), quaternion=sec(False, 0.00022, 0.00022, 0),
             sph_gauss_features=sec(False, 0.00036, 0.00036, 0), bandwidth_sharpness=sec(True, 0.045, 0.0, 10, gamma=0.5),
             lobe_axis=sec(False, 0.003, 0.003, 0))
    s = schedules_from_config(cfg)
    assert set(s) == {"positions", "rgb", "spherical_harmonics", "densities", "scales", "quaternions",
                      "sph_gauss_features", "bandwidth_sharpness", "lobe_axis"}
    assert s["densities"].gamma == (0.0001 / 0.5) ** (1 / 30000) and s["densities"].decay == 30000
    assert s["positions"].delay == 100 and s["positions"].lr == 0.000017
    assert s["spherical_harmonics"].gamma == 1.0 and s["spherical_harmonics"].donotuse == 5
    assert s["bandwidth_sharpness"].gamma == 0.5
    assert schedules_from_config({"rgb": {"scheduler": False, "init_lr": 0.1}})["rgb"].lr == 0.1


def test_tail_extend_and_replace_keep_counters():
    """extend / replace rewrite the tensors and moments on the host side and keep the step counts
    and learning rates (the reference's _cat_tensor / _replace)."""
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule, reset_density, unlock_spherical_harmonics
    n = 10
    P = {"spherical_harmonics": torch.zeros(n, 3, 0), "densities": torch.arange(n, dtype=torch.float32)}
    tail = FusedTrainTail(P, {k: LrSchedule(0.1) for k in P}, roles={"densities": "densities"})
    tail.adam_step = {"spherical_harmonics": 3, "densities": 5}
    tail.exp_avg["densities"].fill_(1.0)
    sh = unlock_spherical_harmonics(tail, 9)
    assert sh.shape == (n, 3, 8) and tail.exp_avg["spherical_harmonics"].shape == (n, 3, 8)
    assert tail.adam_step["spherical_harmonics"] == 3
    d = reset_density(tail)
    assert float(d.max()) == 4.0 and float(tail.exp_avg["densities"].abs().sum()) == 0.0
    assert tail.adam_step["densities"] == 5 and tail.params["densities"] is d


def test_l1_ssim_loss_matches_the_reference_functions():
    """The training loss of scripts/train.py:110-112 (utils/loss_utils.py SSIM) against values and
    image gradients computed by the reference's own functions (tests/golden/make_loss_golden.py),
    on the CPU: equal to float rounding."""
    import numpy as np

    from ray_gauss_b200.losses import l1_loss, l1_ssim_loss, ssim
    d = np.load(os.path.join(ROOT, "tests", "golden", "loss", "loss_l1_ssim.npz"))
    for i in range(2):
        img = torch.from_numpy(d[f"img{i}"]).requires_grad_(True)
        gt = torch.from_numpy(d[f"gt{i}"])
        assert abs(l1_loss(img, gt).item() - float(d[f"l1_{i}"])) <= 1e-7
        assert abs(ssim(img, gt).item() - float(d[f"ssim{i}"])) <= 1e-7
        loss = l1_ssim_loss(img, gt)
        assert abs(loss.item() - float(d[f"loss{i}"])) <= 1e-7
        loss.backward()
        assert np.allclose(img.grad.numpy(), d[f"grad{i}"], rtol=1e-6, atol=1e-10)


def test_gpu_wrappers_refuse_host_tensors(tmp_path):
    """The kernels' Python entry points raise on CPU tensors instead of passing host pointers to
    the device."""
    from ray_gauss_b200.filter3d import compute_3D_filter
    from ray_gauss_b200.io import PlyVertices, write_ply
    from ray_gauss_b200.knn import dist_cuda2
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    with pytest.raises(ValueError, match="CUDA"):
        dist_cuda2(torch.zeros(8, 3))
    with pytest.raises(ValueError, match="CUDA"):
        compute_3D_filter(torch.zeros(8, 3), [])
    tail = FusedTrainTail({"a": torch.zeros(4, 3)}, {"a": LrSchedule(0.1)})
    tail.params["a"].grad = torch.ones(4, 3)
    with pytest.raises(ValueError, match="CUDA"):
        tail.step()
    path = write_ply(str(tmp_path / "p"), [np.zeros((3, 3), np.float32)], ["x", "y", "z"])
    with pytest.raises(ValueError, match="CUDA"):
        PlyVertices(path, "cpu")


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (host cores only) prints one JSON line with the contract keys and
    the reference-arm fields, on a tiny workload."""
    import json
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "20000",
                          "--views", "2", "--steps", "1", "--warmup", "3", "--cpu-rays", "16"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "cpu_baseline"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "Mrays/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
