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
