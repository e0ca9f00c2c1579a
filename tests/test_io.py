"""Scene I/O host logic against fixtures written and read by the reference's scripts/ply.py
(tests/golden/make_ply_golden.py): header parsing, the record layout, byte-identical PLY writing and
the checkpoint tuple of save_model / restore_model (classes/point_cloud.py:922-958).  No device work."""
import os

import numpy as np
import pytest
import torch

from conftest import ROOT

PLY = os.path.join(ROOT, "tests", "golden", "ply")
FILES = {"rgb_full": "rgb_full.ply", "rgb_min": "rgb_min.ply", "gs3d": "gs3d.ply", "trained": "trained.ply",
         "mixed": "mixed_big_endian.ply"}


@pytest.fixture(scope="module")
def expected():
    return dict(np.load(os.path.join(PLY, "expected.npz")))


@pytest.mark.parametrize("tag", list(FILES))
def test_header_and_record_layout_match_the_reference_reader(expected, tag):
    from ray_gauss_b200.io import read_ply_header
    path = os.path.join(PLY, FILES[tag])
    h = read_ply_header(path)
    assert h.names == list(expected[f"{tag}/names"])
    assert h.big_endian == (tag == "mixed")
    assert h.record_bytes == h.numpy_dtype().itemsize
    assert os.path.getsize(path) == h.body_offset + h.n * h.record_bytes
    if f"{tag}/field/{h.names[0]}" in expected:
        with open(path, "rb") as f:
            f.seek(h.body_offset)
            rec = np.fromfile(f, dtype=h.numpy_dtype(), count=h.n)
        for nm in h.names:
            assert np.array_equal(rec[nm], expected[f"{tag}/field/{nm}"]), nm


def test_ascii_and_truncated_files_are_refused(tmp_path):
    from ray_gauss_b200.io import read_ply_header
    p = tmp_path / "a.ply"
    p.write_bytes(b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n1.0\n")
    with pytest.raises(ValueError, match="not binary"):
        read_ply_header(p)
    p.write_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\n")
    with pytest.raises(ValueError, match="end_header"):
        read_ply_header(p)


def test_writers_are_byte_identical_to_the_reference(expected, tmp_path):
    """write_ply (scripts/ply.py:169-269) on the RGB fixture's columns, and write_trained_ply on the
    trained fixture's tensors (convertpth_to_ply.py:60-117), give the reference's files."""
    from ray_gauss_b200.io import write_ply, write_trained_ply
    e = expected
    cols = [np.stack([e[f"rgb_full/field/{a}"] for a in "xyz"], 1),
            np.stack([e[f"rgb_full/field/{c}"] for c in ("red", "green", "blue")], 1),
            e["rgb_full/field/density"], np.stack([e[f"rgb_full/field/s{a}"] for a in "xyz"], 1),
            np.stack([e[f"rgb_full/field/q{a}"] for a in "xyzw"], 1)]
    out = write_ply(str(tmp_path / "rgb"), cols, list(e["rgb_full/names"]))
    assert open(out, "rb").read() == open(os.path.join(PLY, "rgb_full.ply"), "rb").read()
    P = {k: torch.from_numpy(e[f"trained/{k}"]) for k in ("positions", "rgb", "spherical_harmonics", "densities",
                                                           "scales", "quaternions", "sph_gauss_features",
                                                           "bandwidth_sharpness", "lobe_axis")}
    out = write_trained_ply(tmp_path / "t.ply", P, 16, 2, torch.from_numpy(e["trained/gradient_accum_norm"]))
    assert open(out, "rb").read() == open(os.path.join(PLY, "trained.ply"), "rb").read()


def test_checkpoint_tuple_and_optimizer_state_round_trip(tmp_path):
    """save_checkpoint writes save_model's 15-tuple (torch Adam state per manager name) and
    load_checkpoint / load_tail_state restore it as restore_model does."""
    from ray_gauss_b200.io import MANAGER_NAMES, load_checkpoint, load_tail_state, save_checkpoint, tail_state_dict
    from ray_gauss_b200.train_tail import FusedTrainTail, LrSchedule
    g = torch.Generator().manual_seed(0)
    n = 50
    P = {"positions": torch.randn(n, 3, generator=g), "rgb": torch.randn(n, 3, generator=g),
         "spherical_harmonics": torch.randn(n, 3, 3, generator=g), "densities": torch.rand(n, generator=g),
         "scales": torch.randn(n, 3, generator=g), "quaternions": torch.randn(n, 4, generator=g),
         "sph_gauss_features": torch.randn(n, 3, 1, generator=g), "bandwidth_sharpness": torch.randn(n, 1, generator=g),
         "lobe_axis": torch.randn(n, 1, 3, generator=g)}
    tail = FusedTrainTail({k: v.clone() for k, v in P.items()}, {k: LrSchedule(1e-3 * (i + 1)) for i, k in enumerate(P)})
    for i, k in enumerate(P):
        tail.exp_avg[k].normal_(generator=g)
        tail.exp_avg_sq[k].uniform_(generator=g)
        tail.adam_step[k] = 3 + i
        tail.lr[k] = 1e-4 * (i + 1)
    stats = {"xyz_gradient_accum_norm": torch.rand(n, generator=g), "num_accum": torch.rand(n, generator=g)}
    path = tmp_path / "chkpnt700.pth"
    save_checkpoint(path, P, 4, 1, stats, tail_state_dict(tail), 700)
    data = torch.load(path, weights_only=False)
    assert len(data) == 15 and data[0] == 4 and data[10] == 1 and data[14] == 700
    assert torch.equal(data[1], P["positions"]) and torch.equal(data[12], stats["num_accum"])
    st = data[13][MANAGER_NAMES["spherical_harmonics"]]
    assert float(st["state"][0]["step"]) == 5 and st["param_groups"][0]["eps"] == 1e-15
    # the state loads into torch's own Adam, as the reference's load_state_dict does
    opt = torch.optim.Adam([torch.zeros_like(P["rgb"], requires_grad=True)], lr=1.0, eps=1e-15)
    opt.load_state_dict(data[13]["rgb"])
    assert opt.param_groups[0]["lr"] == tail.lr["rgb"]
    c = load_checkpoint(path, device="cpu")
    assert c["iteration"] == 700 and c["harmonic_number"] == 4 and c["num_sph_gauss"] == 1
    assert all(torch.equal(c["params"][k], P[k]) for k in P)
    assert torch.equal(c["stats"]["num_accum_gnv"], torch.zeros(n)) and torch.equal(c["filter_3D"], torch.zeros(n, 1))
    fresh = FusedTrainTail({k: v.clone() for k, v in c["params"].items()}, {k: LrSchedule(1.0) for k in P})
    load_tail_state(fresh, c["optimizer_state"])
    for k in P:
        assert torch.equal(fresh.exp_avg[k], tail.exp_avg[k]) and torch.equal(fresh.exp_avg_sq[k], tail.exp_avg_sq[k])
        assert fresh.adam_step[k] == tail.adam_step[k] and fresh.lr[k] == tail.lr[k] and fresh.manager_step[k] == 0
