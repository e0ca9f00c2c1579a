"""PLY loading on the device (rg_records_to_columns) against fixtures written and read by the
reference's scripts/ply.py, with the loaders' tensors restated from classes/point_cloud.py:298-495
and convertpth_to_ply.py (tests/golden/make_ply_golden.py).  Every value must be equal."""
import os

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu

PLY = os.path.join(ROOT, "tests", "golden", "ply")


@pytest.fixture(scope="module")
def expected():
    return dict(np.load(os.path.join(PLY, "expected.npz")))


def _eq(a, b, what):
    a = a.detach().cpu().numpy()
    assert a.shape == b.shape, (what, a.shape, b.shape)
    assert np.array_equal(a, b), (what, np.abs(a.astype(np.float64) - b).max())


def test_every_property_type_in_big_endian(cuda, expected):
    """int8 .. float64, big-endian, 26-byte unaligned records: FP32 columns equal the reference
    reader's values rounded to float."""
    from ray_gauss_b200.io import PlyVertices
    ply = PlyVertices(os.path.join(PLY, "mixed_big_endian.ply"), cuda)
    names = list(expected["mixed/names"])
    cols = ply.columns(names)
    torch.cuda.synchronize()
    for j, nm in enumerate(names):
        _eq(cols[:, j], expected[f"mixed/field/{nm}"].astype(np.float32), nm)


@pytest.mark.parametrize("tag, kw", [("rgb_full", {}), ("rgb_min", {"default_density": 0.7})])
def test_load_from_ply(cuda, expected, tag, kw):
    from ray_gauss_b200.io import load_from_ply
    out = load_from_ply(os.path.join(PLY, f"{tag}.ply"), 16, 2, kw.get("default_density", 1.0), cuda)
    p = out["params"]
    torch.cuda.synchronize()
    for k in ("positions", "densities", "rgb", "scales", "quaternions"):
        _eq(p[k], expected[f"{tag}/{k}"], k)
    n = p["positions"].shape[0]
    assert p["spherical_harmonics"].shape == (n, 3, 15) and not p["spherical_harmonics"].any()
    assert p["sph_gauss_features"].shape == (n, 3, 2) and p["lobe_axis"].shape == (n, 2, 3)
    f3d = torch.log(torch.full((n, 1), np.float32(0.0001), device=cuda))
    assert torch.equal(out["filter_3D"], f3d)


def test_load_from_gaussian_splatting(cuda, expected):
    from ray_gauss_b200.io import load_from_gaussian_splatting
    out = load_from_gaussian_splatting(os.path.join(PLY, "gs3d.ply"), cuda)
    torch.cuda.synchronize()
    for k in ("positions", "densities", "scales", "quaternions", "rgb", "spherical_harmonics"):
        _eq(out["params"][k], expected[f"gs3d/{k}"], k)
    assert out["harmonic_number"] == 16 and out["params"]["sph_gauss_features"].shape[2] == 0


def test_load_trained_ply_and_write_it_back(cuda, expected, tmp_path):
    from ray_gauss_b200.io import load_trained_ply, write_trained_ply
    out = load_trained_ply(os.path.join(PLY, "trained.ply"), cuda)
    torch.cuda.synchronize()
    for k, v in out["params"].items():
        _eq(v, expected[f"trained/{k}"], k)
    _eq(out["stats"]["xyz_gradient_accum_norm"], expected["trained/gradient_accum_norm"], "gradient_accum_norm")
    assert out["harmonic_number"] == 16 and out["num_sph_gauss"] == 2
    back = write_trained_ply(tmp_path / "back.ply", out["params"], 16, 2, out["stats"]["xyz_gradient_accum_norm"])
    assert open(back, "rb").read() == open(os.path.join(PLY, "trained.ply"), "rb").read()


def test_loaded_scene_renders(cuda, expected):
    """A loaded trained scene goes through the get_data activations into the renderer."""
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews, render_views
    from ray_gauss_b200.engine import Engine
    from ray_gauss_b200.io import load_trained_ply
    from ray_gauss_b200.train_tail import point_cloud_data
    out = load_trained_ply(os.path.join(PLY, "trained.ply"), cuda)
    X = point_cloud_data(out["params"])
    views = BatchedViews([S.sphere_camera(4.0, 32, 24, 50.0, seed=1, device=cuda)], engine=Engine(cuda.index or 0),
                         mode="parity", white_background=True)
    img = render_views(X, views)
    torch.cuda.synchronize()
    assert img.shape == (32 * 24, 3) and torch.isfinite(img).all()
