"""Inference render (the reference's optix_utils.launch_pipeline_test with its cuda_test programs):
the engine against fixtures produced by those programs on the CPU.

Tolerances as for the training forward: parity arithmetic image max-abs <= 1e-4 and Gaussians per
ray equal; fast arithmetic image max-abs <= 1e-3 and per-ray counts at least the reference's (the
fast lists keep, per lane, every Gaussian whose interval meets the chunk)."""
import numpy as np
import pytest
import torch

from conftest import INFER_SCENES, load_golden
from helpers import camera_from_vector

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-4
FAST_IMG_TOL = 1e-3
UNCAPPED = [n for n in INFER_SCENES if n != "infer_capped"]


def _params(c, dev):
    return {k[3:]: torch.tensor(c[k], dtype=torch.float32, device=dev) for k in c if k.startswith("in_")}


def _infer(c, dev, mode, engine=None):
    from ray_gauss_b200.batched import BatchedViews, render_views_inference
    from ray_gauss_b200.engine import Engine
    P = _params(c, dev)
    cam = camera_from_vector(c["cam"], int(c["width"]), int(c["height"]), dev)
    views = BatchedViews([cam], engine=engine or Engine(dev.index or 0), mode=mode, white_background=bool(c["white"]),
                         max_prim_slice=int(c["max_prim_slice"]))
    img, cnt = render_views_inference(P, views, counts=True)
    torch.cuda.synchronize()
    return img.cpu().numpy(), cnt.cpu().numpy()


@pytest.mark.parametrize("name", UNCAPPED)
def test_parity_inference_matches_reference_programs(cuda, name):
    c = load_golden(name)
    img, cnt = _infer(c, cuda, "parity")
    assert np.abs(img - c["ref_image"]).max() <= IMG_TOL
    assert np.array_equal(cnt, c["ref_counts"])


@pytest.mark.parametrize("name", UNCAPPED)
def test_fast_inference_close_to_reference_programs(cuda, name):
    c = load_golden(name)
    img, cnt = _infer(c, cuda, "fast")
    assert np.abs(img - c["ref_image"]).max() <= FAST_IMG_TOL
    assert np.all(cnt >= c["ref_counts"])


def test_counts_are_capped_per_slab_like_the_reference(cuda, oracle):
    """Slabs with more hits than max_prim_slice: the reference keeps the first hits of its traversal
    (so its image, and with it the ray's termination, depends on the traversal order) and counts
    max_prim_slice for the slab.  The engine keeps every hit but caps each slab's count the same way:
    against the oracle with all hits kept and only the counts capped."""
    c = load_golden("infer_capped")
    img, cnt = _infer(c, cuda, "parity")
    ref, rcnt = oracle.render_inference(c["in_positions"], c["in_scales"], c["in_quaternions"], c["in_densities"],
                                        c["ref_rgb"], c["cam"], int(c["width"]), int(c["height"]), bool(c["white"]),
                                        max_prim_slice=1 << 20, count_cap=int(c["max_prim_slice"]))
    assert np.abs(img - ref).max() <= IMG_TOL
    assert np.array_equal(cnt, rcnt)
    assert rcnt.sum() < oracle.render_inference(c["in_positions"], c["in_scales"], c["in_quaternions"],
                                                c["in_densities"], c["ref_rgb"], c["cam"], int(c["width"]),
                                                int(c["height"]), bool(c["white"]), max_prim_slice=1 << 20)[1].sum()


def test_launch_pipeline_test_against_oracle(cuda, oracle):
    """The OptiX-helper mirror (launch_pipeline_test on per-Gaussian colours) against the FP32
    oracle's inference render."""
    from ray_gauss_b200.optix_raycasting.optix_utils import launch_pipeline_test
    c = load_golden("infer_small_object_sh3")
    P = _params(c, cuda)
    cam = camera_from_vector(c["cam"], int(c["width"]), int(c["height"]), cuda)
    rgb = torch.tensor(c["ref_rgb"], device=cuda)
    img, cnt = launch_pipeline_test(None, None, None, None, None, cam, P["densities"], rgb, P["positions"],
                                    P["scales"], P["quaternions"], int(c["max_prim_slice"]), 0, (1, 1),
                                    bool(c["white"]), return_counts=True)
    ref, rcnt = oracle.render_inference(c["in_positions"], c["in_scales"], c["in_quaternions"], c["in_densities"],
                                        c["ref_rgb"], c["cam"], int(c["width"]), int(c["height"]), bool(c["white"]))
    assert np.abs(img.cpu().numpy() - ref).max() <= IMG_TOL
    assert np.array_equal(cnt.cpu().numpy(), rcnt)


def test_batched_inference_equals_single_views(cuda):
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.batched import BatchedViews, render_views_inference
    from ray_gauss_b200.engine import Engine
    p, _, white = S.workload("small_object", n=3000, seed=4)
    P = {k: v.to(cuda) for k, v in p.items()}
    cams = [S.sphere_camera(3.0, w, h, 40.0, seed=k, device=cuda) for k, (w, h) in enumerate(((40, 30), (23, 17)))]
    eng = Engine(cuda.index or 0)
    both, cnt = render_views_inference(P, BatchedViews(cams, engine=eng, mode="parity", white_background=white),
                                       counts=True)
    parts = [render_views_inference(P, BatchedViews([c], engine=eng, mode="parity", white_background=white),
                                    counts=True) for c in cams]
    assert torch.equal(both, torch.cat([p[0] for p in parts]))
    assert torch.equal(cnt, torch.cat([p[1] for p in parts]))
