"""The CPU oracle against the reference's own code (golden fixtures) and analytic cases.

The golden fixtures were produced by tests/golden/make_golden.py from the reference's device
programs (compiled for the CPU with an OptiX-emulation header) and its torch SH twin.  These tests
pin the C restatement used as the oracle everywhere else.
"""
import math

import numpy as np
import pytest

from conftest import INFER_SCENES, SCENES, load_golden
from helpers import rel_l2


def _inputs(c):
    P = {k[3:]: c[k] for k in c if k.startswith("in_")}
    nsg = P["sph_gauss_features"].shape[2]
    return P, nsg


@pytest.mark.parametrize("name", SCENES)
def test_oracle_f32_matches_reference_programs(oracle, name):
    c = load_golden(name)
    P, nsg = _inputs(c)
    W, H = int(c["width"]), int(c["height"])
    sg = P["sph_gauss_features"] if nsg else None
    kap = P["bandwidth_sharpness"] if nsg else None
    ax = P["lobe_axis"] if nsg else None
    rgb = oracle.forward_sh(c["cam"][:3], P["positions"], P["color_features"], sg, kap, ax)
    assert np.abs(rgb - c["ref_rgb"]).max() <= 1e-6
    img, T, st = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, c["cam"],
                                       W, H, bool(c["white"]), int(c["max_prim_slice"]), int(c["jitter"]),
                                       int(c["rnd_sample"]), int(c["iteration"]))
    assert np.abs(img - c["ref_image"]).max() <= 2e-6
    g = oracle.render_backward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, c["cam"], W, H,
                               img, c["dL"], int(c["max_prim_slice"]), int(c["jitter"]), int(c["rnd_sample"]),
                               int(c["iteration"]))
    for k in ("d_rgb", "d_dens", "d_pos", "d_scl", "d_quat"):
        ref = c["ref_" + k] if k != "d_pos" else c["ref_d_pos_geo"]
        assert rel_l2(g[k], ref) <= 1e-5, k
    dsh, dpos, dsg, dkap, dax = oracle.backward_sh(c["cam"][:3], P["positions"], P["color_features"], sg, kap, ax,
                                                   g["d_rgb"].astype(np.float32), ref_quirks=True)
    assert rel_l2(dsh, c["ref_d_sh"]) <= 1e-5
    assert rel_l2(g["d_pos"] + dpos, c["ref_d_pos"]) <= 1e-5
    if nsg:
        assert rel_l2(dsg, c["ref_d_sg"]) <= 1e-5
        assert rel_l2(dkap, c["ref_d_kappa"]) <= 1e-5
        assert rel_l2(dax, c["ref_d_axis"]) <= 1e-5


@pytest.mark.parametrize("name", SCENES)
def test_oracle_f64_close_to_f32_reference(oracle, name):
    """FP64 of the same algorithm sits within FP32 noise of the reference image."""
    c = load_golden(name)
    P, nsg = _inputs(c)
    W, H = int(c["width"]), int(c["height"])
    img, _, _ = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], c["ref_rgb"],
                                      c["cam"], W, H, bool(c["white"]), 1024, int(c["jitter"]),
                                      int(c["rnd_sample"]), int(c["iteration"]), prec="f64")
    assert np.abs(img - c["ref_image"]).max() <= 2e-3


def test_sh_against_reference_torch_twin(oracle):
    """utils/sh_utils.py eval_sh / backward_sh (the reference's torch twin, correct degree-3 derivative)."""
    c = load_golden("sh_twin")
    n = c["pos"].shape[0]
    for deg in range(4):
        sh = c[f"sh{deg}"]
        rgb = oracle.forward_sh(c["campos"], c["pos"], sh, None, None, None, prec="f64")
        assert np.abs(rgb - c[f"rgb{deg}"]).max() <= 2e-6
        dsh, dpos, _, _, _ = oracle.backward_sh(c["campos"], c["pos"], sh, None, None, None, c[f"dL{deg}"],
                                                prec="f64", ref_quirks=False)
        assert rel_l2(dsh, c[f"dsh{deg}"]) <= 1e-5
        assert rel_l2(dpos, c[f"dmean{deg}"]) <= 1e-4
        assert dpos.shape == (n, 3)


def _single_gaussian(d, s=0.1, pos=(0.0, 0.0, 0.0)):
    P = dict(positions=np.array([pos], np.float64), scales=np.array([[s, s, s]], np.float64),
             quaternions=np.array([[1.0, 0.0, 0.0, 0.0]]), densities=np.array([d], np.float64))
    return P


def _axis_camera(eye_z=3.0, W=3, H=3, tan=0.05):
    # looking down -z from (0,0,eye_z): U=(1,0,0), V=(0,-1,0)... any right-handed frame works here
    return np.array([0, 0, eye_z, 1, 0, 0, 0, -1, 0, 0, 0, -1, tan, tan], np.float64)


def test_kat_single_isotropic_gaussian_centre_ray(oracle):
    """Closed form for the centre ray through an isotropic Gaussian: samples on the slab grid from the
    scene-box entry, summed density d*exp(-r^2/2s^2) above 0.1, composited per slab."""
    d, s = 5.0, 0.1
    P = _single_gaussian(d, s)
    cam = _axis_camera(3.0, 1, 1)
    rgb = np.array([[0.2, 0.5, 0.9]])
    img, T, _ = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cam, 1, 1,
                                      True, prec="f64")
    # expected, straight from the definition (the reference's float constants, evaluated in double)
    dt, thr, teps = float(np.float32(0.0025)), float(np.float32(0.1)), float(np.float32(0.003))
    delta = math.sqrt(math.log((d / 0.1) ** 2))
    ext = delta * s
    tenter, texit = 3.0 - ext, 3.0 + ext
    t, Tr, col = tenter, 1.0, np.zeros(3)
    while t < texit and Tr > teps:
        for i in range(8):
            ts = t + i * dt
            w = math.exp(-0.5 * ((ts - 3.0) / s) ** 2)
            sig = d * w if d * w > thr else 0.0
            a = 1.0 - math.exp(-sig * dt)
            col += Tr * a * rgb[0]
            Tr *= 1.0 - a
        t += dt * 8
    expect = col + Tr * 1.0
    assert np.abs(img[0] - expect).max() <= 1e-9
    assert abs(T[0] - Tr) <= 1e-12


def test_kat_density_at_threshold_is_background(oracle):
    """Density <= 0.1 never passes the per-sample mask (and its ellipsoid degenerates): background."""
    for d in (0.1, 0.05):
        P = _single_gaussian(d, 0.3)
        cam = _axis_camera(3.0, 4, 4, 0.1)
        rgb = np.array([[0.0, 0.0, 0.0]])
        for prec in ("f32", "f64"):
            img, T, st = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb,
                                               cam, 4, 4, True, prec=prec)
            assert np.all(img == 1.0) and np.all(T == 1.0)


def test_kat_camera_inside_gaussian_centred_behind_is_dropped(oracle):
    """The reference's ellipsoid test returns its roots in reversed order when the centre projects
    behind the ray origin; a Gaussian containing the camera with its centre behind it is never hit."""
    base = _single_gaussian(4.0, 0.05, pos=(0.0, 0.0, 0.0))
    cam = _axis_camera(3.0, 3, 3, 0.05)
    rgb1 = np.array([[0.3, 0.3, 0.3]])
    img0, _, _ = oracle.render_forward(base["positions"], base["scales"], base["quaternions"], base["densities"],
                                       rgb1, cam, 3, 3, True, prec="f64")
    # add a wide Gaussian centred 0.05 behind the camera (contains the camera)
    P = {k: np.concatenate([base[k], _single_gaussian(4.0, 0.5, pos=(0.0, 0.0, 3.05))[k]]) for k in base}
    rgb2 = np.array([[0.3, 0.3, 0.3], [0.0, 1.0, 0.0]])
    img1, _, _ = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb2, cam, 3, 3,
                                       True, prec="f64")
    # the scene box grows (slab grid anchored at the new entry), so compare loosely: no green tint
    assert np.abs(img1[:, 1] - img1[:, 0]).max() <= 1e-3
    # ...whereas the same Gaussian centred in front of the camera is hit and tints the image green
    P["positions"][1, 2] = 2.95
    img2, _, _ = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb2, cam, 3, 3,
                                       True, prec="f64")
    assert (img2[:, 1] - img2[:, 0]).min() > 1e-2


def test_hit_cap_counts_overflow(oracle):
    """More hits in a slab than max_prim_slice: the reference truncates and counts (forward/...cu:624-629)."""
    rng = np.random.default_rng(0)
    n = 40
    P = dict(positions=rng.normal(0, 0.01, (n, 3)), scales=np.full((n, 3), 0.2), quaternions=np.tile([1.0, 0, 0, 0], (n, 1)),
             densities=np.full(n, 2.0))
    rgb = np.full((n, 3), 0.5)
    cam = _axis_camera(3.0, 2, 2, 0.01)
    _, _, st = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cam, 2, 2,
                                     True, max_prim_slice=8)
    assert st[0] > 0
    _, _, st2 = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cam, 2, 2,
                                      True, max_prim_slice=1024)
    assert st2[0] == 0


@pytest.mark.parametrize("name", INFER_SCENES)
def test_oracle_inference_matches_reference_programs(oracle, name):
    """The inference restatement against the reference's inference programs (cuda_test) run on
    the CPU: image and Gaussians per ray (the per-slab cap included)."""
    c = load_golden(name)
    img, counts = oracle.render_inference(c["in_positions"], c["in_scales"], c["in_quaternions"], c["in_densities"],
                                          c["ref_rgb"], c["cam"], int(c["width"]), int(c["height"]),
                                          bool(c["white"]), int(c["max_prim_slice"]))
    assert np.abs(img - c["ref_image"]).max() <= 2e-6
    assert np.array_equal(counts, c["ref_counts"])


def test_oracle_inference_differs_from_training_forward_only_slightly(oracle):
    """The inference programs sample through the conic space incrementally and clip the slab query
    differently; on a plain scene the two renders agree to the 1e-3 level but not bit for bit."""
    c = load_golden("infer_small_object_sh3")
    args = (c["in_positions"], c["in_scales"], c["in_quaternions"], c["in_densities"], c["ref_rgb"], c["cam"],
            int(c["width"]), int(c["height"]), bool(c["white"]))
    img, _ = oracle.render_inference(*args)
    fwd, _, _ = oracle.render_forward(*args)
    d = np.abs(img - fwd).max()
    assert 0.0 < d <= 1e-3


@pytest.mark.parametrize("workload", ["unbounded", "bounded"])
def test_grid_prefilter_gives_the_scan_results(oracle, workload):
    """The nested-grid candidate prefilter returns the candidate lists of a scan over every
    Gaussian, in the same order: images, transmittances and gradients are bit-identical."""
    from ray_gauss_b200 import synthetic as S
    if workload == "unbounded":
        p = S.unbounded(60_000, seed=3, nsg=0)
        cam = S.ring_cameras(1, seed=3, w_range=(96, 96))[0]
    else:
        p = S.bounded_object(40_000, seed=3, nsg=0)
        cam = S.sphere_camera(4.0, 96, 72, 40.0, seed=3)
    P = {k: np.asarray(v, np.float32) for k, v in p.items()}
    W, H = cam.image_width, cam.image_height
    ids = np.random.default_rng(1).choice(W * H, 600, replace=False).astype(np.int32)
    cv = oracle.camera_vector(cam)
    rgb = oracle.forward_sh(cv[:3], P["positions"], P["color_features"], None, None, None)
    dL = np.random.default_rng(2).normal(0, 1, (ids.size, 3)).astype(np.float32)
    out = {}
    try:
        for on in (True, False):
            oracle.set_grid(on)
            img, T, st = oracle.render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv,
                                               W, H, True, ray_ids=ids)
            g = oracle.render_backward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W, H,
                                       img, dL, ray_ids=ids)
            out[on] = (img, T, st, g)
    finally:
        oracle.set_grid(True)
    assert out[True][2][1] > 0   # hits were found
    assert np.array_equal(out[True][0], out[False][0]) and np.array_equal(out[True][1], out[False][1])
    assert np.array_equal(out[True][2], out[False][2])
    for k in ("d_rgb", "d_dens", "d_pos", "d_scl", "d_quat"):
        assert np.array_equal(out[True][3][k], out[False][3][k]), k


def test_reference_programs_grid_gives_the_scan_results(oracle):
    """The reference programs' OptiX stand-in finds each trace call's primitives through the grid:
    same primitives in the same order as its per-ray scan, so bit-identical outputs."""
    if not oracle.ref_available():
        pytest.skip("reference programs not built (oracle/_ref)")
    from ray_gauss_b200 import synthetic as S
    p = S.unbounded(20_000, seed=5, nsg=0)
    cam = S.ring_cameras(1, seed=5, w_range=(64, 64))[0]
    P = {k: np.asarray(v, np.float32) for k, v in p.items()}
    W, H = cam.image_width, cam.image_height
    ids = np.random.default_rng(3).choice(W * H, 200, replace=False).astype(np.int32)
    cv = oracle.camera_vector(cam).astype(np.float32)
    rgb = oracle.ref_forward_sh(cv[:3], P["positions"], P["color_features"], None, None, None)
    dL = np.random.default_rng(4).normal(0, 1, (W * H, 3)).astype(np.float32)
    out = {}
    try:
        for on in (True, False):
            oracle.set_grid(on)
            img, ovf = oracle.ref_render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb,
                                                 cv, W, H, True, ray_ids=ids)
            g = oracle.ref_render_backward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv,
                                           W, H, img, dL, ray_ids=ids)
            inf, cnt = oracle.ref_render_inference(P["positions"], P["scales"], P["quaternions"], P["densities"],
                                                   rgb, cv, W, H, True, ray_ids=ids)
            out[on] = (img, g, inf, cnt)
    finally:
        oracle.set_grid(True)
    assert np.abs(out[True][0][ids] - 1.0).max() > 0.01   # the rays see the scene
    assert np.array_equal(out[True][0], out[False][0])
    # the backward programs add gradients with float atomics from OpenMP threads, whose order
    # differs from run to run (scan against scan differs by ~3e-7 of the largest entry)
    for k in ("d_rgb", "d_dens", "d_pos", "d_scl", "d_quat"):
        a, b = out[True][1][k], out[False][1][k]
        assert np.abs(a - b).max() <= 2e-6 * np.abs(b).max(), k
    assert np.array_equal(out[True][2], out[False][2]) and np.array_equal(out[True][3], out[False][3])
