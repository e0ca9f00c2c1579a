"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run in a container where the reference tree is mounted at /root/reference (or at $RAYGAUSS_REFERENCE):
    python tests/golden/make_golden.py                     (all fixtures)
    python tests/golden/make_golden.py --inference-only    (the infer_*.npz fixtures only)
It (1) builds oracle/_ref/ — the reference's training device programs
(optix_raycasting/cuda_train/{forward,backward}/gaussians_aabb.cu), its inference programs
(optix_raycasting/cuda_test/gaussians_aabb.cu) and SH kernels (utils/sh_utils.cu) compiled for the CPU with oracle/ref_shim/optix.h standing in for OptiX — and
(2) imports the reference's torch SH twin (utils/sh_utils.py: eval_sh, backward_sh).  The fixtures
hold seeded inputs and those reference outputs; the tests compare the C oracle and the CUDA engine
against them without needing the reference tree.
"""
from __future__ import annotations

import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("RAYGAUSS_REFERENCE", "/root/reference")
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402
from ray_gauss_b200 import synthetic as S  # noqa: E402


def cam_vec_of(cam):
    return O.camera_vector(cam)


def scene_case(name, P, cam, W, H, white=True, max_prim_slice=1024, jitter=0, rnd_sample=0, iteration=0, seed=0):
    f = np.float32
    P = {k: np.asarray(v, f) for k, v in P.items()}
    cv = cam_vec_of(cam).astype(f)
    nsg = P["sph_gauss_features"].shape[2]
    sg = P["sph_gauss_features"] if nsg else None
    kap = P["bandwidth_sharpness"] if nsg else None
    ax = P["lobe_axis"] if nsg else None
    rgb = O.ref_forward_sh(cv[:3], P["positions"], P["color_features"], sg, kap, ax)
    img, ovf = O.ref_render_forward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W, H,
                                    white, max_prim_slice, jitter, rnd_sample, iteration)
    rng = np.random.default_rng(seed + 77)
    target = rng.random(img.shape).astype(f)
    dL = (2.0 * (img - target) / img.size).astype(f)
    g = O.ref_render_backward(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W, H, img, dL,
                              max_prim_slice, jitter, rnd_sample, iteration)
    dsh, dpos_dir, dsg, dkap, dax = O.ref_backward_sh(cv[:3], P["positions"], P["color_features"], sg, kap, ax,
                                                      g["d_rgb"])
    out = dict(cam=cv, width=np.int32(W), height=np.int32(H), white=np.int32(white),
               max_prim_slice=np.int32(max_prim_slice), jitter=np.int32(jitter), rnd_sample=np.int32(rnd_sample),
               iteration=np.int32(iteration), ref_rgb=rgb, ref_image=img, ref_overflow=np.int32(ovf), dL=dL,
               ref_d_rgb=g["d_rgb"], ref_d_dens=g["d_dens"], ref_d_pos_geo=g["d_pos"], ref_d_scl=g["d_scl"],
               ref_d_quat=g["d_quat"], ref_d_sh=dsh, ref_d_pos=g["d_pos"] + dpos_dir, ref_d_sg=dsg, ref_d_kappa=dkap,
               ref_d_axis=dax)
    out.update({"in_" + k: v for k, v in P.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "image mean %.4f" % img.mean(), "overflow", ovf)


def inference_case(name, P, cam, W, H, white=True, max_prim_slice=1024):
    """The reference's inference programs (optix_raycasting/cuda_test/gaussians_aabb.cu): image and
    Gaussians per ray."""
    f = np.float32
    P = {k: np.asarray(v, f) for k, v in P.items()}
    cv = cam_vec_of(cam).astype(f)
    nsg = P["sph_gauss_features"].shape[2]
    sg = P["sph_gauss_features"] if nsg else None
    kap = P["bandwidth_sharpness"] if nsg else None
    ax = P["lobe_axis"] if nsg else None
    rgb = O.ref_forward_sh(cv[:3], P["positions"], P["color_features"], sg, kap, ax)
    img, counts = O.ref_render_inference(P["positions"], P["scales"], P["quaternions"], P["densities"], rgb, cv, W,
                                         H, white, max_prim_slice)
    out = dict(cam=cv, width=np.int32(W), height=np.int32(H), white=np.int32(white),
               max_prim_slice=np.int32(max_prim_slice), ref_rgb=rgb, ref_image=img, ref_counts=counts)
    out.update({"in_" + k: v for k, v in P.items()})
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "image mean %.4f" % img.mean(), "Gaussians per ray %.1f" % counts.mean())


def inference_cases():
    P = S.small_object(600, seed=1)
    P["scales"] = P["scales"] * 4.0
    inference_case("infer_small_object_sh3", P, S.sphere_camera(3.0, 32, 32, 40.0, 1), 32, 32, white=True)
    P = S.bounded_object(500, seed=2)
    P["scales"] = P["scales"] * 6.0
    inference_case("infer_shells_sg8", P, S.sphere_camera(4.0, 28, 24, 40.0, 2), 28, 24, white=False)
    # a per-slab cap the scene exceeds: the reference keeps the first hits of its traversal, so only
    # the oracle (same cap semantics) is compared against this one
    P = S.small_object(600, seed=8)
    P["scales"] = P["scales"] * 6.0
    inference_case("infer_capped", P, S.sphere_camera(3.0, 16, 16, 40.0, 8), 16, 16, white=True, max_prim_slice=4)


def inside_camera_scene(seed=5):
    """A camera inside several large Gaussians, some centred behind it (the reference's root-order
    behaviour drops those) plus a background cloud."""
    rng = np.random.default_rng(seed)
    P = S.small_object(300, seed)
    cam = S.sphere_camera(3.0, 24, 24, 40.0, seed)
    eye = cam.camera_center.numpy().astype(np.float64)
    fwd = -eye / np.linalg.norm(eye)
    big = []
    for k in range(6):
        off = rng.normal(0, 0.05, 3) + fwd * (0.08 if k % 2 == 0 else -0.08)
        big.append(eye + off)
    big = np.array(big)
    P["positions"] = np.concatenate([P["positions"], big])
    P["scales"] = np.concatenate([P["scales"], np.full((6, 3), 0.15) * rng.uniform(0.8, 1.2, (6, 3))])
    P["quaternions"] = np.concatenate([P["quaternions"], S._unit(rng, 6, 4)])
    P["densities"] = np.concatenate([P["densities"], rng.uniform(1.0, 3.0, 6)])
    P["color_features"] = np.concatenate([P["color_features"], rng.normal(0, 0.2, (6, 3, 16))])
    for k in ("sph_gauss_features", "bandwidth_sharpness", "lobe_axis"):
        P[k] = np.concatenate([P[k], np.zeros((6,) + P[k].shape[1:])])
    return P, cam


def sh_twin_case():
    import torch
    sys.path.insert(0, REF)
    from utils import sh_utils as R  # the reference's torch twin of the SH kernels
    rng = np.random.default_rng(11)
    n = 200
    pos = rng.uniform(-1, 1, (n, 3))
    campos = np.array([0.7, -2.6, 1.1])
    out = dict(pos=pos.astype(np.float32), campos=campos.astype(np.float32))
    for deg in range(4):
        sh = rng.normal(0, 0.3, (n, 3, (deg + 1) ** 2))
        dirs = pos - campos
        dirs = dirs / np.linalg.norm(dirs, axis=1, keepdims=True)
        val = R.eval_sh(deg, torch.tensor(sh, dtype=torch.float64), torch.tensor(dirs, dtype=torch.float64)).numpy()
        out[f"sh{deg}"] = sh.astype(np.float32)
        out[f"rgb{deg}"] = (val + 0.5).astype(np.float32)
        dL = rng.normal(0, 1, (n, 3))
        res = R.backward_sh(torch.tensor(pos, dtype=torch.float32), torch.tensor(campos, dtype=torch.float32),
                            torch.tensor(sh, dtype=torch.float32), torch.tensor(dL, dtype=torch.float32))
        out[f"dL{deg}"] = dL.astype(np.float32)
        if isinstance(res, (tuple, list)):
            out[f"dsh{deg}"] = res[0].numpy().astype(np.float32)
            if len(res) > 1:
                out[f"dmean{deg}"] = res[1].numpy().astype(np.float32)
        else:
            out[f"dsh{deg}"] = res.numpy().astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "sh_twin.npz"), **out)
    print("sh_twin", sorted(out.keys()))


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "all", "ref", f"REF={REF}"], check=True)
    if "--inference-only" in sys.argv:
        inference_cases()
        return
    # 1. the small-object distribution (configs' 10k case, thinned) with SH degree 3
    P = S.small_object(600, seed=1)
    P["scales"] = P["scales"] * 4.0
    scene_case("small_object_sh3", P, S.sphere_camera(3.0, 32, 32, 40.0, 1), 32, 32, white=True, seed=1)
    # 2. shells with 8 spherical Gaussians, black background
    P = S.bounded_object(500, seed=2)
    P["scales"] = P["scales"] * 6.0
    scene_case("shells_sg8", P, S.sphere_camera(4.0, 28, 24, 40.0, 2), 28, 24, white=False, seed=2)
    # 3. camera inside Gaussians (root-order behaviour of the ellipsoid test)
    P, cam = inside_camera_scene()
    scene_case("inside_camera", P, cam, 24, 24, white=True, seed=3)
    # 4. jittered rays and random sample offsets (RNG paths), iteration 7
    P = S.small_object(400, seed=4)
    P["scales"] = P["scales"] * 4.0
    scene_case("rng_jitter", P, S.sphere_camera(3.0, 20, 20, 40.0, 4), 20, 20, white=True, jitter=1, rnd_sample=1,
               iteration=7, seed=4)
    # 5. midpoint sampling (rnd_sample = 2), degree-1 SH
    P = S.small_object(400, seed=6)
    P["scales"] = P["scales"] * 4.0
    P["color_features"] = P["color_features"][:, :, :4]
    scene_case("midpoint_sh1", P, S.sphere_camera(3.0, 20, 16, 40.0, 6), 20, 16, white=True, rnd_sample=2, seed=6)
    sh_twin_case()
    inference_cases()


if __name__ == "__main__":
    main()
