"""Generate the densify / prune fixtures in tests/golden/densify/ with the reference's own code.

Run in a container where the reference tree is mounted at /root/reference (or at $RAYGAUSS_REFERENCE):
    python tests/golden/make_densify_golden.py
It builds the reference's PointCloud state by hand (the trained tensors, its per-tensor Adam
optimizers from classes/optimizer.py:init_ConstantLR in an OptimizerManagerDict, a few real Adam
steps so that the moments are non-zero, the densification statistics and filter_3D), then calls the
reference's PointCloud.densify_and_prune (classes/point_cloud.py:1128-1143, which runs
densify_and_clone :1102-1126, densify_and_split :1068-1098, densification_postfix :1034-1066 and
prune_points :497-516 with the optimizer-state surgery of classes/optimizer.py:54-83, 151-164) on the
CPU, and saves its inputs and outputs.

To run on the CPU: modules the reference imports for other paths (the simple-knn CUDA extension,
cupy, imageio, matplotlib, skimage, turtle) are replaced by empty modules; tensors the code
allocates on "cuda" are allocated on the CPU; torch's CPU generator is seeded before the call and
the standard normals of the split samples are regenerated from the same seed (torch.normal(mean,
std) draws one standard normal per element in element order and scales it by std; the script checks
that the reference's samples equal them times std).  The engine test feeds those normals to the
CUDA densify and compares every tensor.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "densify")
REF = os.environ.get("RAYGAUSS_REFERENCE", "/root/reference")

# the reference's optimizer names (utils/optim_utils.py, point_cloud.py:1037-1045) and our tensor names
NAMES = {"xyz": "positions", "rgb": "rgb", "sh": "spherical_harmonics", "density": "densities", "scales": "scales",
         "quaternions": "quaternions", "sph_gauss_features": "sph_gauss_features",
         "bandwidth_sharpness": "bandwidth_sharpness", "lobe_axis": "lobe_axis"}


def _stub_modules():
    for name in ("simple_knn", "simple_knn._C", "cupy", "imageio", "matplotlib", "matplotlib.pyplot", "skimage",
                 "skimage.metrics", "turtle"):
        try:
            if name not in ("simple_knn", "simple_knn._C"):
                importlib.import_module(name)
                continue
        except Exception:
            pass
        m = types.ModuleType(name)
        m.__getattr__ = lambda attr: None
        m.__path__ = []
        sys.modules[name] = m


def _cuda_to_cpu():
    """Allocations the reference makes with device="cuda" go to the CPU."""
    for fn in ("zeros", "ones", "empty", "tensor", "full"):
        orig = getattr(torch, fn)

        def wrapped(*a, _orig=orig, **k):
            if str(k.get("device", "")).startswith("cuda"):
                k["device"] = "cpu"
            return _orig(*a, **k)
        setattr(torch, fn, wrapped)


_SAMPLES = {}


def _capture_normal():
    """Records the std argument and the result of each torch.normal call (the split samples)."""
    orig = torch.normal

    def normal(*a, **k):
        res = orig(*a, **k)
        _SAMPLES["std"] = k.get("std", a[1] if len(a) > 1 else None)
        _SAMPLES["out"] = res
        return res
    torch.normal = normal


def make_case(name, n, nsg, n_sh, seed, max_grad, min_density, extent, PC, opt):
    g = torch.Generator().manual_seed(seed)
    f = torch.float32
    raw = {"positions": torch.randn(n, 3, generator=g), "rgb": torch.rand(n, 3, generator=g),
           "spherical_harmonics": 0.1 * torch.randn(n, 3, n_sh, generator=g),
           "densities": torch.rand(n, generator=g) * 3.5 - 0.5,
           "scales": torch.rand(n, 3, generator=g) * 5.0 - 6.0,
           "quaternions": torch.randn(n, 4, generator=g),
           "sph_gauss_features": torch.randn(n, 3, nsg, generator=g),
           "bandwidth_sharpness": torch.randn(n, nsg, generator=g),
           "lobe_axis": torch.randn(n, nsg, 3, generator=g)}
    pc = PC("float32", "cpu")
    for k, v in raw.items():
        setattr(pc, k, v.to(f).clone().requires_grad_(True))
    managers = {}
    for oname, k in NAMES.items():
        cfg = types.SimpleNamespace(init_lr=1e-3)
        managers[oname] = opt.init_ConstantLR(cfg, getattr(pc, k), lr_list=[], donotuse_steps=0)
    pc.optim_managers = opt.OptimizerManagerDict(managers)
    # three real Adam steps: non-zero moments and step counts, as after training
    for _ in range(3):
        for oname, k in NAMES.items():
            t = getattr(pc, k)
            t.grad = 1e-2 * torch.randn(t.shape, generator=g)
        pc.optim_managers.step()
    num = torch.randint(0, 5, (n,), generator=g).to(f)
    accum = torch.rand(n, generator=g) * 2e-4 * num
    inf_rows = torch.randperm(n, generator=g)[:5]
    accum[inf_rows] = 1e-3                                  # num == 0, accum > 0: mean gradient inf
    num[inf_rows] = 0.0
    pc.xyz_gradient_accum_norm = accum.clone()
    pc.num_accum = num.clone()
    pc.num_accum_gnv = torch.randint(0, 9, (n,), generator=g).to(f)
    pc.filter_3D = torch.rand(n, 1, generator=g) * 2.0 - 7.0
    out = {"max_grad": np.float64(max_grad), "min_density": np.float64(min_density), "extent": np.float64(extent),
           "n_split": np.int32(2)}
    for oname, k in NAMES.items():
        t = getattr(pc, k)
        st = pc.optim_managers.optimizer_manager_dict[oname].optimizer.state[t]
        out[f"in/{k}"] = t.detach().numpy().copy()
        out[f"in_m/{k}"] = st["exp_avg"].numpy().copy()
        out[f"in_v/{k}"] = st["exp_avg_sq"].numpy().copy()
        out[f"in_step/{k}"] = np.int32(int(st["step"]))
    for k in ("xyz_gradient_accum_norm", "num_accum", "num_accum_gnv"):
        out[f"in_stat/{k}"] = getattr(pc, k).numpy().copy()
    out["in_filter_3D"] = pc.filter_3D.numpy().copy()

    _SAMPLES.clear()
    torch.manual_seed(seed + 1)
    pc.densify_and_prune(max_grad, min_density, extent, quiet=True)
    if "std" in _SAMPLES:
        std = _SAMPLES["std"]
        torch.manual_seed(seed + 1)
        z = torch.randn(std.shape)
        assert torch.equal(z * std, _SAMPLES["out"]), "split samples are not z * std"
        out["normals"] = z.numpy()
    else:
        out["normals"] = np.zeros((0, 3), np.float32)
    for oname, k in NAMES.items():
        t = getattr(pc, k)
        st = pc.optim_managers.optimizer_manager_dict[oname].optimizer.state[t]
        out[f"out/{k}"] = t.detach().numpy().copy()
        out[f"out_m/{k}"] = st["exp_avg"].numpy().copy()
        out[f"out_v/{k}"] = st["exp_avg_sq"].numpy().copy()
        out[f"out_step/{k}"] = np.int32(int(st["step"]))
    for k in ("xyz_gradient_accum_norm", "num_accum", "num_accum_gnv"):
        out[f"out_stat/{k}"] = getattr(pc, k).numpy().copy()
    out["out_filter_3D"] = pc.filter_3D.numpy().copy()
    os.makedirs(OUT, exist_ok=True)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(name, "n", n, "->", out["out/positions"].shape[0], "split samples", out["normals"].shape[0])


def main():
    _stub_modules()
    _cuda_to_cpu()
    sys.path.insert(0, REF)
    from classes import optimizer as opt
    from classes.point_cloud import PointCloud
    _capture_normal()
    # clones, splits and the density prune all occur; SH degree 1 and two SG lobes keep the files small
    make_case("mixed", 900, 2, 3, 0, 1e-4, 0.1, 1.0, PointCloud, opt)
    # eight SG lobes, a higher threshold (fewer selections) and a larger extent (more clones than splits)
    make_case("sg8_extent", 420, 8, 3, 1, 2e-4, 0.05, 3.0, PointCloud, opt)


if __name__ == "__main__":
    main()
