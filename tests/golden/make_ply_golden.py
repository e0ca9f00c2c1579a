"""Generate the PLY fixtures in tests/golden/ply/ with the reference's own PLY module.

Run in a container where the reference tree is mounted at /root/reference (or at $RAYGAUSS_REFERENCE):
    python tests/golden/make_ply_golden.py
The reference's scripts/ply.py (numpy only) writes the point-cloud files and reads them back; the
fixtures hold the files and, in expected.npz, every field as the reference's read_ply returns it
plus the tensors the reference's loaders build from them (classes/point_cloud.py:298-394 for RGB
point clouds, :396-495 for 3DGS files, and the trained-scene layout of convertpth_to_ply.py:60-117),
restated here in numpy because those loaders need a CUDA device.  The big-endian, mixed-type file is
written by this script (the reference only writes the host byte order) and read by the reference.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "ply")
REF = os.environ.get("RAYGAUSS_REFERENCE", "/root/reference")


def ref_ply():
    spec = importlib.util.spec_from_file_location("ref_ply", os.path.join(REF, "scripts", "ply.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def main():
    ply = ref_ply()
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(7)
    exp = {}
    f4 = np.float32

    def record(tag, path, fields=True):
        data = ply.read_ply(path)
        exp[f"{tag}/names"] = np.array(data.dtype.names)
        if fields:
            for nm in data.dtype.names:
                exp[f"{tag}/field/{nm}"] = np.asarray(data[nm])
        return data

    # A. RGB point cloud with every optional field (load_from_ply, point_cloud.py:298-394)
    n = 37
    pts = rng.normal(size=(n, 3)).astype(f4)
    cols = rng.integers(0, 256, size=(n, 3), dtype=np.uint8)
    dens = rng.uniform(0.1, 3.0, size=n)                               # float64 in the file
    scl = (rng.uniform(-5, -1, size=(n, 3))).astype(f4)
    quat = rng.normal(size=(n, 4)).astype(f4)
    path = os.path.join(OUT, "rgb_full.ply")
    ply.write_ply(path, [pts, cols, dens, scl, quat],
                  ["x", "y", "z", "red", "green", "blue", "density", "sx", "sy", "sz", "qx", "qy", "qz", "qw"])
    d = record("rgb_full", path)
    colors = np.vstack((d["red"], d["green"], d["blue"])).T / 255 - 0.5
    exp["rgb_full/positions"] = np.vstack((d["x"], d["y"], d["z"])).T.astype(f4)
    exp["rgb_full/densities"] = d["density"].astype(np.float64).astype(f4)
    exp["rgb_full/rgb"] = (colors * 2 * np.sqrt(np.pi)).astype(f4)
    exp["rgb_full/scales"] = np.vstack((d["sx"], d["sy"], d["sz"])).T.astype(f4)
    exp["rgb_full/quaternions"] = np.vstack((d["qx"], d["qy"], d["qz"], d["qw"])).T.astype(f4)

    # B. minimal RGB cloud: double positions, no density (default), no rotation (identity)
    n = 41
    pts = rng.normal(size=(n, 3))                                      # float64 in the file
    cols = rng.integers(0, 256, size=(n, 3), dtype=np.uint8)
    scl = (rng.uniform(-5, -1, size=(n, 3))).astype(f4)
    path = os.path.join(OUT, "rgb_min.ply")
    ply.write_ply(path, [pts, cols, scl], ["x", "y", "z", "red", "green", "blue", "sx", "sy", "sz"])
    d = record("rgb_min", path)
    colors = np.vstack((d["red"], d["green"], d["blue"])).T / 255 - 0.5
    exp["rgb_min/positions"] = np.vstack((d["x"], d["y"], d["z"])).T.astype(f4)
    exp["rgb_min/densities"] = (np.ones(n) * 0.7).astype(f4)          # default_density = 0.7
    exp["rgb_min/rgb"] = (colors * 2 * np.sqrt(np.pi)).astype(f4)
    exp["rgb_min/scales"] = np.vstack((d["sx"], d["sy"], d["sz"])).T.astype(f4)
    q = np.zeros((n, 4))
    q[:, 0] = 1
    exp["rgb_min/quaternions"] = q.astype(f4)

    # C. 3DGS file (load_from_gaussian_splatting, point_cloud.py:396-495): SH degree 3
    n = 260
    names = ["x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(45)]
    names += ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    cols = rng.normal(size=(n, len(names))).astype(f4)
    path = os.path.join(OUT, "gs3d.ply")
    ply.write_ply(path, [cols], names)
    d = record("gs3d", path, fields=False)
    exp["gs3d/positions"] = np.vstack((d["x"], d["y"], d["z"])).T.astype(f4)
    exp["gs3d/densities"] = np.asarray(d["opacity"], f4)
    exp["gs3d/scales"] = np.vstack((d["scale_0"], d["scale_1"], d["scale_2"])).T.astype(f4)
    exp["gs3d/quaternions"] = np.vstack([d[f"rot_{i}"] for i in range(4)]).T.astype(f4)
    exp["gs3d/rgb"] = np.vstack((d["f_dc_0"], d["f_dc_1"], d["f_dc_2"])).T.astype(f4)
    rest = np.zeros((n, 45))
    for i in range(45):
        rest[:, i] = d[f"f_rest_{i}"]
    sh = np.zeros((n, 3, 15), f4)
    for c in range(3):
        sh[:, c, :] = rest[:, 15 * c:15 * (c + 1)].astype(f4)
    exp["gs3d/spherical_harmonics"] = sh

    # D. trained scene as convertpth_to_ply.py writes it: SH degree 3 (16 coefficients), 2 SG lobes
    n, hn, ns = 200, 16, 2
    P = {"positions": rng.normal(size=(n, 3)).astype(f4), "rgb": rng.normal(size=(n, 3)).astype(f4),
         "spherical_harmonics": rng.normal(size=(n, 3, hn - 1)).astype(f4),
         "densities": rng.uniform(0, 4, size=n).astype(f4), "scales": rng.uniform(-6, -1, size=(n, 3)).astype(f4),
         "quaternions": rng.normal(size=(n, 4)).astype(f4),
         "sph_gauss_features": rng.normal(size=(n, 3, ns)).astype(f4),
         "bandwidth_sharpness": rng.normal(size=(n, ns)).astype(f4),
         "lobe_axis": rng.normal(size=(n, ns, 3)).astype(f4)}
    gacc = rng.uniform(0, 1e-3, size=n).astype(f4)
    colors = np.concatenate((P["rgb"][:, :, None], P["spherical_harmonics"]), axis=2)
    fields, data = ["x", "y", "z"], [P["positions"]]
    for c, ch in enumerate("rgb"):
        for h in range(hn):
            data.append(colors[:, c, h])
            fields.append(f"sh{h}{ch}")
    fields.append("density")
    data.append(P["densities"])
    fields.extend(["sx", "sy", "sz"])
    data.append(P["scales"])
    fields.extend(["qx", "qy", "qz", "qw"])
    data.append(P["quaternions"])
    for c, ch in enumerate("rgb"):
        for k in range(ns):
            data.append(P["sph_gauss_features"][:, c, k])
            fields.append(f"sg{k}{ch}")
    for k in range(ns):
        fields.append(f"bandwidth_sharpness{k}")
        data.append(P["bandwidth_sharpness"][:, k])
    for k in range(ns):
        fields.extend([f"lobe_{k}x", f"lobe_{k}y", f"lobe_{k}z"])
        data.append(P["lobe_axis"][:, k])
    fields.append("gradient_accum_norm")
    data.append(gacc)
    path = os.path.join(OUT, "trained.ply")
    ply.write_ply(path, data, fields)
    record("trained", path, fields=False)
    for k, v in P.items():
        exp[f"trained/{k}"] = v
    exp["trained/gradient_accum_norm"] = gacc

    # E. big-endian file with every property type (written here, read by the reference)
    n = 300
    spec = [("a", ">i1", "char"), ("b", ">u1", "uchar"), ("c", ">i2", "short"), ("d", ">u2", "ushort"),
            ("e", ">i4", "int"), ("f", ">u4", "uint"), ("g", ">f4", "float"), ("h", ">f8", "double")]
    rec = np.empty(n, dtype=[(nm, t) for nm, t, _ in spec])
    rec["a"] = rng.integers(-128, 128, n)
    rec["b"] = rng.integers(0, 256, n)
    rec["c"] = rng.integers(-32768, 32768, n)
    rec["d"] = rng.integers(0, 65536, n)
    rec["e"] = rng.integers(-2 ** 31, 2 ** 31, n)
    rec["f"] = rng.integers(0, 2 ** 32, n, dtype=np.uint64)
    rec["g"] = rng.normal(size=n)
    rec["h"] = rng.normal(size=n) * 1e5
    path = os.path.join(OUT, "mixed_big_endian.ply")
    with open(path, "wb") as fh:
        head = ["ply", "format binary_big_endian 1.0", f"element vertex {n}"]
        head += [f"property {pt} {nm}" for nm, _, pt in spec] + ["end_header"]
        fh.write("".join(h + "\n" for h in head).encode())
        rec.tofile(fh)
    record("mixed", path)

    np.savez_compressed(os.path.join(OUT, "expected.npz"), **exp)
    print(f"wrote {len(exp)} arrays and 5 PLY files to {OUT}")


if __name__ == "__main__":
    sys.exit(main())
