"""Scene I/O: binary PLY point clouds and checkpoints of the reference, loaded straight into HBM.

PLY (the reference's reader, scripts/ply.py:62-146, and loaders, classes/point_cloud.py:298-495):
the header is parsed on the host, the vertex records are read once into pinned memory and copied to
the device in one transfer, and ``rg_records_to_columns`` converts the requested fields to FP32
columns of the trained tensors (one kernel, no per-field host copies).

- :func:`load_from_ply`: ``PointCloud.load_from_ply`` (x, y, z, optional density, red/green/blue
  mapped to the SH DC term, optional sx/sy/sz (else the k-NN initial scales of
  :mod:`ray_gauss_b200.knn`) and qx/qy/qz/qw).
- :func:`load_from_gaussian_splatting`: ``PointCloud.load_from_gaussian_splatting`` (3DGS files).
- :func:`load_trained_ply` / :func:`write_trained_ply`: the trained-scene layout written by the
  reference's convertpth_to_ply.py (sh{k}{c}, density, sx.., qx.., sg{k}{c}, bandwidth_sharpness{k},
  lobe_{k}{x,y,z}, gradient_accum_norm), byte for byte.
- :func:`save_checkpoint` / :func:`load_checkpoint`: the ``chkpnt{iteration}.pth`` tuple of
  ``PointCloud.save_model`` / ``restore_model`` (classes/point_cloud.py:922-958), with the optimizer
  state in torch's Adam format per manager, readable by the reference and by
  :func:`load_tail_state`.

Tensors use the reference's attribute names (:data:`ray_gauss_b200.train_tail.RAW_NAMES`).
"""
from __future__ import annotations

import ctypes
import math
import sys
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import check

# PLY type name -> (numpy type code, engine field type), as the reference's table (scripts/ply.py:31-49)
PLY_TYPES = {
    "int8": ("i1", _lib.RG_FIELD_I8), "char": ("i1", _lib.RG_FIELD_I8),
    "uint8": ("u1", _lib.RG_FIELD_U8), "uchar": ("u1", _lib.RG_FIELD_U8),
    "int16": ("i2", _lib.RG_FIELD_I16), "short": ("i2", _lib.RG_FIELD_I16),
    "uint16": ("u2", _lib.RG_FIELD_U16), "ushort": ("u2", _lib.RG_FIELD_U16),
    "int32": ("i4", _lib.RG_FIELD_I32), "int": ("i4", _lib.RG_FIELD_I32),
    "uint32": ("u4", _lib.RG_FIELD_U32), "uint": ("u4", _lib.RG_FIELD_U32),
    "float32": ("f4", _lib.RG_FIELD_F32), "float": ("f4", _lib.RG_FIELD_F32),
    "float64": ("f8", _lib.RG_FIELD_F64), "double": ("f8", _lib.RG_FIELD_F64),
}
FORMATS = {"binary_little_endian": "<", "binary_big_endian": ">"}

# reference optimizer-manager names (classes/point_cloud.py:1037-1046) of the trained tensors
MANAGER_NAMES = {"positions": "xyz", "rgb": "rgb", "spherical_harmonics": "sh", "densities": "density",
                 "scales": "scales", "quaternions": "quaternions", "sph_gauss_features": "sph_gauss_features",
                 "bandwidth_sharpness": "bandwidth_sharpness", "lobe_axis": "lobe_axis"}


@dataclass
class PlyHeader:
    n: int
    properties: list            # [(name, ply type name)]
    big_endian: bool
    body_offset: int
    offsets: dict = field(default_factory=dict)
    record_bytes: int = 0

    @property
    def names(self):
        return [p[0] for p in self.properties]

    def numpy_dtype(self):
        e = ">" if self.big_endian else "<"
        return np.dtype([(name, e + PLY_TYPES[t][0]) for name, t in self.properties])


def read_ply_header(path) -> PlyHeader:
    """Parse the header like the reference (scripts/ply.py:62-82, 120-138): the first line holds
    'ply', the second the format (ASCII is refused), every 'element' line sets the record count and
    every 'property' line adds a field, up to 'end_header'."""
    with open(path, "rb") as f:
        if b"ply" not in f.readline():
            raise ValueError("The file does not start whith the word ply")
        fmt = f.readline().split()[1].decode()
        if fmt == "ascii":
            raise ValueError("The file is not binary")
        if fmt not in FORMATS:
            raise ValueError(f"unknown PLY format {fmt!r}")
        n, props, line = None, [], b""
        while b"end_header" not in line:
            line = f.readline()
            if line == b"":
                raise ValueError("PLY header without end_header")
            if b"element" in line:
                n = int(line.split()[2])
            elif b"property" in line:
                parts = line.split()
                if parts[1] == b"list":
                    raise ValueError("list properties are not supported")
                t = parts[1].decode()
                if t not in PLY_TYPES:
                    raise ValueError(f"unknown PLY property type {t!r}")
                props.append((parts[2].decode(), t))
        body = f.tell()
    if n is None:
        raise ValueError("PLY header without element")
    h = PlyHeader(n, props, FORMATS[fmt] == ">", body)
    off = 0
    for name, t in props:
        h.offsets[name] = off
        off += np.dtype(PLY_TYPES[t][0]).itemsize
    h.record_bytes = off
    return h


class PlyVertices:
    """A binary PLY vertex block resident on one GPU: ``column``/``columns`` convert fields to FP32
    (``rg_records_to_columns``).  ``affine=(div, add, mul_a, mul_b)`` maps v to
    ((v / div) + add) * mul_a * mul_b in double before the float rounding."""

    def __init__(self, path, device="cuda"):
        self.header = read_ply_header(path)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("PLY records are converted on a CUDA device")
        h = self.header
        nbytes = h.n * h.record_bytes
        host = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
        with open(path, "rb") as f:
            f.seek(h.body_offset)
            got = f.readinto(memoryview(host.numpy()))
        if got != nbytes:
            raise ValueError(f"PLY body holds {got} bytes, the header announces {nbytes}")
        self.records = host.to(self.device, non_blocking=True)
        self._host = host                 # kept until the copy has run
        self.lib = _lib.load()

    @property
    def n(self):
        return self.header.n

    @property
    def names(self):
        return self.header.names

    def __contains__(self, name):
        return name in self.header.offsets

    def fill(self, targets):
        """targets: [(name, dst tensor view, affine or None)]: each dst is a float32 view with n
        elements at a constant stride (e.g. a column of an (n, k) tensor); one launch for all."""
        h = self.header
        arr = (_lib.rg_record_field * max(1, len(targets)))()
        for i, (name, dst, affine) in enumerate(targets):
            if name not in h.offsets:
                raise KeyError(name)
            if dst.dtype != torch.float32 or dst.dim() != 1 or dst.numel() != h.n or dst.device != self.device:
                raise ValueError(f"{name}: destination must be a 1-D view of {h.n} float32 values on {self.device}")
            f = arr[i]
            f.offset = h.offsets[name]
            f.type = PLY_TYPES[dict(h.properties)[name]][1]
            f.big_endian = int(h.big_endian)
            f.dst = dst.data_ptr()
            f.dst_stride = dst.stride(0)
            if affine is not None:
                f.affine = 1
                f.div, f.add, f.mul_a, f.mul_b = (float(x) for x in affine)
        with torch.cuda.device(self.device):   # the kernel launches on the current CUDA device
            check(self.lib.rg_records_to_columns(self.records.data_ptr(), h.n, h.record_bytes, arr, len(targets),
                                                 ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)),
                  None, "rg_records_to_columns")

    def columns(self, names, affine=None) -> torch.Tensor:
        out = torch.empty((self.n, len(names)), dtype=torch.float32, device=self.device)
        self.fill([(nm, out[:, j], affine) for j, nm in enumerate(names)])
        return out

    def column(self, name, affine=None) -> torch.Tensor:
        return self.columns([name], affine)[:, 0]


def _stats(n, dev):
    z = lambda: torch.zeros(n, dtype=torch.float32, device=dev)  # noqa: E731
    return {"xyz_gradient_accum_norm": z(), "num_accum": z(), "num_accum_gnv": z()}


def _default_filter_3D(n, dev):
    # log(0.0001) per Gaussian, from the float32 value (classes/point_cloud.py:393-394)
    return torch.log(torch.full((n, 1), np.float32(0.0001), dtype=torch.float32, device=dev))


def load_from_ply(path, sh_nb, sg_nb, default_density, device="cuda") -> dict:
    """``PointCloud.load_from_ply`` (classes/point_cloud.py:298-394).  x, y, z are required;
    density defaults to ``default_density``; red/green/blue are required and become the SH DC term
    ``(c / 255 - 0.5) * 2 * sqrt(pi)`` with zero higher SH and SG terms; missing sx/sy/sz become
    log sqrt of the mean squared distance to the 3 nearest neighbours (the reference's simple-knn
    initialisation); qx/qy/qz/qw default to (1, 0, 0, 0).  Returns ``{"params", "stats", "filter_3D",
    "harmonic_number", "num_sph_gauss"}``."""
    ply = PlyVertices(path, device)
    n, dev = ply.n, ply.device
    if not all(c in ply for c in ("x", "y", "z")):
        raise ValueError("No x,y,z coordinates in the pointcloud")
    if not all(c in ply for c in ("red", "green", "blue")):
        raise ValueError("No color field in the pointcloud")
    p = {"positions": ply.columns(["x", "y", "z"])}
    p["densities"] = (ply.column("density") if "density" in ply else
                      torch.full((n,), np.float32(default_density), dtype=torch.float32, device=dev))
    p["rgb"] = ply.columns(["red", "green", "blue"], affine=(255.0, -0.5, 2.0, math.sqrt(math.pi)))
    p["spherical_harmonics"] = torch.zeros((n, 3, sh_nb - 1), dtype=torch.float32, device=dev)
    p["sph_gauss_features"] = torch.zeros((n, 3, sg_nb), dtype=torch.float32, device=dev)
    p["bandwidth_sharpness"] = torch.zeros((n, sg_nb), dtype=torch.float32, device=dev)
    p["lobe_axis"] = torch.zeros((n, sg_nb, 3), dtype=torch.float32, device=dev)
    if all(c in ply for c in ("sx", "sy", "sz")):
        p["scales"] = ply.columns(["sx", "sy", "sz"])
    else:
        # log sqrt of the mean squared distance to the 3 nearest neighbours (simple-knn distCUDA2)
        from .knn import initial_log_scales
        p["scales"] = initial_log_scales(p["positions"])
    if all(c in ply for c in ("qx", "qy", "qz", "qw")):
        p["quaternions"] = ply.columns(["qx", "qy", "qz", "qw"])
    else:
        q = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        q[:, 0] = 1.0
        p["quaternions"] = q
    return {"params": p, "stats": _stats(n, dev), "filter_3D": _default_filter_3D(n, dev),
            "harmonic_number": sh_nb, "num_sph_gauss": sg_nb}


def load_from_gaussian_splatting(path, device="cuda") -> dict:
    """``PointCloud.load_from_gaussian_splatting`` (classes/point_cloud.py:396-495) for 3DGS files:
    positions x, y, z; densities = opacity as stored; scales = scale_0..2 as stored; quaternions
    rot_0..3 (zeros when absent); rgb = f_dc_0..2; the f_rest_i fields fill the SH channel-major,
    (max i + 1) / 3 coefficients per channel.  No SG terms.  filter_3D is log(0.0001) as for
    :func:`load_from_ply` (the reference leaves it as it was)."""
    ply = PlyVertices(path, device)
    n, dev = ply.n, ply.device
    if not all(c in ply for c in ("x", "y", "z")):
        raise ValueError("No x,y,z coordinates in the pointcloud")
    if "opacity" not in ply:
        raise ValueError("No opacity field in the pointcloud")
    if "scale_0" not in ply:
        raise ValueError("No scale_0 field in the pointcloud")
    if not all(c in ply for c in ("f_dc_0", "f_dc_1", "f_dc_2")):
        raise ValueError("No color field in the pointcloud")
    rest = [int(nm[7:]) for nm in ply.names if nm[:7] == "f_rest_"]
    if not rest:
        raise ValueError("No f_rest_ field in the pointcloud")
    hpc = (max(rest) + 1) // 3
    p = {"positions": ply.columns(["x", "y", "z"]), "densities": ply.column("opacity"),
         "scales": ply.columns(["scale_0", "scale_1", "scale_2"]),
         "rgb": ply.columns(["f_dc_0", "f_dc_1", "f_dc_2"])}
    if all(f"rot_{i}" in ply for i in range(4)):
        p["quaternions"] = ply.columns([f"rot_{i}" for i in range(4)])
    else:
        p["quaternions"] = torch.zeros((n, 4), dtype=torch.float32, device=dev)
    sh = torch.zeros((n, 3, hpc), dtype=torch.float32, device=dev)
    ply.fill([(f"f_rest_{c * hpc + k}", sh[:, c, k], None) for c in range(3) for k in range(hpc)])
    p["spherical_harmonics"] = sh
    p["sph_gauss_features"] = torch.zeros((n, 3, 0), dtype=torch.float32, device=dev)
    p["bandwidth_sharpness"] = torch.zeros((n, 0), dtype=torch.float32, device=dev)
    p["lobe_axis"] = torch.zeros((n, 0, 3), dtype=torch.float32, device=dev)
    return {"params": p, "stats": _stats(n, dev), "filter_3D": _default_filter_3D(n, dev),
            "harmonic_number": hpc + 1, "num_sph_gauss": 0}


_CH = "rgb"


def trained_ply_fields(harmonic_number, num_sph_gauss):
    """Field names of the trained-scene layout, in file order (convertpth_to_ply.py:60-117)."""
    names = ["x", "y", "z"]
    names += [f"sh{k}{_CH[c]}" for c in range(3) for k in range(harmonic_number)]
    names += ["density", "sx", "sy", "sz", "qx", "qy", "qz", "qw"]
    names += [f"sg{k}{_CH[c]}" for c in range(3) for k in range(num_sph_gauss)]
    names += [f"bandwidth_sharpness{k}" for k in range(num_sph_gauss)]
    names += [f"lobe_{k}{a}" for k in range(num_sph_gauss) for a in "xyz"]
    names += ["gradient_accum_norm"]
    return names


def load_trained_ply(path, device="cuda") -> dict:
    """A trained scene in the layout of the reference's convertpth_to_ply.py: every field of the
    point cloud, in one kernel launch."""
    ply = PlyVertices(path, device)
    n, dev = ply.n, ply.device
    hn = sum(1 for nm in ply.names if nm.startswith("sh") and nm.endswith("r") and nm[2:-1].isdigit())
    ns = sum(1 for nm in ply.names if nm.startswith("bandwidth_sharpness"))
    missing = [nm for nm in trained_ply_fields(hn, ns) if nm not in ply]
    if hn < 1 or missing:
        raise ValueError(f"not a trained-scene PLY (missing {missing[:5]})")
    z = lambda *s: torch.empty((n,) + s, dtype=torch.float32, device=dev)  # noqa: E731
    p = {"positions": z(3), "rgb": z(3), "spherical_harmonics": z(3, hn - 1), "densities": z(), "scales": z(3),
         "quaternions": z(4), "sph_gauss_features": z(3, ns), "bandwidth_sharpness": z(ns), "lobe_axis": z(ns, 3)}
    gacc = z()
    t = [(a, p["positions"][:, i], None) for i, a in enumerate("xyz")]
    for c in range(3):
        t.append((f"sh0{_CH[c]}", p["rgb"][:, c], None))
        t += [(f"sh{k}{_CH[c]}", p["spherical_harmonics"][:, c, k - 1], None) for k in range(1, hn)]
        t += [(f"sg{k}{_CH[c]}", p["sph_gauss_features"][:, c, k], None) for k in range(ns)]
    t.append(("density", p["densities"], None))
    t += [(a, p["scales"][:, i], None) for i, a in enumerate(("sx", "sy", "sz"))]
    t += [(a, p["quaternions"][:, i], None) for i, a in enumerate(("qx", "qy", "qz", "qw"))]
    t += [(f"bandwidth_sharpness{k}", p["bandwidth_sharpness"][:, k], None) for k in range(ns)]
    t += [(f"lobe_{k}{a}", p["lobe_axis"][:, k, i], None) for k in range(ns) for i, a in enumerate("xyz")]
    t.append(("gradient_accum_norm", gacc, None))
    ply.fill(t)
    stats = _stats(n, dev)
    stats["xyz_gradient_accum_norm"] = gacc
    return {"params": p, "stats": stats, "filter_3D": _default_filter_3D(n, dev),
            "harmonic_number": hn, "num_sph_gauss": ns}


def write_ply(path, field_list, field_names):
    """The reference's write_ply (scripts/ply.py:169-269): binary in the host byte order, one
    property per 1-D array or per column of a 2-D array, with its numpy type name."""
    fl = [np.asarray(f) for f in (field_list if isinstance(field_list, (list, tuple)) else [field_list])]
    fl = [f.reshape(-1, 1) if f.ndim < 2 else f for f in fl]
    if any(f.ndim > 2 for f in fl) or len({f.shape[0] for f in fl}) != 1:
        raise ValueError("fields must be 1-D or 2-D with one length")
    cols = [(c, f.dtype) for f in fl for c in f.T]
    if len(cols) != len(field_names):
        raise ValueError("wrong number of field names")
    path = str(path)
    if not path.endswith(".ply"):
        path += ".ply"
    head = ["ply", f"format binary_{sys.byteorder}_endian 1.0", f"element vertex {fl[0].shape[0]}"]
    head += [f"property {dt.name} {nm}" for (_, dt), nm in zip(cols, field_names)]
    head.append("end_header")
    rec = np.empty(fl[0].shape[0], dtype=[(nm, dt.str) for (_, dt), nm in zip(cols, field_names)])
    for (c, _), nm in zip(cols, field_names):
        rec[nm] = c
    with open(path, "wb") as f:
        f.write(("".join(line + "\n" for line in head)).encode())
        rec.tofile(f)
    return path


def write_trained_ply(path, params: dict, harmonic_number: int, num_sph_gauss: int,
                      gradient_accum_norm: torch.Tensor):
    """The trained-scene PLY of the reference's convertpth_to_ply.py (field order and types)."""
    np_ = {k: v.detach().cpu().numpy() for k, v in params.items()}
    colors = np.concatenate((np_["rgb"][:, :, None], np_["spherical_harmonics"]), axis=2)
    data = [np_["positions"]]
    data += [colors[:, c, k] for c in range(3) for k in range(harmonic_number)]
    data += [np_["densities"], np_["scales"], np_["quaternions"]]
    data += [np_["sph_gauss_features"][:, c, k] for c in range(3) for k in range(num_sph_gauss)]
    data += [np_["bandwidth_sharpness"][:, k] for k in range(num_sph_gauss)]
    data += [np_["lobe_axis"][:, k] for k in range(num_sph_gauss)]
    data.append(gradient_accum_norm.detach().cpu().numpy())
    return write_ply(path, data, trained_ply_fields(harmonic_number, num_sph_gauss))


# ---- checkpoints (classes/point_cloud.py:922-958) ----

def save_checkpoint(path, params: dict, harmonic_number: int, num_sph_gauss: int, stats: dict,
                    optimizer_state: dict | None, iteration: int):
    """``save_model``'s tuple: (harmonic_number, positions, rgb, spherical_harmonics, densities,
    scales, quaternions, sph_gauss_features, bandwidth_sharpness, lobe_axis, num_sph_gauss,
    xyz_gradient_accum_norm, num_accum, optimizer state dict, iteration)."""
    data = (harmonic_number, params["positions"], params["rgb"], params["spherical_harmonics"], params["densities"],
            params["scales"], params["quaternions"], params["sph_gauss_features"], params["bandwidth_sharpness"],
            params["lobe_axis"], num_sph_gauss, stats["xyz_gradient_accum_norm"], stats["num_accum"],
            optimizer_state if optimizer_state is not None else {}, iteration)
    torch.save(data, path)


def load_checkpoint(path, device="cuda") -> dict:
    """``restore_model``: the tuple of :func:`save_checkpoint` (or of the reference's save_model),
    with num_accum_gnv reset to zero and filter_3D to log(1) = 0 as the reference does."""
    data = torch.load(path, map_location=device, weights_only=False)
    names = ("positions", "rgb", "spherical_harmonics", "densities", "scales", "quaternions", "sph_gauss_features",
             "bandwidth_sharpness", "lobe_axis")
    p = {k: data[1 + i].detach().to(device).float().contiguous() for i, k in enumerate(names)}
    n = p["positions"].shape[0]
    dev = p["positions"].device
    stats = {"xyz_gradient_accum_norm": data[11].detach().to(device).float().contiguous(),
             "num_accum": data[12].detach().to(device).float().contiguous(),
             "num_accum_gnv": torch.zeros(n, dtype=torch.float32, device=dev)}
    return {"params": p, "stats": stats, "filter_3D": torch.zeros((n, 1), dtype=torch.float32, device=dev),
            "harmonic_number": int(data[0]), "num_sph_gauss": int(data[10]), "optimizer_state": data[13],
            "iteration": data[14]}


def tail_state_dict(tail) -> dict:
    """The fused tail's Adam state as the reference's OptimizerManagerDict.get_state_dict()
    (classes/optimizer.py: one torch Adam state dict per manager name)."""
    out = {}
    b1, b2 = tail.betas
    for k in tail.names:
        name = MANAGER_NAMES.get(k, k)
        group = {"lr": tail.lr[k], "betas": (b1, b2), "eps": tail.eps, "weight_decay": 0, "amsgrad": False,
                 "maximize": False, "foreach": None, "capturable": False, "differentiable": False, "fused": None,
                 "params": [0]}
        state = {}
        if tail.adam_step[k] > 0:
            state[0] = {"step": torch.tensor(float(tail.adam_step[k])), "exp_avg": tail.exp_avg[k].clone(),
                        "exp_avg_sq": tail.exp_avg_sq[k].clone()}
        out[name] = {"state": state, "param_groups": [group]}
    return out


def load_tail_state(tail, optimizer_state: dict):
    """Restore moments, step counts and learning rates from a reference-format optimizer state
    (the manager step counters restart at zero, as after the reference's restore_model)."""
    for k in tail.names:
        st = optimizer_state.get(MANAGER_NAMES.get(k, k))
        if st is None:
            continue
        s0 = st.get("state", {}).get(0)
        if s0 is not None:
            tail.exp_avg[k].copy_(s0["exp_avg"])
            tail.exp_avg_sq[k].copy_(s0["exp_avg_sq"])
            tail.adam_step[k] = int(float(s0["step"]))
        if st.get("param_groups"):
            tail.lr[k] = float(st["param_groups"][0]["lr"])
        tail.manager_step[k] = 0
