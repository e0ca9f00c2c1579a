"""CPU oracle for the RayGauss ray caster — TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (the C restatement in ``rg_oracle_impl.h``, FP32 and FP64) and,
when built, ``oracle/_ref/libref_*.so`` (the reference's own device programs compiled for the CPU
against an OptiX-emulation header).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` import this module; the product package never does.

Functions take and return numpy arrays.  ``prec`` selects the instantiation: ``"f32"`` is the
literal FP32 restatement of the reference arithmetic, ``"f64"`` the same algorithm in double.
Reference citations (paths inside the reference project):
  bbox            optix_raycasting/optix_utils.py:34-66, render_optix.py:105-106
  forward_sh      utils/sh_utils.cu:25-119
  backward_sh     utils/sh_utils.cu:121-315
  render_forward  optix_raycasting/cuda_train/forward/gaussians_aabb.cu:324-641
  render_backward optix_raycasting/cuda_train/backward/gaussians_aabb.cu:405-802
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LOCK = threading.Lock()
_LIB = None
_REF = {}


def reference_root() -> str:
    """The reference tree the ``ref`` build compiles from: $RAYGAUSS_REFERENCE, else /root/reference."""
    return os.environ.get("RAYGAUSS_REFERENCE", "/root/reference")


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and, if ``ref`` and the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    root = reference_root()
    if ref and os.path.isdir(root):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={root}"], check=True)


def _lib():
    global _LIB
    with _LOCK:
        if _LIB is None:
            path = os.path.join(_HERE, "liboracle.so")
            if not os.path.exists(path):
                build()
            _LIB = ctypes.CDLL(path)
        return _LIB


def set_grid(on: bool) -> None:
    """Candidate gathering through the nested-grid prefilter (default) or a scan of every Gaussian,
    in the restatement and, when built, in the reference programs' OptiX stand-in."""
    _lib().orc_set_grid(int(bool(on)))
    if ref_available():
        for stage in ("fwd", "bwd", "test"):
            _ref(stage).ref_set_grid(int(bool(on)))


def num_threads() -> int:
    return int(_lib().orc_num_threads())


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(_HERE, "_ref", f"libref_{s}.so")) for s in ("fwd", "bwd", "sh", "test"))


def _ref(stage: str):
    with _LOCK:
        if stage not in _REF:
            _REF[stage] = ctypes.CDLL(os.path.join(_HERE, "_ref", f"libref_{stage}.so"))
        return _REF[stage]


def _dt(prec):
    return np.float32 if prec == "f32" else np.float64


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def camera_vector(cam) -> np.ndarray:
    """14 floats: eye, U, V, W (camera axes in world, from world_view_transform[:3, 0..2]) and
    tan(FoVx/2), tan(FoVy/2) — the launch-parameter record of optix_utils.py:166-177."""
    wvt = np.asarray(cam.world_view_transform.detach().cpu().double().numpy())
    eye = np.asarray(cam.camera_center.detach().cpu().double().numpy())
    v = np.concatenate([eye, wvt[:3, 0], wvt[:3, 1], wvt[:3, 2],
                        [np.tan(cam.FoVx / 2.0), np.tan(cam.FoVy / 2.0)]])
    return v


def bbox(pos, scl, quat, dens, prec="f32"):
    dt = _dt(prec)
    pos, scl, quat, dens = (_c(a, dt) for a in (pos, scl, quat, dens))
    n = pos.shape[0]
    aabb = np.zeros((n, 6), dt)
    scene = np.zeros(6, dt)
    fn = getattr(_lib(), "orc_bbox_" + prec)
    fn(ctypes.c_int(n), _p(pos), _p(scl), _p(quat), _p(dens), _p(aabb), _p(scene))
    return aabb, scene


def forward_sh(campos, pos, sh, sg, kappa, axis, prec="f32"):
    dt = _dt(prec)
    n = pos.shape[0]
    deg = int(round(np.sqrt(sh.shape[2]))) - 1
    nsg = 0 if sg is None else sg.shape[2]
    campos, pos, sh = _c(campos, dt), _c(pos, dt), _c(sh, dt)
    sg = _c(sg if nsg else np.zeros((n, 3, 0)), dt)
    kappa = _c(kappa if nsg else np.zeros((n, 0)), dt)
    axis = _c(axis if nsg else np.zeros((n, 0, 3)), dt)
    rgb = np.zeros((n, 3), dt)
    getattr(_lib(), "orc_forward_sh_" + prec)(
        ctypes.c_int(n), _p(campos), _p(pos), _p(sh), ctypes.c_int(deg), _p(sg), _p(kappa), _p(axis),
        ctypes.c_int(nsg), _p(rgb))
    return rgb


def backward_sh(campos, pos, sh, sg, kappa, axis, drgb, prec="f32", ref_quirks=True):
    dt = _dt(prec)
    n = pos.shape[0]
    deg = int(round(np.sqrt(sh.shape[2]))) - 1
    nsg = 0 if sg is None else sg.shape[2]
    campos, pos, sh, drgb = _c(campos, dt), _c(pos, dt), _c(sh, dt), _c(drgb, dt)
    sg = _c(sg if nsg else np.zeros((n, 3, 0)), dt)
    kappa = _c(kappa if nsg else np.zeros((n, 0)), dt)
    axis = _c(axis if nsg else np.zeros((n, 0, 3)), dt)
    dsh = np.zeros(sh.shape, dt)
    dpos = np.zeros((n, 3), dt)
    dsg = np.zeros((n, 3, nsg), dt)
    dkap = np.zeros((n, nsg), dt)
    dax = np.zeros((n, nsg, 3), dt)
    getattr(_lib(), "orc_backward_sh_" + prec)(
        ctypes.c_int(n), _p(campos), _p(pos), _p(sh), ctypes.c_int(deg), _p(sg), _p(kappa), _p(axis),
        ctypes.c_int(nsg), _p(drgb), _p(dsh), _p(dpos), _p(dsg), _p(dkap), _p(dax),
        ctypes.c_int(1 if ref_quirks else 0))
    return dsh, dpos, dsg, dkap, dax


def render_forward(pos, scl, quat, dens, rgb, cam_vec, width, height, white_bg=True, max_prim_slice=1024,
                   jitter=0, rnd_sample=0, iteration=0, ray_ids=None, aabb=None, scene_box=None, prec="f32",
                   order=None):
    """Image (n_rays, 3) and final transmittance (n_rays,) of the reference forward pass.  ``order``
    (optional permutation of the Gaussians) fixes the order in which a slab's hits are summed."""
    dt = _dt(prec)
    pos, scl, quat, dens, rgb = (_c(a, dt) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, prec)
    aabb, scene_box, cam = _c(aabb, dt), _c(scene_box, dt), _c(cam_vec, dt)
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    order = None if order is None else _c(order, np.int32)
    nr = width * height if ids is None else ids.shape[0]
    out = np.zeros((nr, 3), dt)
    out_t = np.zeros(nr, dt)
    stats = np.zeros(4, np.int64)
    getattr(_lib(), "orc_render_forward_" + prec)(
        ctypes.c_int(pos.shape[0]), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box),
        _p(cam), ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(int(bool(white_bg))),
        ctypes.c_int(max_prim_slice), ctypes.c_int(jitter), ctypes.c_int(rnd_sample),
        ctypes.c_uint(iteration), _p(ids), ctypes.c_int(nr), _p(order), _p(out), _p(out_t), _p(stats))
    return out, out_t, stats


def render_backward(pos, scl, quat, dens, rgb, cam_vec, width, height, ray_colors, dL, max_prim_slice=1024,
                    jitter=0, rnd_sample=0, iteration=0, ray_ids=None, aabb=None, scene_box=None, prec="f32",
                    order=None):
    """Hand adjoint of the reference: dict of d_rgb, d_dens, d_pos, d_scl, d_quat (float64)."""
    dt = _dt(prec)
    pos, scl, quat, dens, rgb = (_c(a, dt) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, prec)
    aabb, scene_box, cam = _c(aabb, dt), _c(scene_box, dt), _c(cam_vec, dt)
    ray_colors, dL = _c(ray_colors, dt), _c(dL, dt)
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    order = None if order is None else _c(order, np.int32)
    nr = width * height if ids is None else ids.shape[0]
    n = pos.shape[0]
    g = {k: np.zeros(s, np.float64) for k, s in
         (("d_rgb", (n, 3)), ("d_dens", (n,)), ("d_pos", (n, 3)), ("d_scl", (n, 3)), ("d_quat", (n, 4)))}
    stats = np.zeros(4, np.int64)
    getattr(_lib(), "orc_render_backward_" + prec)(
        ctypes.c_int(n), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box), _p(cam),
        ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(max_prim_slice), ctypes.c_int(jitter),
        ctypes.c_int(rnd_sample), ctypes.c_uint(iteration), _p(ids), ctypes.c_int(nr), _p(order), _p(ray_colors),
        _p(dL),
        _p(g["d_rgb"]), _p(g["d_dens"]), _p(g["d_pos"]), _p(g["d_scl"]), _p(g["d_quat"]), _p(stats))
    g["stats"] = stats
    return g


def render_inference(pos, scl, quat, dens, rgb, cam_vec, width, height, white_bg=True, max_prim_slice=1024,
                     ray_ids=None, aabb=None, scene_box=None, prec="f32", order=None, count_cap=0):
    """Inference render (the reference's cuda_test programs): image (n_rays, 3) and Gaussians per
    ray (n_rays,) int32.  ``count_cap`` > 0 caps the per-slab counts without dropping hits."""
    dt = _dt(prec)
    pos, scl, quat, dens, rgb = (_c(a, dt) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, prec)
    aabb, scene_box, cam = _c(aabb, dt), _c(scene_box, dt), _c(cam_vec, dt)
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    order = None if order is None else _c(order, np.int32)
    nr = width * height if ids is None else ids.shape[0]
    out = np.zeros((nr, 3), dt)
    counts = np.zeros(nr, np.int32)
    stats = np.zeros(4, np.int64)
    getattr(_lib(), "orc_render_inference_" + prec)(
        ctypes.c_int(pos.shape[0]), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box),
        _p(cam), ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(int(bool(white_bg))),
        ctypes.c_int(max_prim_slice), ctypes.c_int(count_cap), _p(ids), ctypes.c_int(nr), _p(order), _p(out),
        _p(counts), _p(stats))
    return out, counts


# ---- the reference's own device programs, compiled for the CPU (oracle/_ref) ------------------

def ref_render_inference(pos, scl, quat, dens, rgb, cam_vec, width, height, white_bg=True, max_prim_slice=1024,
                         aabb=None, scene_box=None, ray_ids=None):
    """The reference's inference programs: image (n_rays, 3) and Gaussians per ray (n_rays,)."""
    f = np.float32
    pos, scl, quat, dens, rgb = (_c(a, f) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, "f32")
    aabb, scene_box, cam = _c(aabb, f), _c(scene_box, f), _c(cam_vec, f)
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    nr = width * height if ids is None else ids.shape[0]
    out = np.zeros((nr, 3), f)
    counts = np.zeros(nr, np.int32)
    rc = _ref("test").ref_inference(
        ctypes.c_int(pos.shape[0]), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box),
        _p(cam), ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(int(bool(white_bg))),
        ctypes.c_int(max_prim_slice), _p(ids), ctypes.c_int(0 if ids is None else ids.shape[0]), _p(out),
        _p(counts))
    assert rc == 0
    return out, counts


def ref_render_forward(pos, scl, quat, dens, rgb, cam_vec, width, height, white_bg=True, max_prim_slice=1024,
                       jitter=0, rnd_sample=0, iteration=0, aabb=None, scene_box=None, ray_ids=None):
    """The reference forward program; with ``ray_ids`` only those rays are launched and the
    full (W*H, 3) image holds zeros elsewhere."""
    f = np.float32
    pos, scl, quat, dens, rgb = (_c(a, f) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, "f32")
    aabb, scene_box, cam = _c(aabb, f), _c(scene_box, f), _c(cam_vec, f)
    out = np.zeros((width * height, 3), f)
    ovf = np.zeros(1, np.int32)
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    rc = _ref("fwd").ref_forward(
        ctypes.c_int(pos.shape[0]), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box),
        _p(cam), ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(int(bool(white_bg))),
        ctypes.c_int(max_prim_slice), ctypes.c_int(jitter), ctypes.c_int(rnd_sample), ctypes.c_uint(iteration),
        _p(ids), ctypes.c_int(0 if ids is None else ids.shape[0]), _p(out), _p(ovf))
    assert rc == 0
    return out, int(ovf[0])


def ref_render_backward(pos, scl, quat, dens, rgb, cam_vec, width, height, ray_colors, dL, max_prim_slice=1024,
                        jitter=0, rnd_sample=0, iteration=0, aabb=None, scene_box=None, ray_ids=None):
    f = np.float32
    pos, scl, quat, dens, rgb = (_c(a, f) for a in (pos, scl, quat, dens, rgb))
    if aabb is None or scene_box is None:
        aabb, scene_box = bbox(pos, scl, quat, dens, "f32")
    aabb, scene_box, cam = _c(aabb, f), _c(scene_box, f), _c(cam_vec, f)
    ray_colors, dL = _c(ray_colors, f), _c(dL, f)
    n = pos.shape[0]
    g = {k: np.zeros(s, f) for k, s in
         (("d_rgb", (n, 3)), ("d_dens", (n,)), ("d_pos", (n, 3)), ("d_scl", (n, 3)), ("d_quat", (n, 4)))}
    ids = None if ray_ids is None else _c(ray_ids, np.int32)
    rc = _ref("bwd").ref_backward(
        ctypes.c_int(n), _p(pos), _p(scl), _p(quat), _p(dens), _p(rgb), _p(aabb), _p(scene_box), _p(cam),
        ctypes.c_int(width), ctypes.c_int(height), ctypes.c_int(max_prim_slice), ctypes.c_int(jitter),
        ctypes.c_int(rnd_sample), ctypes.c_uint(iteration), _p(ids), ctypes.c_int(0 if ids is None else ids.shape[0]),
        _p(ray_colors), _p(dL), _p(g["d_dens"]),
        _p(g["d_rgb"]), _p(g["d_pos"]), _p(g["d_scl"]), _p(g["d_quat"]))
    assert rc == 0
    return g


def ref_forward_sh(campos, pos, sh, sg, kappa, axis):
    f = np.float32
    n = pos.shape[0]
    deg = int(round(np.sqrt(sh.shape[2]))) - 1
    nsg = 0 if sg is None else sg.shape[2]
    campos, pos, sh = _c(campos, f), _c(pos, f), _c(sh, f)
    sg = _c(sg if nsg else np.zeros((n, 3, 0)), f)
    kappa = _c(kappa if nsg else np.zeros((n, 0)), f)
    axis = _c(axis if nsg else np.zeros((n, 0, 3)), f)
    rgb = np.zeros((n, 3), f)
    _ref("sh").ref_forward_sh(_p(campos), _p(pos), _p(sh), _p(sg), _p(kappa), _p(axis), ctypes.c_uint(nsg),
                              ctypes.c_int(deg), ctypes.c_int(n), _p(rgb))
    return rgb


def ref_backward_sh(campos, pos, sh, sg, kappa, axis, drgb):
    f = np.float32
    n = pos.shape[0]
    deg = int(round(np.sqrt(sh.shape[2]))) - 1
    nsg = 0 if sg is None else sg.shape[2]
    campos, pos, sh, drgb = _c(campos, f), _c(pos, f), _c(sh, f), _c(drgb, f)
    sg = _c(sg if nsg else np.zeros((n, 3, 0)), f)
    kappa = _c(kappa if nsg else np.zeros((n, 0)), f)
    axis = _c(axis if nsg else np.zeros((n, 0, 3)), f)
    dsh = np.zeros(sh.shape, f)
    dpos = np.zeros((n, 3), f)
    dsg = np.zeros((n, 3, nsg), f)
    dkap = np.zeros((n, nsg), f)
    dax = np.zeros((n, nsg, 3), f)
    _ref("sh").ref_backward_sh(_p(campos), _p(pos), _p(sh), _p(sg), _p(kappa), _p(axis), ctypes.c_uint(nsg),
                               ctypes.c_int(deg), ctypes.c_int(n), _p(drgb), _p(dsh), _p(dpos), _p(dsg),
                               _p(dkap), _p(dax))
    return dsh, dpos, dsg, dkap, dax
