"""Host-side engine: owns one ``rg_engine`` (C ABI) per CUDA device and turns torch tensors into
the C structs.  All calls are ordered on torch's current CUDA stream and never synchronise.

PyTorch supplies device memory and streams only; every kernel is in the engine library.
"""
from __future__ import annotations

import ctypes
import math
import threading
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check

_ENGINES: dict[int, "Engine"] = {}
_ENG_LOCK = threading.Lock()


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(device):
    """torch's current stream on ``device`` (the engine entry points make the engine's device
    current for the call and restore the caller's device afterwards)."""
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


@dataclass
class GaussianBatch:
    """The rg_gaussians struct plus references that keep its tensors alive."""
    struct: _lib.rg_gaussians
    keep: tuple
    n: int
    sh_degree: int
    nsg: int
    storage: int


def _as_storage(t, storage):
    want = torch.bfloat16 if storage == _lib.RG_STORAGE_BF16 else torch.float32
    return t.detach().to(want).contiguous()


def make_gaussians(positions, scales, quaternions, densities, color_features, sph_gauss_features=None,
                   bandwidth_sharpness=None, lobe_axis=None, storage=None) -> GaussianBatch:
    """Validate shapes/dtypes (the reference contract, classes/point_cloud.py:729-739) and build the
    C struct.  ``storage`` defaults to BF16 when colour features are stored in bfloat16."""
    n = positions.shape[0]
    if positions.shape != (n, 3) or scales.shape != (n, 3) or quaternions.shape != (n, 4):
        raise ValueError("positions/scales must be (N,3) and quaternions (N,4)")
    if densities.reshape(-1).shape[0] != n:
        raise ValueError("densities must have N entries")
    if color_features.dim() != 3 or color_features.shape[0] != n or color_features.shape[1] != 3:
        raise ValueError("color_features must be (N,3,(deg+1)^2)")
    ncoef = color_features.shape[2]
    deg = int(round(math.sqrt(ncoef))) - 1
    if (deg + 1) ** 2 != ncoef or deg > 3:
        raise ValueError("color_features last dim must be 1, 4, 9 or 16")
    nsg = 0 if sph_gauss_features is None or sph_gauss_features.numel() == 0 else sph_gauss_features.shape[2]
    if nsg > _lib.RG_MAX_SG:
        raise ValueError(f"at most {_lib.RG_MAX_SG} spherical Gaussians per point")
    if storage is None:
        storage = _lib.RG_STORAGE_BF16 if color_features.dtype == torch.bfloat16 else _lib.RG_STORAGE_F32
    dev = positions.device
    if dev.type != "cuda":
        raise ValueError("the ray caster runs on CUDA tensors only")
    for t in (scales, quaternions, densities, color_features, sph_gauss_features, bandwidth_sharpness, lobe_axis):
        if t is not None and t.numel() and t.device != dev:
            raise ValueError("every Gaussian tensor must be on the positions' CUDA device")
    f32 = lambda t: t.detach().to(torch.float32).contiguous()
    pos, scl, quat = f32(positions), f32(scales), f32(quaternions)
    if quat.data_ptr() % 16:
        quat = quat.clone()
    dens = _as_storage(densities.reshape(-1), storage)
    col = _as_storage(color_features, storage)
    if nsg:
        sg = _as_storage(sph_gauss_features, storage)
        kap = f32(bandwidth_sharpness)
        ax = f32(lobe_axis)
        if sg.shape != (n, 3, nsg) or kap.shape != (n, nsg) or ax.shape != (n, nsg, 3):
            raise ValueError("SG tensors must be (N,3,nsg), (N,nsg), (N,nsg,3)")
    else:
        sg = kap = ax = None
    s = _lib.rg_gaussians()
    s.positions, s.scales, s.quaternions = pos.data_ptr(), scl.data_ptr(), quat.data_ptr()
    s.densities, s.color_features = dens.data_ptr(), col.data_ptr()
    s.sph_gauss_features = sg.data_ptr() if nsg else None
    s.bandwidth_sharpness = kap.data_ptr() if nsg else None
    s.lobe_axis = ax.data_ptr() if nsg else None
    s.n, s.sh_degree, s.num_sph_gauss, s.storage = n, deg, nsg, storage
    return GaussianBatch(s, (pos, scl, quat, dens, col, sg, kap, ax), n, deg, nsg, storage)


def camera_record(cam, supersampling=(1, 1)) -> _lib.rg_camera:
    """rg_camera of a reference-style camera (optix_utils.py:166-177): eye, world_view_transform[:3,0..2],
    tan(FoV/2), ray grid = image size x supersampling."""
    wvt = cam.world_view_transform.detach().to("cpu", torch.float32)
    eye = cam.camera_center.detach().to("cpu", torch.float32)
    r = _lib.rg_camera()
    for i in range(3):
        r.eye[i] = float(eye[i])
        r.u[i] = float(wvt[i, 0])
        r.v[i] = float(wvt[i, 1])
        r.w[i] = float(wvt[i, 2])
    r.tan_half_fovx = math.tan(cam.FoVx / 2.0)
    r.tan_half_fovy = math.tan(cam.FoVy / 2.0)
    r.width = int(cam.image_width) * int(supersampling[0])
    r.height = int(cam.image_height) * int(supersampling[1])
    return r


def cameras_tensor(records, device) -> torch.Tensor:
    """Pack rg_camera records into a device byte tensor (the kernels read cameras from device memory)."""
    n = len(records)
    buf = (_lib.rg_camera * n)(*records)
    host = torch.frombuffer(bytearray(bytes(buf)), dtype=torch.uint8)
    return host.to(device, non_blocking=False)


def settings_struct(white_background=True, jitter=0, rnd_sample=0, max_prim_slice=1024, iteration=0,
                    mode=_lib.RG_MODE_PARITY, sh_quirk=True) -> _lib.rg_settings:
    s = _lib.rg_settings()
    s.white_background = int(bool(white_background))
    s.jitter = int(jitter)
    s.rnd_sample = int(rnd_sample)
    s.max_prim_slice = int(max_prim_slice)
    s.iteration = int(iteration) & 0xFFFFFFFF
    s.mode = int(mode)
    s.sh_quirk = int(bool(sh_quirk))
    return s


class Engine:
    """One rg_engine on one CUDA device."""

    def __init__(self, device=None):
        self.lib = _lib.load()
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device if isinstance(device, int) else torch.device(device).index or 0)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(self.lib.rg_create(ctypes.byref(h), self.device.index), None, "rg_create")
        self.h = h
        self.generation = 0          # bumped by every BVH build/refit and colour pass
        self._cam_cache = {}
        self.timers = None           # optional {step name: [(start, end) cuda events]}
        self._built_n = -1

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.rg_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # -- plumbing -------------------------------------------------------------------------------
    def reserve(self, n, n_views=1, n_rays=0):
        check(self.lib.rg_reserve(self.h, int(n), int(n_views), int(n_rays)), self.h, "rg_reserve")

    def set_tuning(self, chunk_slabs=None, blocks_per_sm=None, list_capacity=None, record_hits=None,
                   diagnostics=None):
        """Change the given values and keep the others.  blocks_per_sm 0: as many as fit;
        record_hits 1 / -1 switches the forward's hit-list record on / off; diagnostics 1 makes the
        render kernels count node visits, leaf tests, list entries, slab steps and entry-slabs."""
        cur = self.get_tuning()
        new = dict(chunk_slabs=chunk_slabs, blocks_per_sm=blocks_per_sm, list_capacity=list_capacity,
                   record_hits=record_hits, diagnostics=diagnostics)
        cur.update({k: int(v) for k, v in new.items() if v is not None})
        t = _lib.rg_tuning(cur["chunk_slabs"], cur["blocks_per_sm"], cur["list_capacity"], cur["record_hits"],
                           cur["diagnostics"])
        check(self.lib.rg_set_tuning(self.h, ctypes.byref(t)), self.h, "rg_set_tuning")

    def get_tuning(self):
        t = _lib.rg_tuning()
        check(self.lib.rg_get_tuning(self.h, ctypes.byref(t)), self.h, "rg_get_tuning")
        return dict(chunk_slabs=t.chunk_slabs, blocks_per_sm=t.blocks_per_sm, list_capacity=t.list_capacity,
                    record_hits=t.record_hits, diagnostics=t.diagnostics)

    def status(self, reset=False):
        st = _lib.rg_status()
        check(self.lib.rg_get_status(self.h, ctypes.byref(st), int(bool(reset)), _stream(self.device)), self.h, "rg_get_status")
        return {k: int(getattr(st, k)) for k, _ in _lib.rg_status._fields_}

    def leaf_order(self, n):
        out = torch.empty((n,), dtype=torch.int32, device=self.device)
        check(self.lib.rg_leaf_order(self.h, _ptr(out), _stream(self.device)), self.h, "rg_leaf_order")
        return out

    def kernel_launches(self) -> int:
        return int(self.lib.rg_kernel_launches(self.h))

    def cameras(self, cams, supersampling=(1, 1)):
        """Device camera table for a list of reference-style cameras (cached per camera object)."""
        key = tuple((id(c), c.world_view_transform.data_ptr(), c.world_view_transform._version,
                     c.camera_center._version, float(c.FoVx), float(c.FoVy), int(c.image_width),
                     int(c.image_height)) for c in cams) + (tuple(supersampling),)
        hit = self._cam_cache.get(key)
        if hit is not None:
            return hit
        recs = [camera_record(c, supersampling) for c in cams]
        t = cameras_tensor(recs, self.device)
        if len(self._cam_cache) > 256:
            self._cam_cache.clear()
        self._cam_cache[key] = (t, recs, cams)
        return self._cam_cache[key]

    def _timed(self, name):
        return _Timer(self.timers, name)

    # -- the C-ABI steps ----------------------------------------------------------------------------
    def ellipsoids_bbox(self, g: GaussianBatch, aabb_out=None, scene_box_out=None):
        check(self.lib.rg_ellipsoids_bbox(self.h, ctypes.byref(g.struct), _ptr(aabb_out), _ptr(scene_box_out),
                                          _stream(self.device)), self.h, "rg_ellipsoids_bbox")

    def bvh_build(self):
        check(self.lib.rg_bvh_build(self.h, _stream(self.device)), self.h, "rg_bvh_build")
        self.generation += 1

    def bvh_refit(self):
        check(self.lib.rg_bvh_refit(self.h, _stream(self.device)), self.h, "rg_bvh_refit")
        self.generation += 1

    def forward_sh(self, g: GaussianBatch, cams_t, n_cams, rgb_out=None):
        check(self.lib.rg_forward_sh(self.h, ctypes.byref(g.struct), _ptr(cams_t), int(n_cams), _ptr(rgb_out),
                                     _stream(self.device)), self.h, "rg_forward_sh")
        self.generation += 1

    def launch_forward(self, cams_t, n_cams, settings, ray_colors, final_T=None):
        with self._timed("launch_forward"):
                check(self.lib.rg_launch_forward(self.h, _ptr(cams_t), int(n_cams), ctypes.byref(settings),
                                             _ptr(ray_colors), _ptr(final_T), _stream(self.device)), self.h, "rg_launch_forward")

    def launch_backward(self, cams_t, n_cams, settings, ray_colors, dL):
        with self._timed("launch_backward"):
            check(self.lib.rg_launch_backward(self.h, _ptr(cams_t), int(n_cams), ctypes.byref(settings),
                                              _ptr(ray_colors), _ptr(dL), _stream(self.device)), self.h, "rg_launch_backward")

    def backward_sh(self, g: GaussianBatch, cams_t, n_cams, settings, grads: dict):
        s = _lib.rg_gradients()
        for k in ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
                  "bandwidth_sharpness", "lobe_axis"):
            t = grads.get(k)
            setattr(s, k, t.data_ptr() if t is not None else None)
        check(self.lib.rg_backward_sh(self.h, ctypes.byref(g.struct), _ptr(cams_t), int(n_cams), ctypes.byref(settings),
                                      ctypes.byref(s), _stream(self.device)), self.h, "rg_backward_sh")

    # -- composite steps (RenderOptixFunction forward/backward) --------------------------------------
    def render_forward(self, g: GaussianBatch, cams_t, n_cams, n_rays, settings, refit=False, final_T=False,
                       rgb_out=None):
        """RenderOptixFunction.forward: bbox -> BVH build (or refit) -> colour -> forward launch."""
        ray_colors = torch.empty((n_rays, 3), dtype=torch.float32, device=self.device)
        fT = torch.empty((n_rays,), dtype=torch.float32, device=self.device) if final_T else None
        self.reserve(0, 0, n_rays)   # sizes the hit-list record once per ray count (no-op afterwards)
        with self._timed("prepare"):
            self.ellipsoids_bbox(g)
            if refit and self._built_n == g.n:
                self.bvh_refit()
            else:
                self.bvh_build()
                self._built_n = g.n
            self.forward_sh(g, cams_t, n_cams, rgb_out)
        self.launch_forward(cams_t, n_cams, settings, ray_colors, fT)
        return ray_colors, fT

    def launch_inference(self, cams_t, n_cams, settings, ray_colors, counts=None):
        with self._timed("launch_inference"):
            check(self.lib.rg_launch_inference(self.h, _ptr(cams_t), int(n_cams), ctypes.byref(settings),
                                               _ptr(ray_colors), _ptr(counts), _stream(self.device)), self.h,
                  "rg_launch_inference")

    def render_inference(self, g: GaussianBatch, cams_t, n_cams, n_rays, settings, refit=False, counts=False):
        """Inference render (optix_utils.py:302-373 with the cuda_test programs): bbox -> BVH build
        (or refit) -> colour -> inference launch.  Returns (ray colours (R,3), Gaussians per ray
        (R,) int32 or None)."""
        ray_colors = torch.empty((n_rays, 3), dtype=torch.float32, device=self.device)
        cnt = torch.empty((n_rays,), dtype=torch.int32, device=self.device) if counts else None
        with self._timed("prepare"):
            self.ellipsoids_bbox(g)
            if refit and self._built_n == g.n:
                self.bvh_refit()
            else:
                self.bvh_build()
                self._built_n = g.n
            self.forward_sh(g, cams_t, n_cams)
        self.launch_inference(cams_t, n_cams, settings, ray_colors, cnt)
        return ray_colors, cnt

    def alloc_grads(self, g: GaussianBatch):
        n, dev = g.n, self.device
        f = dict(dtype=torch.float32, device=dev)
        out = dict(positions=torch.empty((n, 3), **f), scales=torch.empty((n, 3), **f),
                   quaternions=torch.empty((n, 4), **f), densities=torch.empty((n,), **f),
                   color_features=torch.empty((n, 3, (g.sh_degree + 1) ** 2), **f))
        if g.nsg:
            out["sph_gauss_features"] = torch.empty((n, 3, g.nsg), **f)
            out["bandwidth_sharpness"] = torch.empty((n, g.nsg), **f)
            out["lobe_axis"] = torch.empty((n, g.nsg, 3), **f)
        return out

    def render_backward(self, g: GaussianBatch, cams_t, n_cams, settings, ray_colors, dL, grads=None):
        grads = grads if grads is not None else self.alloc_grads(g)
        s = _lib.rg_gradients()
        for k in ("positions", "scales", "quaternions", "densities", "color_features", "sph_gauss_features",
                  "bandwidth_sharpness", "lobe_axis"):
            t = grads.get(k)
            setattr(s, k, t.data_ptr() if t is not None else None)
        self.launch_backward(cams_t, n_cams, settings, ray_colors, dL)
        with self._timed("backward_sh"):
            check(self.lib.rg_backward_sh(self.h, ctypes.byref(g.struct), _ptr(cams_t), int(n_cams),
                                          ctypes.byref(settings), ctypes.byref(s), _stream(self.device)), self.h, "rg_backward_sh")
        return grads


class _Timer:
    def __init__(self, timers, name):
        self.timers, self.name = timers, name

    def __enter__(self):
        if self.timers is not None:
            self.ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            self.ev[0].record()
        return self

    def __exit__(self, *exc):
        if self.timers is not None:
            self.ev[1].record()
            self.timers.setdefault(self.name, []).append(self.ev)
        return False


def engine_for(device) -> Engine:
    """The process-wide engine of a CUDA device (created on first use)."""
    idx = torch.device(device).index
    if idx is None:
        idx = torch.cuda.current_device()
    with _ENG_LOCK:
        e = _ENGINES.get(idx)
        if e is None:
            e = Engine(idx)
            _ENGINES[idx] = e
        return e
