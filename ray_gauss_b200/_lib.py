"""ctypes binding of the engine's C ABI (include/raygauss_b200.h).

The shared library ``ray_gauss_b200/_lib/libraygauss_b200.so`` is built in-tree from
``ray_gauss_b200/csrc`` (``ray_gauss_b200.build.build_library``).  There is no fallback: if the
library is missing or cannot be loaded, importing the engine raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libraygauss_b200.so")

RG_OK = 0
RG_STORAGE_F32 = 0
RG_STORAGE_BF16 = 1
RG_MODE_PARITY = 0
RG_MODE_FAST = 1
RG_MAX_SG = 16
MAX_VIEWS = 64

ERRORS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "call order violated", 5: "capacity exceeded"}


class rg_camera(ctypes.Structure):
    _fields_ = [("eye", ctypes.c_float * 3), ("u", ctypes.c_float * 3), ("v", ctypes.c_float * 3),
                ("w", ctypes.c_float * 3), ("tan_half_fovx", ctypes.c_float), ("tan_half_fovy", ctypes.c_float),
                ("width", ctypes.c_int32), ("height", ctypes.c_int32)]


class rg_gaussians(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("scales", ctypes.c_void_p), ("quaternions", ctypes.c_void_p),
                ("densities", ctypes.c_void_p), ("color_features", ctypes.c_void_p),
                ("sph_gauss_features", ctypes.c_void_p), ("bandwidth_sharpness", ctypes.c_void_p),
                ("lobe_axis", ctypes.c_void_p), ("n", ctypes.c_int64), ("sh_degree", ctypes.c_int32),
                ("num_sph_gauss", ctypes.c_int32), ("storage", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class rg_settings(ctypes.Structure):
    _fields_ = [("white_background", ctypes.c_int32), ("jitter", ctypes.c_int32), ("rnd_sample", ctypes.c_int32),
                ("max_prim_slice", ctypes.c_int32), ("iteration", ctypes.c_uint32), ("mode", ctypes.c_int32),
                ("sh_quirk", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class rg_gradients(ctypes.Structure):
    _fields_ = [("positions", ctypes.c_void_p), ("scales", ctypes.c_void_p), ("quaternions", ctypes.c_void_p),
                ("densities", ctypes.c_void_p), ("color_features", ctypes.c_void_p),
                ("sph_gauss_features", ctypes.c_void_p), ("bandwidth_sharpness", ctypes.c_void_p),
                ("lobe_axis", ctypes.c_void_p)]


class rg_status(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("hit_pairs", "slabs", "slab_cap_exceeded", "list_passes",
                                                "chunk_splits", "stack_overflows", "watchdog_trips",
                                                "nonfinite_inputs", "traversals", "node_visits", "leaf_tests",
                                                "list_entries", "slab_steps", "entry_slabs", "replayed_chunks",
                                                "record_overflows", "record_words")]


class rg_tuning(ctypes.Structure):
    _fields_ = [("chunk_slabs", ctypes.c_int32), ("blocks_per_sm", ctypes.c_int32),
                ("list_capacity", ctypes.c_int32), ("record_hits", ctypes.c_int32), ("diagnostics", ctypes.c_int32)]


RG_TAIL_MAX_TENSORS = 12


class rg_adam_tensor(ctypes.Structure):
    _fields_ = [("param", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("exp_avg", ctypes.c_void_p),
                ("exp_avg_sq", ctypes.c_void_p), ("width", ctypes.c_int32), ("active", ctypes.c_int32),
                ("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("one_minus_beta1", ctypes.c_float), ("one_minus_beta2", ctypes.c_float),
                ("bias1", ctypes.c_float), ("bias2_sqrt", ctypes.c_float)]


class rg_train_tail(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("n_tensors", ctypes.c_int32), ("idx_positions", ctypes.c_int32),
                ("idx_densities", ctypes.c_int32), ("idx_scales", ctypes.c_int32), ("idx_quaternions", ctypes.c_int32),
                ("idx_lobe_axis", ctypes.c_int32), ("normalize_quaternions", ctypes.c_int32),
                ("normalize_lobe_axis", ctypes.c_int32), ("max_scale", ctypes.c_float), ("min_scale", ctypes.c_void_p),
                ("grad_norm_accum", ctypes.c_void_p), ("num_accum", ctypes.c_void_p),
                ("num_accum_gnv", ctypes.c_void_p), ("step_scalars", ctypes.c_void_p),
                ("tensors", rg_adam_tensor * RG_TAIL_MAX_TENSORS)]


RG_RECORD_MAX_FIELDS = 1024
RG_FIELD_I8, RG_FIELD_U8, RG_FIELD_I16, RG_FIELD_U16, RG_FIELD_I32, RG_FIELD_U32, RG_FIELD_F32, RG_FIELD_F64 = range(8)


class rg_record_field(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_int32), ("type", ctypes.c_int32), ("big_endian", ctypes.c_int32),
                ("affine", ctypes.c_int32), ("dst", ctypes.c_void_p), ("dst_stride", ctypes.c_int64),
                ("div", ctypes.c_double), ("add", ctypes.c_double), ("mul_a", ctypes.c_double),
                ("mul_b", ctypes.c_double)]


RG_DENSIFY_MAX_TENSORS = 48
RG_DENSIFY_COPY, RG_DENSIFY_OLD_ONLY, RG_DENSIFY_ZERO, RG_DENSIFY_DENSITIES, RG_DENSIFY_LOG_SCALES, \
    RG_DENSIFY_POSITIONS = range(6)


class rg_densify_tensor(ctypes.Structure):
    _fields_ = [("src", ctypes.c_void_p), ("dst", ctypes.c_void_p), ("width", ctypes.c_int32),
                ("kind", ctypes.c_int32)]


class rg_densify(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("grad_accum", ctypes.c_void_p), ("num_accum", ctypes.c_void_p),
                ("log_scales", ctypes.c_void_p), ("quaternions", ctypes.c_void_p), ("densities", ctypes.c_void_p),
                ("grad_threshold", ctypes.c_float), ("scale_threshold", ctypes.c_float),
                ("min_density", ctypes.c_float), ("split_scale_mul", ctypes.c_float), ("n_split", ctypes.c_int32),
                ("planned", ctypes.c_int32), ("workspace", ctypes.c_void_p), ("n_clone", ctypes.c_int64),
                ("n_split_sel", ctypes.c_int64), ("n_out", ctypes.c_int64), ("n_kept", ctypes.c_int64),
                ("kept_clones", ctypes.c_int64), ("kept_splits", ctypes.c_int64)]


assert ctypes.sizeof(rg_camera) == 64
assert ctypes.sizeof(rg_gaussians) == 88
assert ctypes.sizeof(rg_settings) == 32

# name -> (restype, argtypes)
_P = ctypes.c_void_p
SIGNATURES = {
    "rg_abi_version": (ctypes.c_int, []),
    "rg_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "rg_last_cuda_error": (ctypes.c_char_p, [_P]),
    "rg_kernel_launches": (ctypes.c_uint64, [_P]),
    "rg_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int]),
    "rg_destroy": (ctypes.c_int, [_P]),
    "rg_reserve": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64]),
    "rg_set_tuning": (ctypes.c_int, [_P, ctypes.POINTER(rg_tuning)]),
    "rg_get_tuning": (ctypes.c_int, [_P, ctypes.POINTER(rg_tuning)]),
    "rg_ellipsoids_bbox": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, _P, _P]),
    "rg_bvh_build": (ctypes.c_int, [_P, _P]),
    "rg_bvh_refit": (ctypes.c_int, [_P, _P]),
    "rg_forward_sh": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32, _P, _P]),
    "rg_launch_forward": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.POINTER(rg_settings), _P, _P, _P]),
    "rg_launch_backward": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.POINTER(rg_settings), _P, _P, _P]),
    "rg_launch_inference": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.POINTER(rg_settings), _P, _P, _P]),
    "rg_render_inference": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32,
                                           ctypes.POINTER(rg_settings), ctypes.c_int32, _P, _P, _P, _P]),
    "rg_backward_sh": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32,
                                      ctypes.POINTER(rg_settings), ctypes.POINTER(rg_gradients), _P]),
    "rg_render_forward": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32,
                                         ctypes.POINTER(rg_settings), ctypes.c_int32, _P, _P, _P, _P]),
    "rg_render_backward": (ctypes.c_int, [_P, ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32,
                                          ctypes.POINTER(rg_settings), _P, _P, ctypes.POINTER(rg_gradients), _P]),
    "rg_get_status": (ctypes.c_int, [_P, ctypes.POINTER(rg_status), ctypes.c_int32, _P]),
    "rg_leaf_order": (ctypes.c_int, [_P, _P, _P]),
    "rg_render_forward_noalloc": (ctypes.c_int, [ctypes.POINTER(rg_gaussians), _P, ctypes.c_int32,
                                                 ctypes.POINTER(rg_settings), _P, _P, _P]),
    "rg_noalloc_get_status": (ctypes.c_int, [ctypes.POINTER(rg_status), _P]),
    "rg_train_tail_step": (ctypes.c_int, [ctypes.POINTER(rg_train_tail), _P]),
    "rg_records_to_columns": (ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(rg_record_field),
                                             ctypes.c_int32, _P]),
    "rg_compute_3d_filter": (ctypes.c_int, [_P, ctypes.c_int64, _P, ctypes.c_int32, ctypes.c_float, _P, _P, _P, _P]),
    "rg_knn_workspace_bytes": (ctypes.c_int, [ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]),
    "rg_knn_mean_dist": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, _P]),
    "rg_densify_workspace_bytes": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "rg_densify_plan": (ctypes.c_int, [ctypes.POINTER(rg_densify), _P]),
    "rg_densify_apply": (ctypes.c_int, [ctypes.POINTER(rg_densify), _P, ctypes.POINTER(rg_densify_tensor),
                                        ctypes.c_int32, _P]),
}

_LOCK = threading.Lock()
_LIB = None


def load(path: str = LIB_PATH):
    """Load the engine library (raises if it is missing; there is no CPU fallback)."""
    global _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not os.path.exists(path):
            raise RuntimeError(f"raygauss_b200 CUDA library not built: {path} is missing "
                               "(run ray_gauss_b200.build.build_library())")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.rg_abi_version() != 3:
            raise RuntimeError("raygauss_b200 ABI version mismatch")
        _LIB = lib
        return lib


class RgError(RuntimeError):
    pass


def check(rc: int, engine_handle=None, what: str = "") -> None:
    if rc == RG_OK:
        return
    msg = ERRORS.get(rc, f"error {rc}")
    detail = ""
    if engine_handle is not None and _LIB is not None:
        d = _LIB.rg_last_cuda_error(engine_handle)
        detail = d.decode() if d else ""
    raise RgError(f"{what}: {msg}" + (f" ({detail})" if detail else ""))
