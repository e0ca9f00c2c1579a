"""The C-ABI library: it builds for sm_100a, loads, exports every symbol include/raygauss_b200.h
declares, and its structs have the layout the Python binding assumes.  No GPU compute here."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "raygauss_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^RG_API\s+[\w\s\*]+?\b(rg_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("rg_create", "rg_destroy", "rg_ellipsoids_bbox", "rg_bvh_build", "rg_bvh_refit", "rg_forward_sh",
              "rg_launch_forward", "rg_launch_backward", "rg_backward_sh", "rg_render_forward",
              "rg_render_backward", "rg_get_status"):
        assert s in syms


def test_library_exports_every_declared_symbol(engine_lib):
    from ray_gauss_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(rg_\w+)", out.stdout))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(engine_lib, s)
        if s in _lib.SIGNATURES:
            assert getattr(engine_lib, s).argtypes is not None


def test_build_targets_sm100a_only():
    mk = open(os.path.join(ROOT, "ray_gauss_b200", "csrc", "Makefile")).read()
    arch = re.findall(r"-gencode\s+arch=(\S+)", mk)
    assert arch == ["compute_100a,code=sm_100a"]


def test_struct_layout_matches_c(tmp_path):
    from ray_gauss_b200 import _lib
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "raygauss_b200.h"\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(rg_camera),'
                   ' sizeof(rg_gaussians), sizeof(rg_settings), sizeof(rg_gradients), sizeof(rg_status),'
                   ' sizeof(rg_tuning), offsetof(rg_gaussians, n), offsetof(rg_camera, width),'
                   ' offsetof(rg_settings, mode)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    expect = [ctypes.sizeof(_lib.rg_camera), ctypes.sizeof(_lib.rg_gaussians), ctypes.sizeof(_lib.rg_settings),
              ctypes.sizeof(_lib.rg_gradients), ctypes.sizeof(_lib.rg_status), ctypes.sizeof(_lib.rg_tuning),
              _lib.rg_gaussians.n.offset, _lib.rg_camera.width.offset, _lib.rg_settings.mode.offset]
    assert vals == expect


def test_error_strings_and_abi(engine_lib):
    assert engine_lib.rg_abi_version() == 3
    assert engine_lib.rg_error_string(0) == b"ok"
    assert b"invalid" in engine_lib.rg_error_string(1)
    assert engine_lib.rg_error_string(99) == b"unknown error"


def test_invalid_arguments_rejected_without_gpu(engine_lib):
    from ray_gauss_b200 import _lib
    # null output handle
    assert engine_lib.rg_create(None, 0) == 1
    # null engine on every entry point
    assert engine_lib.rg_reserve(None, 10, 1, 0) == 1
    assert engine_lib.rg_ellipsoids_bbox(None, None, None, None, None) == 1
    assert engine_lib.rg_bvh_build(None, None) == 4
    assert engine_lib.rg_launch_forward(None, None, 1, None, None, None, None) == 1
    st = _lib.rg_status()
    assert engine_lib.rg_get_status(None, ctypes.byref(st), 0, None) == 1
    assert engine_lib.rg_noalloc_get_status(None, None) == 1
    assert engine_lib.rg_render_forward_noalloc(None, None, 1, None, None, None, None) == 1
    assert engine_lib.rg_destroy(None) == 0


def test_create_without_device_fails_cleanly(engine_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert engine_lib.rg_create(ctypes.byref(h), 0) == 1
    assert not h.value
