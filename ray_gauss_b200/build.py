"""In-tree build of the engine library (sm_100a) with nvcc via ray_gauss_b200/csrc/Makefile."""
from __future__ import annotations

import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))


def build_library(verbose: bool = False) -> str:
    """Compile ray_gauss_b200/_lib/libraygauss_b200.so (incremental) and return its path."""
    cmd = ["make", "-C", os.path.join(_HERE, "csrc"), "-j8"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("engine build failed:\n" + (out.stdout or "") + (out.stderr or ""))
    return os.path.join(_HERE, "_lib", "libraygauss_b200.so")
