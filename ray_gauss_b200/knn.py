"""Mean squared distance to the three nearest neighbours (the simple-knn extension's distCUDA2,
submodules/simple-knn/spatial.cu:14-25), the initial scale of a point cloud without scales
(classes/point_cloud.py:374-378): ``scales = log(sqrt(clamp_min(dist_cuda2(points), 1e-7)))``."""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from ._lib import check


def dist_cuda2(points: torch.Tensor) -> torch.Tensor:
    """(N,) mean of the three smallest squared distances from each point to the others (exact;
    missing neighbours count as FLT_MAX like the extension: two neighbours give about FLT_MAX / 3,
    one or none +inf)."""
    if points.dtype != torch.float32 or not points.is_contiguous() or points.dim() != 2 or points.shape[1] != 3:
        raise ValueError("points: (N, 3) FP32 contiguous")
    if not points.is_cuda:
        raise ValueError("dist_cuda2 runs on CUDA tensors")
    n = points.shape[0]
    lib = _lib.load()
    nb = ctypes.c_uint64()
    check(lib.rg_knn_workspace_bytes(n, ctypes.byref(nb)), None, "rg_knn_workspace_bytes")
    ws = torch.empty(int(nb.value), dtype=torch.uint8, device=points.device)
    out = torch.empty(n, dtype=torch.float32, device=points.device)
    with torch.cuda.device(points.device):   # the kernels launch on the current CUDA device
        check(lib.rg_knn_mean_dist(points.data_ptr(), n, out.data_ptr(), ws.data_ptr(),
                                   ctypes.c_void_p(torch.cuda.current_stream(points.device).cuda_stream)),
              None, "rg_knn_mean_dist")
    return out


def initial_log_scales(points: torch.Tensor) -> torch.Tensor:
    """(N, 3) log scales of classes/point_cloud.py:376-377."""
    dist2 = torch.clamp_min(dist_cuda2(points), 0.0000001)
    return torch.log(torch.sqrt(dist2))[..., None].repeat(1, 3)
