"""The 3D minimum-size filter (``PointCloud.compute_3D_filter``, classes/point_cloud.py:1153-1215)
in two kernels instead of a Python loop of torch launches per training camera.

``compute_3D_filter(positions, cameras)`` returns the (N, 1) log filter the reference stores in
``filter_3D``: for every Gaussian the smallest depth over the cameras that see it (depth > 0.2 and
projection inside the image widened by 15 % on each side), the largest seen depth for Gaussians no
camera sees, and log(0.5 * depth / focal) with the largest focal length of the cameras.  Cameras
follow the reference's contract (``world_view_transform``, ``FoVx``, ``FoVy``, ``image_width``,
``image_height``); R and T are the first three rows and the last row of ``world_view_transform``.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from ._lib import check


def fov2focal(fov, pixels):
    """utils/graphics_utils.py: pixels / (2 tan(fov / 2))."""
    return pixels / (2 * math.tan(fov / 2))


def camera_table(cameras):
    """(n_cams, 20) float32 rows of rg_filter_camera and the largest focal length (a Python float,
    compared in double like the reference's loop)."""
    rows, focal = [], 0.0
    for cam in cameras:
        wvt = cam.world_view_transform.detach().to("cpu", torch.float32).numpy()
        W, H = cam.image_width, cam.image_height
        fx, fy = fov2focal(cam.FoVx, W), fov2focal(cam.FoVy, H)
        row = np.empty(20, np.float32)
        row[0:9] = wvt[:3, :3].reshape(-1)
        row[9:12] = wvt[3, :3]
        row[12:20] = [fx, fy, W / 2.0, H / 2.0, -0.15 * W, W * 1.15, -0.15 * H, 1.15 * H]
        rows.append(row)
        if focal < fx:
            focal = fx
        if focal < fy:
            focal = fy
    return np.stack(rows) if rows else np.zeros((0, 20), np.float32), focal


def compute_3D_filter(positions: torch.Tensor, cameras) -> torch.Tensor:
    if positions.dtype != torch.float32 or not positions.is_contiguous() or positions.dim() != 2:
        raise ValueError("positions: (N, 3) FP32 contiguous")
    if not positions.is_cuda:
        raise ValueError("compute_3D_filter runs on CUDA tensors")
    dev = positions.device
    n = positions.shape[0]
    table, focal = camera_table(cameras)
    if not len(table):
        raise ValueError("compute_3D_filter needs at least one camera")
    cams = torch.from_numpy(table).to(dev)
    inv_focal = float(np.float32(1.0) / np.float32(focal))   # torch divides by a Python number this way
    depth = torch.empty(n, dtype=torch.float32, device=dev)
    mx = torch.empty(1, dtype=torch.int32, device=dev)
    out = torch.empty((n, 1), dtype=torch.float32, device=dev)
    lib = _lib.load()
    with torch.cuda.device(dev):   # the kernels launch on the current CUDA device
        check(lib.rg_compute_3d_filter(positions.data_ptr(), n, cams.data_ptr(), len(table), inv_focal,
                                       depth.data_ptr(), mx.data_ptr(), out.data_ptr(),
                                       ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
              None, "rg_compute_3d_filter")
    return out
