"""Shared helpers of the test suite (cameras from golden vectors, error metrics)."""
import math
from types import SimpleNamespace

import numpy as np
import torch


def camera_from_vector(cv, width, height, device="cpu"):
    """Reference-style camera whose world_view_transform[:3, 0..2] are the U, V, W axes of cv."""
    cv = np.asarray(cv, np.float64)
    wvt = np.eye(4)
    wvt[:3, 0], wvt[:3, 1], wvt[:3, 2] = cv[3:6], cv[6:9], cv[9:12]
    return SimpleNamespace(camera_center=torch.tensor(cv[:3], dtype=torch.float32, device=device),
                           world_view_transform=torch.tensor(wvt, dtype=torch.float32, device=device),
                           FoVx=2.0 * math.atan(float(np.float32(cv[12]))), FoVy=2.0 * math.atan(float(np.float32(cv[13]))),
                           image_width=int(width), image_height=int(height))


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def psnr(a, b):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 20.0 * math.log10(1.0 / math.sqrt(mse))
