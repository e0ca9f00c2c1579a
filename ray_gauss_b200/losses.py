"""The training loss of the reference (scripts/train.py:110-112): (1 - 0.2) L1 + 0.2 (1 - SSIM) of
the rendered image against the ground truth, with the SSIM of utils/loss_utils.py:17-64: an 11-tap
Gaussian window of standard deviation 1.5 (normalised in float32), per-channel local means,
variances and covariance by 2-D convolution with zero padding, C1 = 0.01^2, C2 = 0.03^2, averaged
over the map.  The window is built once per device and channel count, so the loss can run inside a
captured CUDA graph after a first eager call."""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F

_WINDOWS = {}


def gaussian_window(size: int = 11, sigma: float = 1.5, channels: int = 3, device=None,
                    dtype=torch.float32) -> torch.Tensor:
    """(channels, 1, size, size): the outer product of the normalised 1-D Gaussian
    exp(-(x - size // 2)^2 / (2 sigma^2)), x = 0..size-1, evaluated in double and rounded to float
    before the normalisation."""
    key = (size, sigma, channels, str(device), dtype)
    w = _WINDOWS.get(key)
    if w is None:
        g = torch.tensor([math.exp(-((x - size // 2) ** 2) / float(2 * sigma ** 2)) for x in range(size)],
                         dtype=torch.float32)
        g = (g / g.sum()).unsqueeze(1)
        w2 = g.mm(g.t()).unsqueeze(0).unsqueeze(0)
        w = w2.expand(channels, 1, size, size).contiguous().to(device=device, dtype=dtype)
        _WINDOWS[key] = w
    return w


def l1_loss(img: torch.Tensor, gt: torch.Tensor) -> torch.Tensor:
    return torch.abs(img - gt).mean()


def ssim(img1: torch.Tensor, img2: torch.Tensor, window_size: int = 11) -> torch.Tensor:
    """Mean SSIM of two (C, H, W) or (N, C, H, W) images."""
    c = img1.size(-3)
    w = gaussian_window(window_size, 1.5, c, img1.device, img1.dtype)
    pad = window_size // 2
    mu1 = F.conv2d(img1, w, padding=pad, groups=c)
    mu2 = F.conv2d(img2, w, padding=pad, groups=c)
    mu1_sq, mu2_sq, mu12 = mu1.pow(2), mu2.pow(2), mu1 * mu2
    s1 = F.conv2d(img1 * img1, w, padding=pad, groups=c) - mu1_sq
    s2 = F.conv2d(img2 * img2, w, padding=pad, groups=c) - mu2_sq
    s12 = F.conv2d(img1 * img2, w, padding=pad, groups=c) - mu12
    c1, c2 = 0.01 ** 2, 0.03 ** 2
    m = ((2 * mu12 + c1) * (2 * s12 + c2)) / ((mu1_sq + mu2_sq + c1) * (s1 + s2 + c2))
    return m.mean()


def l1_ssim_loss(img: torch.Tensor, gt: torch.Tensor, lambda_ssim: float = 0.20) -> torch.Tensor:
    """(1 - lambda) L1 + lambda (1 - SSIM) of (3, H, W) images (scripts/train.py:110-112)."""
    return (1.0 - lambda_ssim) * l1_loss(img, gt) + lambda_ssim * (1.0 - ssim(img, gt))


def views_l1_ssim_loss(ray_colors: torch.Tensor, target: torch.Tensor, views, lambda_ssim: float = 0.20):
    """The per-image loss averaged over the views of a batched render: packed (R, 3) ray colours
    and targets are cut into each view's (H, W, 3) image and permuted to (3, H, W) like the
    reference's image_mean.permute(2, 0, 1)."""
    if tuple(views.supersampling) != (1, 1):
        raise ValueError("l1_ssim needs supersampling (1, 1): reduce supersampled images to the target size first")
    total = 0.0
    for v, cam in enumerate(views.cameras):
        a, b = views.offsets[v], views.offsets[v + 1]
        h, w = cam.image_height, cam.image_width
        img = ray_colors[a:b].reshape(h, w, 3).permute(2, 0, 1)
        gt = target[a:b].reshape(h, w, 3).permute(2, 0, 1)
        total = total + l1_ssim_loss(img, gt, lambda_ssim)
    return total / len(views.cameras)
