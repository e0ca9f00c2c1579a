"""Seeded synthetic Gaussian scenes and pinhole cameras with the shapes and value distributions of
the five benchmark workloads (no datasets or trained scenes are available offline).

The parameter tensors follow the reference renderer's input contract
(``classes/point_cloud.py:729-739`` ``PointCloud.get_data``): positions (N,3); scales (N,3) already
exponentiated; quaternions (N,4) in (w,x,y,z) order; densities (N,) passed raw; colour features
(N,3,16) channel-major SH degree 3; SG amplitudes (N,3,nsg); SG sharpness (N,nsg) after softplus;
SG lobe axes (N,nsg,3) unit length.  Cameras expose the attributes the renderer reads from the
reference's ``Camera`` (``classes/cameras.py:17-60``): ``camera_center``, ``world_view_transform``
(the transposed world-to-view matrix of ``utils/graphics_utils.py:38-49``), ``FoVx``, ``FoVy``,
``image_width`` and ``image_height``.

Workloads (seed 0 unless given):
  small_object      10k Gaussians uniform in [-1,1]^3, SH3, one 200x200 view, 40 deg, radius 3
  bounded_object    300k Gaussians on 8 sphere/ellipsoid shells, SH3 + 8 SG, one 800x800 view
  unbounded_1m      1M Gaussians (80% unit ball, 20% log-uniform radius 1-50), SH3 + 8 SG,
                    16 views of uneven size 400x300..1600x1200, 50 deg, ring radius 3-5
  unbounded_3m      3M Gaussians, same layout, 4 views 1920x1080
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class Camera:
    """Pinhole camera with the reference ``Camera`` attributes the renderer reads."""
    camera_center: torch.Tensor
    world_view_transform: torch.Tensor
    FoVx: float
    FoVy: float
    image_width: int
    image_height: int

    def to(self, device):
        return Camera(self.camera_center.to(device), self.world_view_transform.to(device), self.FoVx, self.FoVy,
                      self.image_width, self.image_height)


def look_at_camera(eye, target, width, height, fovx=None, fovy=None, device="cpu") -> Camera:
    """Camera at ``eye`` looking at ``target`` with COLMAP axes (x right, y down, z forward)."""
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(target, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    up = np.array([0.0, 0.0, 1.0])
    if abs(fwd @ up) > 0.99:
        up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    down = np.cross(fwd, right)
    c2w_rot = np.stack([right, down, fwd], axis=1)          # columns: camera axes in world
    w2c = np.eye(4)
    w2c[:3, :3] = c2w_rot.T
    w2c[:3, 3] = -c2w_rot.T @ eye
    wvt = torch.tensor(w2c.T, dtype=torch.float32, device=device)
    if fovx is None:
        fovx = 2.0 * math.atan(math.tan(fovy / 2.0) * width / height)
    if fovy is None:
        fovy = 2.0 * math.atan(math.tan(fovx / 2.0) * height / width)
    center = torch.tensor(eye, dtype=torch.float32, device=device)
    return Camera(center, wvt, float(fovx), float(fovy), int(width), int(height))


def _unit(rng, n, d):
    v = rng.standard_normal((n, d))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _softplus(x):
    return np.log1p(np.exp(-np.abs(x))) + np.maximum(x, 0.0)


def _finish(pos, log_s, dens, nsg, rng, sh_std=0.2, sg_std=0.1):
    n = pos.shape[0]
    quat = _unit(rng, n, 4)
    sh = rng.normal(0.0, sh_std, (n, 3, 16))
    out = dict(positions=pos, scales=np.exp(log_s), quaternions=quat, densities=dens, color_features=sh)
    if nsg:
        out["sph_gauss_features"] = rng.normal(0.0, sg_std, (n, 3, nsg))
        out["bandwidth_sharpness"] = rng.uniform(1.0, 20.0, (n, nsg))
        out["lobe_axis"] = _unit(rng, n * nsg, 3).reshape(n, nsg, 3)
    else:
        out["sph_gauss_features"] = np.zeros((n, 3, 0))
        out["bandwidth_sharpness"] = np.zeros((n, 0))
        out["lobe_axis"] = np.zeros((n, 0, 3))
    return out


def small_object(n=10_000, seed=0):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, (n, 3))
    log_s = rng.normal(math.log(0.02), 0.3, (n, 3))
    dens = _softplus(rng.standard_normal(n))
    return _finish(pos, log_s, dens, 0, rng)


def bounded_object(n=300_000, seed=0, nsg=8):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.9, 0.9, (8, 3))
    radii = rng.uniform(0.2, 0.6, (8, 3))
    iso = rng.random(8) < 0.5
    radii[iso] = radii[iso, :1]                                  # half spheres, half ellipsoids
    which = rng.integers(0, 8, n)
    pos = centers[which] + _unit(rng, n, 3) * radii[which]
    pos = np.clip(pos, -1.5, 1.5)
    log_s = rng.normal(math.log(0.01), 0.4, (n, 3))
    dens = rng.lognormal(0.0, 1.0, n)
    return _finish(pos, log_s, dens, nsg, rng)


def unbounded(n=1_000_000, seed=0, nsg=8):
    rng = np.random.default_rng(seed)
    n_in = int(round(0.8 * n))
    r_in = rng.random(n_in) ** (1.0 / 3.0)
    p_in = _unit(rng, n_in, 3) * r_in[:, None]
    r_out = np.exp(rng.uniform(math.log(1.0), math.log(50.0), n - n_in))
    p_out = _unit(rng, n - n_in, 3) * r_out[:, None]
    pos = np.concatenate([p_in, p_out])
    radius = np.concatenate([np.ones(n_in), r_out])
    log_s = rng.normal(math.log(0.015), 0.5, (n, 3)) + np.log(radius)[:, None]
    dens = rng.lognormal(0.0, 1.0, n)
    perm = rng.permutation(n)
    out = _finish(pos[perm], log_s[perm], dens[perm], nsg, rng)
    return out


def ring_cameras(n_views=16, seed=0, w_range=(400, 1600), fovy_deg=50.0, radius=(3.0, 5.0), device="cpu",
                 sizes=None):
    """Inward-facing cameras on a ring; uneven resolutions W ~ U[w_range], H = 0.75 W."""
    rng = np.random.default_rng(seed + 1000)
    cams = []
    for i in range(n_views):
        if sizes is not None:
            w, h = sizes[i % len(sizes)]
        else:
            w = int(rng.integers(w_range[0], w_range[1] + 1))
            h = int(round(0.75 * w))
        ang = 2.0 * math.pi * (i + rng.random() * 0.5) / n_views
        r = rng.uniform(*radius)
        eye = [r * math.cos(ang), r * math.sin(ang), rng.uniform(-0.5, 0.5)]
        cams.append(look_at_camera(eye, [0.0, 0.0, 0.0], w, h, fovy=math.radians(fovy_deg), device=device))
    return cams


def sphere_camera(radius, width, height, fov_deg=40.0, seed=0, device="cpu"):
    rng = np.random.default_rng(seed + 2000)
    u = _unit(rng, 1, 3)[0]
    return look_at_camera(radius * u, [0.0, 0.0, 0.0], width, height, fovx=math.radians(fov_deg),
                          fovy=math.radians(fov_deg), device=device)


def workload(name, seed=0, device="cpu", dtype=torch.float32, n=None):
    """(params dict of torch tensors, list of cameras, white_background) for a named workload."""
    if name == "small_object":
        p = small_object(n or 10_000, seed)
        cams = [sphere_camera(3.0, 200, 200, 40.0, seed, device)]
        white = True
    elif name == "bounded_object":
        p = bounded_object(n or 300_000, seed)
        cams = [sphere_camera(4.0, 800, 800, 40.0, seed, device)]
        white = True
    elif name == "unbounded_1m":
        p = unbounded(n or 1_000_000, seed)
        cams = ring_cameras(16, seed, device=device)
        white = True
    elif name == "unbounded_3m":
        p = unbounded(n or 3_000_000, seed)
        cams = ring_cameras(4, seed, device=device, sizes=[(1920, 1080)])
        white = True
    else:
        raise ValueError(f"unknown workload {name!r}")
    t = {k: torch.as_tensor(v, dtype=dtype, device=device).contiguous() for k, v in p.items()}
    return t, cams, white
