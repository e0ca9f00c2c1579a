"""The fused 3D filter against the reference's compute_3D_filter (classes/point_cloud.py:1153-1215)
restated in torch on the same cameras.  The depths come from a 3x3 product whose summation order
inside torch is not specified, so values must agree within 1e-6 relative."""
import math

import pytest
import torch

pytestmark = pytest.mark.gpu


def _reference(xyz, cameras):
    distance = torch.ones((xyz.shape[0]), device=xyz.device) * 100000.0
    valid_points = torch.zeros((xyz.shape[0]), device=xyz.device, dtype=torch.bool)
    focal_length = 0.
    for camera in cameras:
        wvt = camera.world_view_transform.to(xyz.device)
        R, T = wvt[:3, :3], wvt[3, :3]
        xyz_cam = xyz @ R + T[None, :]
        valid_depth = xyz_cam[:, 2] > 0.2
        x, y, z = xyz_cam[:, 0], xyz_cam[:, 1], xyz_cam[:, 2]
        z = torch.clamp(z, min=0.001)
        focal_x = camera.image_width / (2 * math.tan(camera.FoVx / 2))
        focal_y = camera.image_height / (2 * math.tan(camera.FoVy / 2))
        x = x / z * focal_x + camera.image_width / 2.0
        y = y / z * focal_y + camera.image_height / 2.0
        in_screen = torch.logical_and(torch.logical_and(x >= -0.15 * camera.image_width, x <= camera.image_width * 1.15),
                                      torch.logical_and(y >= -0.15 * camera.image_height, y <= 1.15 * camera.image_height))
        valid = torch.logical_and(valid_depth, in_screen)
        distance[valid] = torch.min(distance[valid], z[valid])
        valid_points = torch.logical_or(valid_points, valid)
        focal_length = max(focal_length, focal_x, focal_y)
    distance[~valid_points] = distance[valid_points].max()
    filter_3D = 0.5 * distance / focal_length
    return torch.log(filter_3D[..., None]), valid_points


@pytest.mark.parametrize("n, views", [(20_000, 16), (70_001, 600)])
def test_compute_3D_filter_matches_reference(cuda, n, views):
    """Unbounded cloud (some Gaussians behind or beside every camera); 600 cameras take two
    shared-memory stages."""
    from ray_gauss_b200 import synthetic as S
    from ray_gauss_b200.filter3d import compute_3D_filter
    p = S.unbounded(n, seed=3, nsg=0)
    xyz = torch.as_tensor(p["positions"], dtype=torch.float32, device=cuda).contiguous()
    cams = S.ring_cameras(views, seed=4, device=cuda)
    ref, seen = _reference(xyz, cams)
    out = compute_3D_filter(xyz, cams)
    torch.cuda.synchronize()
    assert 0 < int(seen.sum()) < n
    assert out.shape == (n, 1) and torch.isfinite(out).all()
    assert torch.allclose(out, ref, rtol=1e-6, atol=0), (out - ref).abs().max().item()
    assert float((out == ref).float().mean()) > 0.99
