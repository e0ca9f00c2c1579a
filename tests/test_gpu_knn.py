"""The k-NN initial scales (simple-knn distCUDA2, submodules/simple-knn/simple_knn.cu:126-221):
mean of the three smallest squared distances to the other points, against a brute force over all
pairs in torch.  The brute force evaluates dx*dx + dy*dy + dz*dz without contraction, so values
agree within 2e-6 relative."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _brute(p, chunk=512):
    n = p.shape[0]
    out = torch.empty(n, dtype=torch.float32, device=p.device)
    for i0 in range(0, n, chunk):
        q = p[i0:i0 + chunk]
        d = q[:, None, :] - p[None, :, :]
        d2 = d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2]
        idx = torch.arange(i0, i0 + q.shape[0], device=p.device)
        d2[torch.arange(q.shape[0], device=p.device), idx] = float("inf")
        k = min(3, n - 1)
        best = torch.topk(d2, k, dim=1, largest=False).values if k > 0 else d2[:, :0]
        if k < 3:
            best = torch.cat([best, torch.full((q.shape[0], 3 - k), np.finfo(np.float32).max, device=p.device)], 1)
        out[i0:i0 + q.shape[0]] = (best[:, 0] + best[:, 1] + best[:, 2]) / 3.0
    return out


def _cloud(n, seed):
    g = torch.Generator().manual_seed(seed)
    p = torch.randn(n, 3, generator=g) * 0.3
    far = torch.rand(n, generator=g) < 0.1                      # 10 % far out (sparse boxes)
    p[far] *= 40.0
    p[: n // 50] = p[n // 50: 2 * (n // 50)]                    # exact duplicates: distance 0
    p[n // 2: n // 2 + 5] = p[n // 2 + 5]                       # six copies of one point: mean 0
    return p


@pytest.mark.parametrize("n", [5000, 70_001])
def test_knn_mean_dist_matches_brute_force(cuda, n):
    from ray_gauss_b200.knn import dist_cuda2
    p = _cloud(n, 1).to(cuda).contiguous()
    got = dist_cuda2(p)
    ref = _brute(p)
    torch.cuda.synchronize()
    assert torch.allclose(got, ref, rtol=2e-6, atol=0), (got - ref).abs().max().item()
    assert float((got == 0).float().sum()) >= 6                 # the six copies see three zeros


def test_knn_fewer_than_three_neighbours(cuda):
    from ray_gauss_b200.knn import dist_cuda2
    for n in (1, 2):                      # FLT_MAX + FLT_MAX overflows
        p = torch.randn(n, 3, device=cuda)
        assert torch.isinf(dist_cuda2(p)).all()
    p = torch.randn(3, 3, device=cuda)     # two neighbours: (d0 + d1 + FLT_MAX) / 3
    fmax = np.float32(np.finfo(np.float32).max)
    got = dist_cuda2(p).cpu().numpy()
    assert np.all(got == fmax / np.float32(3.0))   # d0 + d1 vanishes against FLT_MAX
    p = torch.tensor([[0.0, 0, 0], [1.0, 0, 0], [0, 2.0, 0], [0, 0, 3.0]], device=cuda)
    got = dist_cuda2(p).cpu().numpy()
    assert np.allclose(got, [(1 + 4 + 9) / 3, (1 + 5 + 10) / 3, (4 + 5 + 13) / 3, (9 + 10 + 13) / 3], rtol=1e-6)


def test_load_from_ply_without_scales_uses_knn(cuda, tmp_path):
    from ray_gauss_b200.io import load_from_ply, write_ply
    g = np.random.default_rng(3)
    pts = g.normal(size=(3000, 3)).astype(np.float32)
    cols = g.integers(0, 256, size=(3000, 3), dtype=np.uint8)
    path = write_ply(str(tmp_path / "pc"), [pts, cols], ["x", "y", "z", "red", "green", "blue"])
    out = load_from_ply(path, 4, 0, 1.0, cuda)
    ref = torch.log(torch.sqrt(torch.clamp_min(_brute(torch.from_numpy(pts).to(cuda)), 1e-7)))[..., None].repeat(1, 3)
    torch.cuda.synchronize()
    assert torch.allclose(out["params"]["scales"], ref, rtol=2e-6, atol=2e-6)
    assert math.isclose(float(out["params"]["quaternions"][:, 0].min()), 1.0)
