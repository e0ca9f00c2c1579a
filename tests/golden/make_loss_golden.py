"""Generate tests/golden/loss/loss_l1_ssim.npz with the reference's own loss functions.

Run in a container where the reference tree is mounted at /root/reference (or at $RAYGAUSS_REFERENCE):
    python tests/golden/make_loss_golden.py
utils/loss_utils.py (torch only) computes l1_loss, ssim and the training loss of
scripts/train.py:110-112, (1 - 0.2) L1 + 0.2 (1 - SSIM), with its gradient with respect to the
rendered image, on seeded (3, H, W) image pairs of two shapes, on the CPU.
"""
import importlib.util
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("RAYGAUSS_REFERENCE", "/root/reference")


def main():
    spec = importlib.util.spec_from_file_location("ref_loss", os.path.join(REF, "utils", "loss_utils.py"))
    L = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(L)
    g = torch.Generator().manual_seed(12)
    out = {}
    for i, (h, w) in enumerate(((20, 24), (17, 9))):
        img = torch.rand((3, h, w), generator=g).requires_grad_(True)
        gt = torch.rand((3, h, w), generator=g)
        l1 = L.l1_loss(img, gt)
        s = L.ssim(img, gt)
        loss = (1.0 - 0.20) * l1 + 0.20 * (1.0 - s)
        loss.backward()
        out[f"img{i}"] = img.detach().numpy()
        out[f"gt{i}"] = gt.numpy()
        out[f"l1_{i}"] = np.float32(l1.item())
        out[f"ssim{i}"] = np.float32(s.item())
        out[f"loss{i}"] = np.float32(loss.item())
        out[f"grad{i}"] = img.grad.numpy()
    os.makedirs(os.path.join(HERE, "loss"), exist_ok=True)
    np.savez_compressed(os.path.join(HERE, "loss", "loss_l1_ssim.npz"), **out)
    print("wrote", os.path.join(HERE, "loss", "loss_l1_ssim.npz"))


if __name__ == "__main__":
    sys.exit(main())
