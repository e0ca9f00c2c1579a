import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
SCENES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                if not p.endswith("sh_twin.npz") and not os.path.basename(p).startswith("infer_"))
# inference-program fixtures (image + Gaussians per ray)
INFER_SCENES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "infer_*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a engine)")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def engine_lib():
    from ray_gauss_b200 import _lib
    from ray_gauss_b200.build import build_library
    build_library()
    return _lib.load()


@pytest.fixture(scope="session")
def cuda(engine_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
