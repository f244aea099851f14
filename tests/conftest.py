import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gpu-sextractor_b200"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    import sexgpu
    ctx = sexgpu.Context(0)
    yield ctx
    ctx.close()


@pytest.fixture(scope="session")
def masks():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "conv_masks.json")) as f:
        d = json.load(f)
    import numpy as np
    return {k: np.array(v, np.float32) for k, v in d.items()}
