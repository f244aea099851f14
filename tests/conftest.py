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


def synthetic_nnw(seed=11):
    """A seeded 10-10-1 star/galaxy network in the .nnw layout (the real
    weights are the user's file; parity does not depend on their values).
    Returns (nn, inbias, inscale, weights, biases, outbias, outscale)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nn = [10, 10, 1]
    inbias = rng.uniform(-1.0, 1.0, 10)
    inscale = rng.uniform(0.3, 1.5, 10)
    weights = [rng.normal(0.0, 0.6, (10, 10)), rng.normal(0.0, 1.0, (10, 1))]
    biases = [rng.normal(0.0, 0.3, 10), rng.normal(0.0, 0.3, 1)]
    return nn, inbias, inscale, weights, biases, [0.05], [0.9]


def write_nnw(path, net):
    """Write a network of synthetic_nnw() as a .nnw file."""
    nn, inbias, inscale, weights, biases, outbias, outscale = net
    fmt = lambda v: " ".join("%.17g" % x for x in v)
    lines = ["NNW", "# synthetic network for the tests", " %d %s" % (len(nn), " ".join(str(n) for n in nn)), "",
             fmt(inbias), fmt(inscale), ""]
    for l in range(len(nn) - 1):
        for j in range(nn[l + 1]):
            lines.append(fmt([weights[l][i][j] for i in range(nn[l])] + [biases[l][j]]))
        lines.append("")
    lines += [fmt(outbias), fmt(outscale)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
