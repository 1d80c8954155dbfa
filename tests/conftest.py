import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine's kernels")


def load_circuits():
    """Golden circuits: {key: (n, ops, reference_state)}."""
    with open(os.path.join(GOLDEN, "circuits.json")) as f:
        meta = json.load(f)
    states = np.load(os.path.join(GOLDEN, "circuits.npz"))
    out = {}
    for key, m in meta.items():
        ops = []
        for op in m["ops"]:
            if op[0] == "Unitary":
                ops.append(("Unitary", tuple(op[1]), (), np.array(op[3]) + 1j * np.array(op[4])))
            else:
                ops.append((op[0], tuple(op[1]), tuple(op[2])))
        out[key] = (m["n"], ops, states[key])
    return out


@pytest.fixture(scope="session")
def golden_circuits():
    return load_circuits()


@pytest.fixture(scope="session")
def cuda_required():
    """GPU tests fail (they do not skip) when no GPU is present."""
    import torch

    assert torch.cuda.is_available(), "this test needs a CUDA GPU"
    return True
