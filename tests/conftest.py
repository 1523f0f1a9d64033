import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_cases.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_cases():
    """{name: (off, ind, trine, total)} produced by the reference itself."""
    data = np.load(GOLDEN)
    names = sorted({k.split("__")[0] for k in data.files})
    return {n: (data[f"{n}__off"], data[f"{n}__ind"], data[f"{n}__trine"],
                int(data[f"{n}__total"][0])) for n in names}


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
