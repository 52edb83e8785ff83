import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libfvm_b200.so")
    config.addinivalue_line("markers", "slow: long-running GPU test at full configuration size")


@pytest.fixture(scope="session")
def golden():
    import json
    import numpy as np
    z = np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))
    return z, json.loads(str(z["manifest"])), json.loads(str(z["params"]))
