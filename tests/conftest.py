import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


@pytest.fixture(scope="session")
def golden_fir():
    import numpy as np

    return np.load(os.path.join(ROOT, "tests", "golden", "fir_golden.npz"))


@pytest.fixture(scope="session")
def golden_biquad():
    import numpy as np

    return np.load(os.path.join(ROOT, "tests", "golden", "biquad_golden.npz"))


def case_keys(npz, prefix):
    return sorted({k[: -len("_meta")] for k in npz.files if k.startswith(prefix) and k.endswith("_meta")})
