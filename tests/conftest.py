import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libdelta_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    g = ROOT / "tests" / "golden"
    return {name: dict(np.load(g / f"{name}.npz", allow_pickle=False)) for name in ("pairs", "drivers", "dynamics")}


@pytest.fixture(scope="session")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but CUDA is not available")
    from delta_b200.narrowphase import Context

    c = Context(0)
    yield c
    c.close()
