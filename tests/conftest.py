import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from hlr_b200 import build_native as _native  # noqa: E402

if not _native.LIB.exists():
    _native.build()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a / B200)")


_CACHE = {}


def built(name: str, factory):
    """Session cache of host-built matrices (construction takes seconds)."""
    if name not in _CACHE:
        _CACHE[name] = factory()
    return _CACHE[name]


@pytest.fixture(scope="session")
def c1_small():
    import hlr_b200 as hlr
    return built("c1_small", lambda: hlr.build(hlr.Problem.log1d(2048)))


@pytest.fixture(scope="session")
def c1():
    import hlr_b200 as hlr
    return built("c1", lambda: hlr.build(hlr.Problem.log1d(8192)))


@pytest.fixture(scope="session")
def c2_small():
    import hlr_b200 as hlr
    return built("c2_small", lambda: hlr.build(hlr.Problem.exp3d(4096)))


@pytest.fixture(scope="session")
def c3_small():
    import hlr_b200 as hlr
    return built("c3_small", lambda: hlr.build(hlr.Problem.laplace_sphere(refine=4, uniform=True)))


def relerr(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
