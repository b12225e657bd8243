import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

# Parity tolerance on log10 likelihoods (the accuracy bound is 1e-5 relative
# on log10).  ATOL only matters for scores within 0.1 of zero, where a relative
# bound alone would ask for more than FP32 arithmetic can carry.
RTOL = 1e-5
ATOL = 1e-6


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a)")


def assert_log10_close(got, want, rtol=RTOL, atol=ATOL, what=""):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, (got.shape, want.shape)
    err = np.abs(got - want)
    bound = rtol * np.abs(want) + atol
    bad = ~(err <= bound)
    if bad.any():
        i = np.flatnonzero(bad)[:10]
        raise AssertionError(
            f"{what}: {bad.sum()} of {len(got)} outside |d| <= {rtol}*|ref| + {atol}; "
            f"first: idx {i.tolist()} got {got[i].tolist()} want {want[i].tolist()}")
    return float(err.max()) if len(err) else 0.0


@pytest.fixture(scope="session")
def engine():
    import gpupairhmm_b200 as g
    e = g.Engine(mode=g.MODE_ENGINE)
    yield e
    e.close()


@pytest.fixture(scope="session")
def plain_engine():
    import gpupairhmm_b200 as g
    e = g.Engine(mode=g.MODE_PLAIN)
    yield e
    e.close()
