"""Test configuration: the `gpu` marker, import paths and shared helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "for-qaoa_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


# Parity tolerances (fixed by the spec of the path being replaced):
STATE_RTOL = 1e-12   # state vector: max |a - b| <= 1e-12 * max |b|
ENERGY_RTOL = 1e-12  # <C>
GRAD_TOL = 1e-8      # gradients, relative to max(1, max |g|)


def assert_state_close(a, b, rtol=STATE_RTOL, what="state"):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    scale = np.abs(b).max()
    err = np.abs(a - b).max()
    assert err <= rtol * scale, "%s: max|diff| = %.3e > %.1e * %.3e" % (what, err, rtol, scale)
    l2 = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert l2 <= rtol, "%s: relative L2 diff %.3e > %.1e" % (what, l2, rtol)


def complete_int(n, rng, lo=1, hi=10):
    return np.triu(rng.integers(lo, hi + 1, size=(n, n)).astype(np.float64), 1)


def gnp_fp(n, rng, p=0.5):
    return np.triu(rng.random((n, n)), 1) * np.triu(rng.random((n, n)) < p, 1)


def gnp_int(n, rng, p=0.5, lo=1, hi=10):
    return complete_int(n, rng, lo, hi) * np.triu(rng.random((n, n)) < p, 1)


def angles(rng, P):
    return rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    return O


@pytest.fixture(scope="session")
def fq():
    import forqaoa
    return forqaoa


@pytest.fixture(scope="session")
def ctx(fq):
    c = fq.Context(0)
    yield c
    c.close()
