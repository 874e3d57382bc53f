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


# ---- light cones: <C> of a large state from small exact simulations ------
def random_regular(n, d, rng):
    """Seeded pairing model, retried until the graph is simple."""
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), d))
        pairs = stubs.reshape(-1, 2)
        if np.any(pairs[:, 0] == pairs[:, 1]):
            continue
        e = {tuple(sorted(p)) for p in pairs.tolist()}
        if len(e) == len(pairs):
            return sorted(e)


def weighted_graph(n, edges, rng):
    W = np.zeros((n, n))
    for u, v in edges:
        W[u, v] = rng.random()
    return W


def ball(adj, seeds, r):
    cur = set(seeds)
    for _ in range(r):
        cur |= {x for u in cur for x in adj[u]}
    return cur


def light_cone_energy(oracle, n, edges, W, gammas, betas):
    """<C> after p QAOA layers as a sum of edge terms, each simulated by the
    oracle on the edges within distance p-1 of the edge (its light cone)."""
    p = len(gammas)
    adj = {u: set() for u in range(n)}
    for u, v in edges:
        adj[u].add(v)
        adj[v].add(u)
    total = 0.0
    for u, v in edges:
        inner = ball(adj, (u, v), p - 1)
        sub_edges = [(a, b) for a, b in edges if a in inner or b in inner]
        nodes = sorted({x for e in sub_edges for x in e})
        idx = {x: i for i, x in enumerate(nodes)}
        m = len(nodes)
        Ws = np.zeros((m, m))
        for a, b in sub_edges:
            i, j = sorted((idx[a], idx[b]))
            Ws[i, j] = W[a, b]
        psi = oracle.qaoa_logical(Ws, gammas, betas)
        z = np.arange(1 << m)
        par = ((z >> idx[u]) ^ (z >> idx[v])) & 1
        zz = np.sum(np.abs(psi) ** 2 * (1 - 2 * par))
        total += W[u, v] * (1 - zz) / 2
    return total



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
