"""Benchmark config 3 on the GPU: N=32 (a 64 GiB state), a random 3-regular
graph with FP64 weights in [0, 1).

<C> of the full 32-qubit state is checked exactly through light cones: for
p layers, <Z_u Z_v> depends only on the edges within distance p-1 of
{u, v}, so each edge's term is simulated by the oracle on that subgraph
(at most 14 qubits for p = 2 on a 3-regular graph) and the terms are
summed.  At p = 3 (the config's depth, whose light cones cover most of the
graph) the fused engine is checked against the reference's own schedule
(cost sweep, RX chunks of C = 13, block swaps) run by this library's
per-kernel entry points."""
import numpy as np
import pytest

from conftest import ENERGY_RTOL, light_cone_energy, random_regular, weighted_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config3():
    rng = np.random.default_rng(32)
    n = 32
    edges = random_regular(n, 3, rng)
    assert len(edges) == 48
    W = weighted_graph(n, edges, rng)
    return n, edges, W, rng


def test_n32_p2_light_cone(ctx, oracle, config3):
    n, edges, W, rng = config3
    g, b = rng.uniform(0, np.pi, 2), rng.uniform(0, np.pi / 2, 2)
    st = ctx.state(n)
    try:
        e = ctx.qaoa_forward(st, W, g, b)
    finally:
        st.free()
    want = light_cone_energy(oracle, n, edges, W, g, b)
    assert abs(e - want) <= ENERGY_RTOL * abs(want), (e, want)


def test_n32_p3_fused_matches_reference_schedule(ctx, config3):
    n, edges, W, rng = config3
    g, b = rng.uniform(0, np.pi, 3), rng.uniform(0, np.pi / 2, 3)
    st = ctx.state(n)
    try:
        e_fused = ctx.qaoa_forward(st, W, g, b)
    finally:
        st.free()
    st = ctx.state(n)
    try:
        Wr = ctx.reference_schedule(st, W, 13, g, b)
        e_ref = ctx.expectation(st, Wr)
    finally:
        st.free()
    assert abs(e_fused - e_ref) <= ENERGY_RTOL * abs(e_ref), (e_fused, e_ref)


def test_n33_max_size_light_cone(ctx, oracle):
    """The largest state the library takes: N=33 (128 GiB, every one of the
    21 fixed-bit slots of the cut tables in use), p=2 on a random 3-regular
    graph with FP64 weights, <C> against the light-cone sum of the oracle;
    then integer weights (the two-level phase tables), p=1."""
    rng = np.random.default_rng(33)
    n = 33
    edges = random_regular(n - 1, 3, rng) + [(31, 32)]  # vertex 32 joins by one edge
    W = weighted_graph(n, edges, rng)
    g, b = rng.uniform(0, np.pi, 2), rng.uniform(0, np.pi / 2, 2)
    st = ctx.state(n)
    try:
        e = ctx.qaoa_forward(st, W, g, b)
        want = light_cone_energy(oracle, n, edges, W, g, b)
        assert abs(e - want) <= ENERGY_RTOL * abs(want), (e, want)
        Wi = np.where(W > 0, rng.integers(1, 10, W.shape), 0).astype(float)
        g1, b1 = rng.uniform(0, np.pi, 1), rng.uniform(0, np.pi / 2, 1)
        e = ctx.qaoa_forward(st, Wi, g1, b1)
        want = light_cone_energy(oracle, n, edges, Wi, g1, b1)
        assert abs(e - want) <= ENERGY_RTOL * abs(want), (e, want)
    finally:
        st.free()
