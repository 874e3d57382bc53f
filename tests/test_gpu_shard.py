"""GPU parity of the sharded (D > 0) path: every shard of the state on this
one GPU, the passes through the C ABI (fq_shard_layer,
fq_shard_layer_after_swap, fq_rx_targets, fq_shard_expectation), the all-to-all as chunk copies (`local_exchange`,
the same data movement `dist_exchange` does across GPUs), the schedule of
for-qaoa_b200/sharded.py.  The gathered state, in logical order by the
label map, and the summed <C> are checked against the oracle, and at
N=24 against the single-GPU engine."""
import sys

import numpy as np
import pytest

from conftest import (PKG, ENERGY_RTOL, assert_state_close, complete_int, gnp_fp, gnp_int,
                      angles)

pytestmark = pytest.mark.gpu
sys.path.insert(0, PKG)


def run_sharded(fq, N, D, W, g, b, fuse=True, logical=True):
    import torch
    import sharded
    prev = torch.cuda.current_stream()
    stream, ctx = sharded.shard_context(0)
    try:
        shards = [sharded.ShardOps(ctx, N, D, r, "cuda") for r in range(1 << D)]
        labels, gfin = sharded.forward(shards, sharded.local_exchange, N, D, W, g, b, fuse=fuse)
        e = sum(s.expectation(gfin) for s in shards)
        psi = torch.cat([s.buf for s in shards]).cpu().numpy()
        torch.cuda.synchronize()
        return (sharded.to_logical(psi, labels) if logical else psi), e
    finally:
        ctx.close()
        torch.cuda.set_stream(prev)


def graph(kind, n, rng):
    return {"int": complete_int(n, rng), "fp": gnp_fp(n, rng), "neg": complete_int(n, rng, -6, 6),
            "sparse": gnp_int(n, rng, 0.3), "huge": complete_int(n, rng, 1, 5000)}[kind]


@pytest.mark.parametrize("N,D,P,kind", [
    (14, 1, 2, "int"), (15, 2, 3, "fp"), (16, 1, 1, "neg"), (17, 2, 2, "sparse"),
    (19, 1, 3, "int"), (21, 2, 2, "int"), (22, 1, 2, "fp"), (20, 3, 2, "int"), (18, 1, 2, "huge"),
])
def test_sharded_matches_oracle(fq, oracle, N, D, P, kind):
    rng = np.random.default_rng(31 * N + D)
    W = graph(kind, N, rng)
    g, b = angles(rng, P)
    psi, e = run_sharded(fq, N, D, W, g, b)
    want = oracle.qaoa_logical(W, g, b)
    assert_state_close(psi, want, what=f"sharded N={N} D={D}")
    eo = oracle.expectation(want, W)
    assert abs(e - eo) <= ENERGY_RTOL * max(1.0, abs(eo))


def test_sharded_matches_engine_n24(fq, ctx):
    rng = np.random.default_rng(2424)
    N, D, P = 24, 2, 3
    W = complete_int(N, rng)
    g, b = angles(rng, P)
    psi, e = run_sharded(fq, N, D, W, g, b)
    st = ctx.state(N)
    try:
        ef = ctx.qaoa_forward(st, W, g, b)
        want = st.to_host()
    finally:
        st.free()
    assert_state_close(psi, want, what="sharded N=24 D=2 vs engine")
    assert abs(e - ef) <= ENERGY_RTOL * abs(ef)


@pytest.mark.parametrize("N,D,P,kind", [
    (25, 1, 3, "int"), (26, 2, 2, "fp"), (26, 1, 2, "huge"), (28, 4, 2, "int"), (27, 3, 3, "neg"),
])
def test_swapped_in_rx_inside_first_pass(fq, N, D, P, kind):
    """fq_shard_layer_after_swap rotates the swapped-in qubits inside the
    layer's first pass (N-D >= 24, D <= 4): the same state as the rotation
    in a pass of its own after each exchange, bit for bit with one
    swapped-in qubit (the same formula on the same operands), within
    rounding with several (their order differs)."""
    rng = np.random.default_rng(17 * N + D)
    W = graph(kind, N, rng)
    g, b = angles(rng, P)
    # Both schedules leave the same label map: compare in physical order.
    psi_f, e_f = run_sharded(fq, N, D, W, g, b, fuse=True, logical=False)
    psi_s, e_s = run_sharded(fq, N, D, W, g, b, fuse=False, logical=False)
    if D == 1:
        assert np.array_equal(psi_f, psi_s)
    else:
        assert_state_close(psi_f, psi_s, what=f"fused vs separate N={N} D={D}")
    assert abs(e_f - e_s) <= ENERGY_RTOL * abs(e_s)


def test_sharded_fused_schedule_matches_engine_n26(fq, ctx):
    rng = np.random.default_rng(2626)
    N, D, P = 26, 2, 4
    W = complete_int(N, rng)
    g, b = angles(rng, P)
    psi, e = run_sharded(fq, N, D, W, g, b, fuse=True)
    st = ctx.state(N)
    try:
        ef = ctx.qaoa_forward(st, W, g, b)
        want = st.to_host()
    finally:
        st.free()
    assert_state_close(psi, want, what="sharded N=26 D=2 (fused) vs engine")
    assert abs(e - ef) <= ENERGY_RTOL * abs(ef)


def test_shard_needs_the_context_on_the_current_stream(fq):
    import sharded
    c = fq.Context(0)  # a private stream: exchanges on torch's stream would race it
    try:
        with pytest.raises(ValueError):
            sharded.ShardOps(c, 14, 1, 0, "cuda")
    finally:
        c.close()


def test_shard_arguments_rejected(fq, ctx):
    import torch
    buf = torch.empty(1 << 12, dtype=torch.complex128, device="cuda")
    W = np.triu(np.ones((13, 13)), 1)
    with pytest.raises(fq.FQError):   # a shard of 12 qubits is below the minimum of 13
        ctx.shard_layer(buf.data_ptr(), 13, 1, 0, W, 0.3, 0.2, True)
    buf = torch.empty(1 << 13, dtype=torch.complex128, device="cuda")
    W = np.triu(np.ones((14, 14)), 1)
    with pytest.raises(fq.FQError):   # rank outside [0, 2^D)
        ctx.shard_layer(buf.data_ptr(), 14, 1, 2, W, 0.3, 0.2, True)
    with pytest.raises(fq.FQError):   # non-finite angle of the swapped-in qubits
        ctx.shard_layer_after_swap(buf.data_ptr(), 14, 1, 0, W, 0.3, 0.2, float("nan"))
