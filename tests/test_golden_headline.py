"""The headline workload pinned to the reference itself: N=30, p=5, K_30 with
integer weights 1..10 and the benchmark's seeded angles, run by FOR-QAOA's
unmodified single-device CUDA path at its own profiled chunk size (C = 11,
src/Weighted.cpp:115-138) on a B200 (tests/golden/gen_golden.py ... k30).
The fixture holds 4096 sampled amplitudes, the probability mass of 256
blocks, the norm and <C> of the reference's final state (physical order),
and its relabelled graph.

CPU tests check the fixture's own consistency and that the graph relabelling
this library applies (fq_relabel_graph, src/swap.cu:27-50) reproduces the
reference's bit for bit; the GPU test runs the fused engine on the same
inputs, permutes its logical-order state into the reference's physical order
and compares everything the fixture holds at 1e-12."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, ENERGY_RTOL, STATE_RTOL

PATH = os.path.join(GOLDEN, "headline", "k30_int_c11_p5.npz")


@pytest.fixture(scope="module")
def fix():
    return np.load(PATH)


def test_fixture_is_the_benchmark_workload(fix):
    rng = np.random.default_rng(30)
    n, P = 30, 5
    W = np.triu(rng.integers(1, 11, size=(n, n)).astype(np.float64), 1)
    rng.integers(1, 11, size=(n, n))  # the benchmark's second graph
    g = rng.uniform(0, np.pi, P)
    b = rng.uniform(0, np.pi / 2, P)
    assert int(fix["n"]) == n and int(fix["C"]) == 11
    assert np.array_equal(fix["graph"], W)
    assert np.array_equal(fix["gammas"], g) and np.array_equal(fix["betas"], b)


def test_fixture_self_consistent(fix):
    assert abs(float(fix["norm"]) - 1.0) < 1e-12
    assert abs(fix["abs2_sum_by_block"].sum() - float(fix["norm"])) < 1e-12
    # <C> lies between 0 and the total weight.
    assert 0 < float(fix["energy"]) < fix["graph"].sum()
    idx = fix["sample_idx"]
    assert np.all(np.diff(idx) > 0) and idx[0] == 0 and idx[-1] == (1 << 30) - 1
    # Each block's mass bounds the samples inside it.
    blk = idx >> 22
    p = np.abs(fix["sample_amp"]) ** 2
    for k in np.unique(blk):
        assert p[blk == k].sum() <= fix["abs2_sum_by_block"][k] * (1 + 1e-12)


def test_relabel_matches_reference(fq, fix):
    """The reference schedule at C = 11 moves qubit blocks (0, 11, 11) and
    (0, 22, 8) every layer; the same relabelling of the input graph gives the
    reference's final graph exactly."""
    g = np.array(fix["graph"], dtype=np.float64)
    for _ in range(len(fix["gammas"])):
        g = fq.relabel_graph(g, 0, 11, 11)
        g = fq.relabel_graph(g, 0, 22, 8)
    assert np.array_equal(g, fix["graph_final"])


def _device_view(ptr, n):
    """complex128 torch view (no copy) of 2^n amplitudes at a device address."""
    import torch

    class _Iface:
        pass

    o = _Iface()
    o.__cuda_array_interface__ = {"shape": (1 << n, 2), "typestr": "<f8", "strides": None,
                                  "data": (int(ptr.value), False), "version": 3}
    return torch.view_as_complex(torch.as_tensor(o, device="cuda"))


@pytest.mark.gpu
def test_fused_engine_vs_reference_n30(ctx, fq, fix):
    """Fused engine (11 sweeps, logical order) against the reference's own
    CUDA run (30 launches per layer, physical order) at N=30."""
    import torch
    n, C = int(fix["n"]), int(fix["C"])
    P = len(fix["gammas"])
    st, ph = ctx.state(n), ctx.state(n)
    try:
        e = ctx.qaoa_forward(st, fix["graph"], fix["gammas"], fix["betas"], energy=True)
        lab = fq.reference_label_map(n, C, P)
        ctx.permute_qubits(st, ph, np.argsort(lab))
        ctx.synchronize()
        v = _device_view(ph.ptr, n)
        idx = torch.as_tensor(fix["sample_idx"], device="cuda")
        amp = v[idx].cpu().numpy()
        blocks = (v.real ** 2 + v.imag ** 2).view(256, -1).sum(dim=1).cpu().numpy()
        norm = float(blocks.sum())
        torch.cuda.synchronize()
        del v
    finally:
        st.free()
        ph.free()
    ref = fix["sample_amp"]
    assert np.abs(amp - ref).max() <= STATE_RTOL * np.abs(ref).max()
    assert np.abs(blocks - fix["abs2_sum_by_block"]).max() <= 1e-12
    assert abs(norm - float(fix["norm"])) <= 1e-12
    assert abs(e - float(fix["energy"])) <= ENERGY_RTOL * float(fix["energy"])
