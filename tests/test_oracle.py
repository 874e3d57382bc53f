"""CPU tests of the oracle: pinned to the reference's own outputs (golden
vectors made by running FOR-QAOA's unmodified CUDA code), to known-answer
cases, to a numpy restatement and to finite differences."""
import glob
import os

import numpy as np
import pytest

from conftest import (GOLDEN, assert_state_close, complete_int, gnp_fp, angles)

GOLDEN_FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def test_golden_fixtures_present():
    assert len(GOLDEN_FILES) >= 8


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=[os.path.basename(p) for p in GOLDEN_FILES])
def test_oracle_matches_reference_golden(oracle, path):
    d = np.load(path)
    sv, gfin, lab = oracle.weighted_run(d["graph"], int(d["C"]), d["gammas"], d["betas"])
    if "state" in d.files:
        assert_state_close(sv, d["state"], what="oracle vs reference " + path)
    else:
        ref = d["sample_amp"]
        got = sv[d["sample_idx"]]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        blocks = (np.abs(sv) ** 2).reshape(256, -1).sum(axis=1)
        assert np.abs(blocks - d["abs2_sum_by_block"]).max() <= 1e-12
    # The relabelled graph is moved, never recomputed: bit-identical.
    assert np.array_equal(gfin, d["graph_final"])
    assert abs(np.vdot(sv, sv).real - 1) < 1e-12


def numpy_logical(W, gam, bet, amp0):
    N = W.shape[0]
    z = np.arange(1 << N)
    Cz = sum(W[i, j] * (((z >> i) & 1) ^ ((z >> j) & 1))
             for i in range(N) for j in range(i + 1, N))
    Wt = W[np.triu_indices(N, 1)].sum()
    sv = np.full(1 << N, amp0, complex)
    for p in range(len(gam)):
        sv = sv * np.exp(1j * gam[p] * (2 * Cz - Wt) / 2)
        c, s = np.cos(bet[p] / 2), np.sin(bet[p] / 2)
        for t in range(N):
            a = sv.reshape(-1, 2, 1 << t)
            q0 = a[:, 0, :].copy()
            q1 = a[:, 1, :].copy()
            a[:, 0, :] = c * q0 - 1j * s * q1
            a[:, 1, :] = -1j * s * q0 + c * q1
            sv = a.reshape(-1)
    return sv, Cz


@pytest.mark.parametrize("N,C,P", [(2, 1, 1), (5, 2, 3), (8, 3, 4), (9, 4, 2), (11, 5, 3)])
def test_oracle_vs_numpy_and_label_map(oracle, N, C, P):
    rng = np.random.default_rng(N * 100 + C)
    W = complete_int(N, rng)
    g, b = angles(rng, P)
    ref, Cz = numpy_logical(W, g, b, oracle.init_amp(N))
    lo = oracle.qaoa_logical(W, g, b)
    assert_state_close(lo, ref)
    ph, _, lab = oracle.weighted_run(W, C, g, b)
    assert_state_close(oracle.to_logical(ph, lab), ref)
    assert np.array_equal(oracle.cut_values(W), Cz)


def test_kat_gamma_zero(oracle):
    # RX(b)|+> = exp(-i b/2)|+>: every amplitude is 2^(-N/2) exp(-i N sum(b)/2).
    N, P = 10, 3
    rng = np.random.default_rng(5)
    W = complete_int(N, rng)
    b = rng.uniform(0, np.pi / 2, P)
    sv = oracle.qaoa_logical(W, np.zeros(P), b)
    want = 2.0 ** (-N / 2) * np.exp(-1j * N * b.sum() / 2)
    assert np.abs(sv - want).max() < 1e-14


def test_kat_beta_zero(oracle):
    # Without mixing only phases change: |psi|^2 uniform, <C> = W/2.
    N, P = 9, 2
    rng = np.random.default_rng(6)
    W = gnp_fp(N, rng)
    g = rng.uniform(0, np.pi, P)
    sv = oracle.qaoa_logical(W, g, np.zeros(P))
    assert np.abs(np.abs(sv) ** 2 - 2.0 ** -N).max() < 1e-15
    assert abs(oracle.expectation(sv, W) - W.sum() / 2) < 1e-12 * W.sum()


def test_cut_values_and_S(oracle):
    rng = np.random.default_rng(7)
    for W in (complete_int(10, rng, -5, 5), gnp_fp(9, rng)):
        N = W.shape[0]
        z = np.arange(1 << N)
        brute = sum(W[i, j] * (((z >> i) & 1) ^ ((z >> j) & 1))
                    for i in range(N) for j in range(i + 1, N))
        np.testing.assert_allclose(oracle.cut_values(W), brute, rtol=0, atol=1e-12)
        np.testing.assert_allclose(oracle.cost_diag_S(W), 2 * brute - W.sum(), rtol=0,
                                   atol=1e-12)


@pytest.mark.parametrize("N,P,kind", [(6, 3, "int"), (8, 2, "fp"), (7, 4, "int")])
def test_oracle_adjoint_vs_finite_differences(oracle, N, P, kind):
    rng = np.random.default_rng(N + P)
    W = complete_int(N, rng) if kind == "int" else gnp_fp(N, rng)
    g, b = angles(rng, P)
    e, gg, gb = oracle.energy_grad(W, g, b)
    assert abs(e - oracle.expectation(oracle.qaoa_logical(W, g, b), W)) < 1e-12 * abs(e)
    h = 1e-6
    fd_g, fd_b = [], []
    for k in range(P):
        gp, gm = g.copy(), g.copy()
        gp[k] += h
        gm[k] -= h
        fd_g.append((oracle.expectation(oracle.qaoa_logical(W, gp, b), W) -
                     oracle.expectation(oracle.qaoa_logical(W, gm, b), W)) / (2 * h))
        bp, bm = b.copy(), b.copy()
        bp[k] += h
        bm[k] -= h
        fd_b.append((oracle.expectation(oracle.qaoa_logical(W, g, bp), W) -
                     oracle.expectation(oracle.qaoa_logical(W, g, bm), W)) / (2 * h))
    # Central differences carry ~eps*|E|/h of roundoff: compare to the scale.
    scale = max(1.0, np.abs(gg).max(), np.abs(gb).max())
    assert np.abs(gg - fd_g).max() < 1e-6 * scale
    assert np.abs(gb - fd_b).max() < 1e-6 * scale


def test_swap_and_relabel_are_involutions(oracle):
    rng = np.random.default_rng(9)
    N = 10
    sv = rng.normal(size=1 << N) + 1j * rng.normal(size=1 << N)
    a = sv.copy()
    oracle.swap_gate_conti(a, N, 1, 5, 3)
    assert not np.allclose(a, sv)
    oracle.swap_gate_conti(a, N, 1, 5, 3)
    assert np.array_equal(a, sv)
    W = complete_int(N, rng)
    g2 = oracle.mapping_after_swap_conti(oracle.mapping_after_swap_conti(W, 0, 4, 3), 0, 4, 3)
    assert np.array_equal(g2, W)


@pytest.mark.parametrize("n,p", [(12, 1), (12, 2), (10, 3)])
def test_light_cone_energy_matches_full_state(oracle, n, p):
    """The light-cone sum that checks the 32-qubit GPU run equals the full
    oracle simulation where both fit."""
    from conftest import light_cone_energy, random_regular, weighted_graph
    rng = np.random.default_rng(100 + n + p)
    edges = random_regular(n, 3, rng)
    W = weighted_graph(n, edges, rng)
    g, b = rng.uniform(0, np.pi, p), rng.uniform(0, np.pi / 2, p)
    full = oracle.expectation(oracle.qaoa_logical(W, g, b), W)
    assert abs(light_cone_energy(oracle, n, edges, W, g, b) - full) <= 1e-13 * abs(full)
