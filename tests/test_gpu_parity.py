"""GPU parity: every kernel entry point of the C ABI against the CPU oracle
(seeded inputs at sizes the oracle finishes in seconds), against the golden
vectors produced by the reference's own CUDA code, and at full sizes through
size-independent properties."""
import glob
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from conftest import (STATE_RTOL, GOLDEN, PKG, ENERGY_RTOL, assert_state_close, complete_int, gnp_fp,
                      gnp_int, angles)

pytestmark = pytest.mark.gpu

GOLDEN_FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def rand_state(rng, n):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def graph_of(kind, n, rng):
    if kind == "int":
        return complete_int(n, rng)
    if kind == "fp":
        return gnp_fp(n, rng)
    if kind == "neg":
        return complete_int(n, rng, -5, 5)
    if kind == "sparse":
        return gnp_int(n, rng, 0.2)
    if kind == "wide":  # integer cut range too wide for the shared two-level table
        return complete_int(n, rng, 1, 500)
    if kind == "huge":  # integer weights past the phase table: the FP64 path
        return complete_int(n, rng, 1, 5000)
    if kind == "zero":  # no edges: C = 0, only the mixer acts
        return np.zeros((n, n))
    raise ValueError(kind)


# ------------------------------------------------------------ cost phase --

@pytest.mark.parametrize("n", [5, 11, 12, 14, 17])
@pytest.mark.parametrize("kind", ["int", "fp", "neg"])
def test_cost_phase_vs_oracle(ctx, oracle, n, kind):
    rng = np.random.default_rng(n * 7 + len(kind))
    W = graph_of(kind, n, rng)
    g1d = oracle.upper_tri_to_1d(W)
    st = ctx.state(n)
    try:
        # layer 0: launch-control init (write-only)
        want = np.zeros(1 << n, complex)
        oracle.cost_phase(want, n, 0.7, g1d, True)
        st.from_host(rand_state(rng, n))  # garbage the kernel must not read
        ctx.cost_phase(st, 0.7, W, True)
        assert_state_close(st.to_host(), want, what="cost init")
        # later layer: multiply
        v = rand_state(rng, n)
        st.from_host(v)
        want = v.copy()
        oracle.cost_phase(want, n, 2.1, g1d, False)
        ctx.cost_phase(st, 2.1, W, False)
        assert_state_close(st.to_host(), want, what="cost mul")
    finally:
        st.free()


@pytest.mark.parametrize("n", [6, 12, 15, 20])
@pytest.mark.parametrize("kind", ["int", "neg", "fp"])
def test_cut_diagonal_vs_oracle(ctx, oracle, n, kind):
    rng = np.random.default_rng(n + 3)
    W = graph_of(kind, n, rng)
    got = ctx.cut_diagonal(n, W)
    want = oracle.cut_values(W)
    if kind == "fp":
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * max(1, W.sum()))
    else:
        assert np.array_equal(got, want)  # integer weights: bit-exact


# ------------------------------------------------------------------- RX --

@pytest.mark.parametrize("n,chunk,targets", [
    (8, 8, [0, 1, 2, 3, 4, 5, 6, 7]), (12, 12, list(range(12))), (12, 10, [0, 3, 9]),
    (14, 13, list(range(13))), (16, 13, [12, 0, 7]), (13, 13, [12]), (20, 11, [10, 2]),
])
def test_rx_chunk_vs_oracle(ctx, oracle, n, chunk, targets):
    rng = np.random.default_rng(n + len(targets))
    v = rand_state(rng, n)
    st = ctx.state(n)
    try:
        st.from_host(v)
        ctx.rx_chunk(st, chunk, targets, 1.234)
        want = v.copy()
        oracle.multi_rotate_x(want, n, targets, 1.234)
        assert_state_close(st.to_host(), want, what="rx_chunk")
    finally:
        st.free()


@pytest.mark.parametrize("n,targets", [(20, [0, 5, 13, 19]), (14, [13]), (9, [8, 0]),
                                       (22, list(range(12, 22)))])
def test_rx_targets_vs_oracle(ctx, oracle, n, targets):
    rng = np.random.default_rng(n)
    v = rand_state(rng, n)
    st = ctx.state(n)
    try:
        st.from_host(v)
        ctx.rx_targets(st, targets, -0.6)
        want = v.copy()
        oracle.multi_rotate_x(want, n, targets, -0.6)
        assert_state_close(st.to_host(), want, what="rx_targets")
    finally:
        st.free()


def test_rx_chunk_rejects_bad_targets(ctx, fq):
    st = ctx.state(12)
    try:
        for chunk, t in [(10, [10]), (10, [1, 1]), (14, [0]), (10, [-1])]:
            with pytest.raises(fq.FQError) as e:
                ctx.rx_chunk(st, chunk, t, 0.3)
            assert e.value.status == fq.ERR_INVALID
    finally:
        st.free()


# ----------------------------------------------------------------- swap --

@pytest.mark.parametrize("n,out,inn,k", [
    (12, 0, 6, 6), (14, 0, 5, 5), (16, 2, 9, 4), (13, 0, 12, 1), (20, 0, 10, 10),
    (18, 7, 11, 3), (20, 0, 12, 8), (15, 3, 8, 5), (22, 0, 11, 11), (21, 9, 18, 3),
    (10, 0, 1, 1), (24, 0, 12, 12),
    # small blocks whose sub-tile rows take in the free bits above the out
    # block (the reference's last swap of a layer, e.g. swap(0, 24, 2) at N=26)
    (16, 0, 10, 2), (20, 0, 18, 2), (14, 1, 7, 3), (18, 0, 14, 4), (26, 0, 24, 2),
])
def test_swap_blocks_vs_oracle(ctx, oracle, n, out, inn, k):
    rng = np.random.default_rng(n * 31 + k)
    v = rand_state(rng, n)
    st = ctx.state(n)
    try:
        st.from_host(v)
        ctx.swap_blocks(st, out, inn, k)
        want = v.copy()
        oracle.swap_gate_conti(want, n, out, inn, k)
        assert np.array_equal(st.to_host(), want)  # pure data movement: bit-exact
    finally:
        st.free()


# ----------------------------------------------- reference golden vectors --

def _check_golden(d, sv):
    if "state" in d.files:
        assert_state_close(sv, d["state"], what="vs reference output")
    else:
        ref = d["sample_amp"]
        assert np.abs(sv[d["sample_idx"]] - ref).max() <= 1e-12 * np.abs(ref).max()
        blocks = (np.abs(sv) ** 2).reshape(256, -1).sum(axis=1)
        assert np.abs(blocks - d["abs2_sum_by_block"]).max() <= 1e-12


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=[os.path.basename(p) for p in GOLDEN_FILES])
def test_reference_schedule_vs_golden(ctx, path):
    """The reference's own layer loop through our per-launcher kernels
    reproduces the reference's output, physical order and relabelled graph."""
    d = np.load(path)
    n = int(d["n"])
    st = ctx.state(n)
    try:
        gfin = ctx.reference_schedule(st, d["graph"], int(d["C"]), d["gammas"], d["betas"])
        _check_golden(d, st.to_host())
        assert np.array_equal(gfin, d["graph_final"])
    finally:
        st.free()


@pytest.mark.parametrize("path", GOLDEN_FILES, ids=[os.path.basename(p) for p in GOLDEN_FILES])
def test_fused_engine_vs_golden(ctx, fq, path):
    """The fused engine (logical order) permuted into the reference's
    physical order reproduces the reference's output."""
    d = np.load(path)
    n = int(d["n"])
    P = len(d["gammas"])
    st, ph = ctx.state(n), ctx.state(n)
    try:
        ctx.qaoa_forward(st, d["graph"], d["gammas"], d["betas"], energy=False)
        lab = fq.reference_label_map(n, int(d["C"]), P)
        inv = np.argsort(lab)
        ctx.permute_qubits(st, ph, inv)
        _check_golden(d, ph.to_host())
    finally:
        st.free()
        ph.free()


# --------------------------------------------------------- fused engine --

@pytest.mark.parametrize("n,P,kind", [
    (2, 1, "int"), (3, 2, "fp"), (7, 3, "neg"), (11, 2, "int"), (12, 1, "int"), (12, 3, "fp"),
    (13, 2, "neg"), (16, 4, "int"), (17, 2, "sparse"), (20, 3, "fp"), (21, 2, "int"),
    (22, 2, "int"), (14, 2, "wide"), (15, 2, "huge"), (16, 1, "zero"),
    # paired strided tiles with FP64 weights (phases from products of
    # exponentials): rows of 4 (N=22) and 2 (N=23) amplitudes
    (22, 3, "fp"), (23, 2, "fp"), (23, 3, "huge"),
])
def test_fused_forward_vs_oracle(ctx, oracle, n, P, kind):
    rng = np.random.default_rng(n * 13 + P)
    W = graph_of(kind, n, rng)
    g, b = angles(rng, P)
    st = ctx.state(n)
    try:
        e = ctx.qaoa_forward(st, W, g, b, energy=True)
        want = oracle.qaoa_logical(W, g, b)
        assert_state_close(st.to_host(), want, what="fused forward")
        ew = oracle.expectation(want, W)
        assert abs(e - ew) <= ENERGY_RTOL * abs(ew)
    finally:
        st.free()


def test_tile_cut_tables_follow_graph_and_size(fq):
    """The per-tile cut tables a context keeps between calls are rebuilt when
    the weights or N change: every call matches a fresh context bit for bit,
    whatever ran on the context before it."""
    rng = np.random.default_rng(77)
    graphs = {21: [complete_int(21, rng), gnp_fp(21, rng)], 22: [complete_int(22, rng)]}
    g, b = angles(rng, 3)
    order = [(21, 0), (21, 0), (21, 1), (22, 0), (21, 0), (21, 1), (21, 1)]
    fresh = {}
    for n, i in set(order):
        c = fq.Context(0)
        try:
            st = c.state(n)
            e = c.qaoa_forward(st, graphs[n][i], g, b, energy=True)
            fresh[(n, i)] = (st.to_host(), e)
            st.free()
        finally:
            c.close()
    c = fq.Context(0)
    try:
        for n, i in order:
            st = c.state(n)
            e = c.qaoa_forward(st, graphs[n][i], g, b, energy=True)
            got = st.to_host()
            st.free()
            want, ew = fresh[(n, i)]
            assert np.array_equal(got, want), (n, i)
            assert e == ew, (n, i)
    finally:
        c.close()


@pytest.mark.parametrize("beta", [0.0, np.pi / 2 - 1e-9, 2.5, np.pi, 4.0, -1.0, 7.0])
def test_fused_forward_mixer_angle_range(ctx, oracle, beta):
    """Both reduced-gate forms (tan and cot) and angles outside [0, pi/2)."""
    n, P = 14, 2
    rng = np.random.default_rng(11)
    W = complete_int(n, rng)
    g = rng.uniform(0, np.pi, P)
    b = np.array([beta, 0.3])
    st = ctx.state(n)
    try:
        ctx.qaoa_forward(st, W, g, b, energy=False)
        assert_state_close(st.to_host(), oracle.qaoa_logical(W, g, b), what="beta=%g" % beta)
    finally:
        st.free()


def test_expectation_vs_oracle(ctx, oracle):
    rng = np.random.default_rng(21)
    for n, kind in [(9, "int"), (12, "fp"), (16, "neg"), (18, "int")]:
        W = graph_of(kind, n, rng)
        v = rand_state(rng, n)
        st = ctx.state(n)
        try:
            st.from_host(v)
            e = ctx.expectation(st, W)
            ew = oracle.expectation(v, W)
            assert abs(e - ew) <= ENERGY_RTOL * abs(ew)
        finally:
            st.free()


def test_permute_qubits_vs_oracle(ctx, oracle):
    rng = np.random.default_rng(3)
    n = 13
    v = rand_state(rng, n)
    perm = rng.permutation(n)
    a, b = ctx.state(n), ctx.state(n)
    try:
        a.from_host(v)
        ctx.permute_qubits(a, b, perm)
        assert np.array_equal(b.to_host(), oracle.permute_qubits(v, perm))
    finally:
        a.free()
        b.free()


def test_config1_k20_p5(ctx, oracle):
    """Benchmark config 1: K_20, integer weights 1..10, p = 5, full state."""
    rng = np.random.default_rng(2020)
    W = complete_int(20, rng)
    g, b = angles(rng, 5)
    st = ctx.state(20)
    try:
        e = ctx.qaoa_forward(st, W, g, b)
        want = oracle.qaoa_logical(W, g, b)
        assert_state_close(st.to_host(), want)
        ew = oracle.expectation(want, W)
        assert abs(e - ew) <= ENERGY_RTOL * ew
    finally:
        st.free()


# ------------------------------------------------ full-size properties --

def test_kat_gamma_zero_n28(ctx):
    """gamma = 0: RX(b)|+> = exp(-ib/2)|+>, so every amplitude equals
    2^(-N/2) exp(-i N sum(b) / 2) exactly up to rounding."""
    n, P = 28, 3
    rng = np.random.default_rng(28)
    W = complete_int(n, rng)
    b = rng.uniform(0, np.pi / 2, P)
    st = ctx.state(n)
    try:
        e = ctx.qaoa_forward(st, W, np.zeros(P), b)
        v = st.to_host()
        want = 2.0 ** (-n / 2) * np.exp(-1j * n * b.sum() / 2)
        assert np.abs(v - want).max() <= 1e-12 * abs(want)
        assert abs(e - W.sum() / 2) <= ENERGY_RTOL * W.sum()
    finally:
        st.free()


def test_engines_agree_n26(ctx, fq):
    """Two independent GPU paths at N=26: the fused engine and the reference
    schedule (cost / RX chunks of 13 / block swaps), mapped to one order."""
    n, P, C = 26, 3, 13
    rng = np.random.default_rng(26)
    W = complete_int(n, rng)
    g, b = angles(rng, P)
    a, r, ph = ctx.state(n), ctx.state(n), ctx.state(n)
    try:
        ea = ctx.qaoa_forward(a, W, g, b)
        gfin = ctx.reference_schedule(r, W, C, g, b)
        er = ctx.expectation(r, gfin)
        assert abs(ea - er) <= ENERGY_RTOL * ea
        lab = fq.reference_label_map(n, C, P)
        ctx.permute_qubits(a, ph, np.argsort(lab))
        assert_state_close(ph.to_host(), r.to_host(), what="fused vs reference schedule")
    finally:
        for s in (a, r, ph):
            s.free()


def test_state_diff_matches_host(ctx):
    rng = np.random.default_rng(5)
    n = 15
    a = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    b = a + 1e-9 * (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n))
    sa, sb = ctx.state(n), ctx.state(n)
    try:
        sa.from_host(a)
        sb.from_host(b)
        d = ctx.state_diff(sa, sb)
    finally:
        sa.free()
        sb.free()
    assert d["max_abs_diff"] == pytest.approx(np.abs(a - b).max(), rel=1e-12)
    assert d["max_abs_b"] == pytest.approx(np.abs(b).max(), rel=1e-12)
    assert d["l2_diff"] == pytest.approx(np.linalg.norm(a - b), rel=1e-10)
    assert d["l2_b"] == pytest.approx(np.linalg.norm(b), rel=1e-12)


@pytest.mark.parametrize("kind", ["int", "fp"])
def test_config2_n30_p5_full_state(ctx, fq, kind):
    """Benchmark config 2 (K_30, integer weights 1..10, p=5, C=12) at full
    size, and the same with FP64 weights (G(30, 0.5)): the fused engine
    against the reference schedule (cost sweep, RX chunks of C=12, block
    swaps) on every one of the 2^30 amplitudes, in one qubit order,
    compared on the device (1e-12 of max|psi| and relative L2).  At N=30 the
    engine's layer-0 pass runs on paired strided tiles with the lane-bit
    qubit, alternating its exchange direction from tile to tile."""
    n, P, C = 30, 5, 12
    rng = np.random.default_rng(30)
    W = complete_int(n, rng) if kind == "int" else gnp_fp(n, rng)
    g, b = angles(rng, P)
    a, r, ph = ctx.state(n), ctx.state(n), ctx.state(n)
    try:
        ea = ctx.qaoa_forward(a, W, g, b)
        gfin = ctx.reference_schedule(r, W, C, g, b)
        er = ctx.expectation(r, gfin)
        lab = fq.reference_label_map(n, C, P)
        ctx.permute_qubits(a, ph, np.argsort(lab))
        d = ctx.state_diff(ph, r)
    finally:
        for s in (a, r, ph):
            s.free()
    assert abs(ea - er) <= ENERGY_RTOL * ea
    assert d["max_abs_diff"] <= STATE_RTOL * d["max_abs_b"], d
    assert d["l2_diff"] <= STATE_RTOL * d["l2_b"], d


def test_weighted_cli_engines_agree():
    exe = os.path.join(PKG, "weighted")
    with tempfile.TemporaryDirectory() as td:
        outs, es = [], []
        for eng in ("reference", "fused"):
            f = os.path.join(td, eng + ".bin")
            r = subprocess.run([exe, "3", "14", "0", "5", "14", "--engine", eng, "--weights",
                                "int", "--angles", "random", "--seed", "3", "--expect",
                                "--dump", f], capture_output=True, text=True, timeout=120)
            assert r.returncode == 0, r.stderr
            assert "Total simulation time" in r.stdout
            es.append(float(r.stdout.split("<C> :")[1].split()[0]))
            outs.append(np.fromfile(f, dtype=np.complex128))
        assert_state_close(outs[1], outs[0], what="CLI fused vs reference")
        assert abs(es[0] - es[1]) <= ENERGY_RTOL * es[0]


@pytest.mark.parametrize("engine", ["fused", "reference"])
def test_weighted_cli_dump_validates(engine):
    """The CLI's dump with its label-map and circuit sidecars passes the
    independent dense check (validate_dump.py), for a weighted graph whose
    state does change under a wrong relabelling."""
    exe = os.path.join(PKG, "weighted")
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "s.bin")
        r = subprocess.run([exe, "3", "13", "0", "5", "13", "--engine", engine, "--weights",
                            "int", "--angles", "random", "--seed", "7", "--dump", f],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        v = subprocess.run([sys.executable, os.path.join(PKG, "validate_dump.py"), f, "13", "3",
                            "--tol", "1e-12"], capture_output=True, text=True, timeout=300)
        assert v.returncode == 0, v.stdout + v.stderr
        assert v.stdout.startswith("PASS")


def test_weighted_cli_rejects_multi_device():
    exe = os.path.join(PKG, "weighted")
    r = subprocess.run([exe, "1", "12", "1", "4", "8"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and "D=1" in r.stderr


def test_refapi_unweighted_bitmask_path(fq, oracle, tmp_path):
    """A program written against the reference-style C++ API only
    (tests/refapi_unweighted.cpp, compiled here against include/refapi and
    libforqaoa.so) runs the reference's layer loop on an unweighted graph of
    64-bit neighbour masks; its state, mapped through the reference's label
    map, matches the oracle on the same unit-weight graph."""
    import shutil
    cxx = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "refapi_unweighted"
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(os.path.dirname(here), "include")
    r = subprocess.run([cxx, "-std=c++17", "-I", inc, os.path.join(here, "refapi_unweighted.cpp"),
                        "-L", PKG, "-lforqaoa", "-Xlinker", "-rpath=" + PKG, "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    N, P, C = 14, 2, 5
    out = tmp_path / "s.bin"
    r = subprocess.run([str(exe), str(P), str(N), str(C), "11", str(out)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    W = np.zeros((N, N))
    for line in open(str(out) + ".edges"):
        i, j = map(int, line.split())
        W[i, j] = 1.0
    want = oracle.qaoa_logical(W, np.full(P, 0.7), np.full(P, 0.45))
    phys = np.fromfile(out, dtype=np.complex128)
    lab = fq.reference_label_map(N, C, P)
    y = np.arange(1 << N)
    x = np.zeros_like(y)
    for b, q in enumerate(lab):
        x |= ((y >> b) & 1) << int(q)
    got = np.empty_like(phys)
    got[x] = phys
    assert_state_close(got, want, what="C++ API, unweighted graph")


def test_refapi_state_setup_and_copies(oracle, tmp_path):
    """stateCpyHostToDevice, stateInitDeviceState and prepare
    (src/state.cpp:162-219,328-336) through a program written only against
    the reference-style C++ API (tests/refapi_state_io.cpp): an uploaded host
    state is what the next kernel (multiRotateX on the first C qubits) acts
    on, checked against the oracle; the device state resets to |0...0>; the
    chunk size is recorded and C < 1 is refused."""
    import shutil
    cxx = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path / "refapi_state_io"
    here = os.path.dirname(os.path.abspath(__file__))
    inc = os.path.join(os.path.dirname(here), "include")
    r = subprocess.run([cxx, "-std=c++17", "-I", inc, os.path.join(here, "refapi_state_io.cpp"),
                        "-L", PKG, "-lforqaoa", "-Xlinker", "-rpath=" + PKG, "-o", str(exe)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    N, C, angle = 15, 6, 0.83
    pre = tmp_path / "st"
    r = subprocess.run([str(exe), str(N), str(C), str(angle), str(pre)], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split("\n")[:4] == ["createState |0> ok", "stateCpyHostToDevice + multiRotateX ok",
                                        "stateInitDeviceState ok", "prepare ok"]
    sv_in = np.fromfile(str(pre) + ".in", dtype=np.complex128)
    got = np.fromfile(str(pre) + ".out", dtype=np.complex128)
    want = oracle.multi_rotate_x(sv_in.copy(), N, list(range(C)), angle)
    assert_state_close(got, want, what="host state uploaded, then RX on qubits 0..C-1")
