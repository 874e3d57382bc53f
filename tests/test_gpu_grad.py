"""GPU tests of the adjoint gradient (fq_qaoa_energy_grad): against the FP64
CPU adjoint of the oracle (1e-8, relative to max(1, |g|)), against central
finite differences of the GPU energy, the benchmark config of 26 qubits and
10 layers, and the reverse sweep's two schedules (fused two-layer passes,
the default, and one sweep per pass with FQ_FUSE=0) over every tile
schedule a layer-completing pass can have."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ENERGY_RTOL, GRAD_TOL, PKG, complete_int, gnp_fp, gnp_int, angles

pytestmark = pytest.mark.gpu


def graph_of(kind, n, rng):
    return {"int": complete_int(n, rng), "fp": gnp_fp(n, rng), "neg": complete_int(n, rng, -5, 5),
            "sparse": gnp_int(n, rng, 0.3), "wide": complete_int(n, rng, 1, 500),
            "huge": complete_int(n, rng, 1, 5000), "zero": np.zeros((n, n))}[kind]


def check_grad(got, want):
    scale = max(1.0, np.abs(want).max())
    err = np.abs(np.asarray(got) - np.asarray(want)).max()
    assert err <= GRAD_TOL * scale, "grad err %.3e (scale %.3e)" % (err, scale)


@pytest.mark.parametrize("n,P,kind", [
    (2, 1, "int"), (4, 3, "fp"), (7, 2, "neg"), (10, 4, "int"), (12, 3, "fp"), (12, 2, "int"),
    (13, 2, "int"), (14, 3, "fp"), (16, 2, "neg"), (17, 3, "sparse"), (20, 2, "int"),
    (21, 2, "fp"), (14, 2, "wide"), (15, 2, "huge"), (10, 2, "wide"), (14, 2, "zero"),
    (9, 3, "zero"),
])
def test_energy_grad_vs_oracle(ctx, oracle, n, P, kind):
    rng = np.random.default_rng(7 * n + P)
    W = graph_of(kind, n, rng)
    g, b = angles(rng, P)
    e, gg, gb = ctx.energy_grad(n, W, g, b)
    eo, ggo, gbo = oracle.energy_grad(W, g, b)
    assert abs(e - eo) <= ENERGY_RTOL * max(1.0, abs(eo))
    check_grad(gg, ggo)
    check_grad(gb, gbo)


@pytest.mark.parametrize("n", [9, 15])
def test_energy_grad_vs_finite_differences(ctx, n):
    rng = np.random.default_rng(n)
    W = complete_int(n, rng)
    P = 3
    g, b = angles(rng, P)
    _, gg, gb = ctx.energy_grad(n, W, g, b)
    st = ctx.state(n)
    h = 1e-6
    try:
        def E(gv, bv):
            return ctx.qaoa_forward(st, W, gv, bv)
        fd_g = [(E(g + h * np.eye(P)[k], b) - E(g - h * np.eye(P)[k], b)) / (2 * h)
                for k in range(P)]
        fd_b = [(E(g, b + h * np.eye(P)[k]) - E(g, b - h * np.eye(P)[k])) / (2 * h)
                for k in range(P)]
    finally:
        st.free()
    # Central differences carry ~eps*|E|/h of roundoff: compare relative to scale.
    scale = max(1.0, np.abs(gg).max(), np.abs(gb).max())
    assert np.abs(gg - fd_g).max() <= 1e-6 * scale
    assert np.abs(gb - fd_b).max() <= 1e-6 * scale


def test_config4_n26_p10(ctx, oracle):
    """Benchmark config 4: K_26, integer weights 1..10, p = 10."""
    rng = np.random.default_rng(2610)
    W = complete_int(26, rng)
    g, b = angles(rng, 10)
    e, gg, gb = ctx.energy_grad(26, W, g, b)
    eo, ggo, gbo = oracle.energy_grad(W, g, b)
    assert abs(e - eo) <= ENERGY_RTOL * abs(eo)
    check_grad(gg, ggo)
    check_grad(gb, gbo)


def test_energy_grad_matches_forward_energy(ctx):
    rng = np.random.default_rng(5)
    n = 18
    W = gnp_fp(n, rng)
    g, b = angles(rng, 4)
    e, _, _ = ctx.energy_grad(n, W, g, b)
    st = ctx.state(n)
    try:
        ef = ctx.qaoa_forward(st, W, g, b)
    finally:
        st.free()
    assert abs(e - ef) <= ENERGY_RTOL * abs(ef)


GRAD_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, %(pkg)r)
import forqaoa
cases = json.loads(sys.stdin.read())
out = []
with forqaoa.Context(0) as ctx:
    for c in cases:
        e, gg, gb = ctx.energy_grad(c["n"], np.array(c["W"]), np.array(c["g"]), np.array(c["b"]))
        out.append({"e": e, "gg": gg.tolist(), "gb": gb.tolist()})
print(json.dumps(out))
"""


# The pass that completes a layer alternates between the contiguous pass and
# the last strided pass, whose tile schedule is L0 (N 16, 24), L01
# (17..21, 25..30) or L021 (22, 23) (up to 15 qubits the whole instance runs
# in shared memory, one CTA or one cluster); P = 1 has no fused pass; "huge" weights
# take one phase table per layer, FP64 weights with a large sum ("wide" plus
# a quarter) one sincos per amplitude.
@pytest.mark.parametrize("fuse", ["1", "0"])
def test_reverse_schedules_match_oracle(oracle, fuse):
    rng = np.random.default_rng(404)
    cs = []
    for n, P, kind in ((13, 3, "int"), (16, 4, "fp"), (17, 2, "neg"), (20, 5, "int"),
                       (22, 3, "int"), (23, 4, "fp"), (24, 3, "int"), (24, 2, "huge"),
                       (21, 5, "wide"), (19, 4, "huge"), (25, 1, "int"), (18, 6, "sparse")):
        W = graph_of(kind, n, rng)
        if kind == "wide":
            W = W + 0.25 * (W > 0)
        g, b = angles(rng, P)
        cs.append({"n": n, "W": W.tolist(), "g": g.tolist(), "b": b.tolist()})
    env = dict(os.environ, FQ_FUSE=fuse)
    res = subprocess.run([sys.executable, "-c", GRAD_CHILD % {"pkg": PKG}],
                         input=json.dumps(cs), capture_output=True, text=True, env=env,
                         timeout=900)
    assert res.returncode == 0, res.stderr[-2000:]
    got = json.loads(res.stdout.strip().splitlines()[-1])
    for c, r in zip(cs, got):
        eo, ggo, gbo = oracle.energy_grad(np.array(c["W"]), np.array(c["g"]), np.array(c["b"]))
        assert abs(r["e"] - eo) <= ENERGY_RTOL * abs(eo), c["n"]
        check_grad(r["gg"], ggo)
        check_grad(r["gb"], gbo)
