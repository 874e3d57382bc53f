"""GPU tests of the adjoint gradient (fq_qaoa_energy_grad): against the FP64
CPU adjoint of the oracle (1e-8, relative to max(1, |g|)), against central
finite differences of the GPU energy, and the benchmark config of 26 qubits
and 10 layers."""
import numpy as np
import pytest

from conftest import ENERGY_RTOL, GRAD_TOL, complete_int, gnp_fp, gnp_int, angles

pytestmark = pytest.mark.gpu


def graph_of(kind, n, rng):
    return {"int": complete_int(n, rng), "fp": gnp_fp(n, rng), "neg": complete_int(n, rng, -5, 5),
            "sparse": gnp_int(n, rng, 0.3), "wide": complete_int(n, rng, 1, 500),
            "huge": complete_int(n, rng, 1, 5000)}[kind]


def check_grad(got, want):
    scale = max(1.0, np.abs(want).max())
    err = np.abs(np.asarray(got) - np.asarray(want)).max()
    assert err <= GRAD_TOL * scale, "grad err %.3e (scale %.3e)" % (err, scale)


@pytest.mark.parametrize("n,P,kind", [
    (2, 1, "int"), (4, 3, "fp"), (7, 2, "neg"), (10, 4, "int"), (12, 3, "fp"), (12, 2, "int"),
    (13, 2, "int"), (14, 3, "fp"), (16, 2, "neg"), (17, 3, "sparse"), (20, 2, "int"),
    (21, 2, "fp"), (14, 2, "wide"), (15, 2, "huge"), (10, 2, "wide"),
])
def test_energy_grad_vs_oracle(ctx, oracle, n, P, kind):
    rng = np.random.default_rng(7 * n + P)
    W = graph_of(kind, n, rng)
    g, b = angles(rng, P)
    e, gg, gb = ctx.energy_grad(n, W, g, b)
    eo, ggo, gbo = oracle.energy_grad(W, g, b)
    assert abs(e - eo) <= ENERGY_RTOL * abs(eo)
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
