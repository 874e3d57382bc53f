"""GPU test of fq_expectation_noalloc, the <C> entry point for callers that
cannot allocate device memory (their memory belongs to another allocator,
or cudaMalloc's implicit synchronisation is not acceptable to them).

It is called through the C ABI on states made by the library, twice in a
row on the same inputs, and must match the allocating entry point
fq_expectation within the energy tolerance of the parity tests.  The file
is named to be collected last, and must pass alone in a fresh process as
well as after the other tests (the first call on a device sets up the
scratch address)."""
import ctypes

import numpy as np
import pytest

from conftest import ENERGY_RTOL, complete_int, gnp_fp, angles

pytestmark = pytest.mark.gpu


def noalloc_energy(fq, st, W, stream):
    g = np.ascontiguousarray(W, dtype=np.float64)
    e = np.zeros(1)
    dp = ctypes.POINTER(ctypes.c_double)
    status = fq.lib().fq_expectation_noalloc(st.ptr, st.n, g.ctypes.data_as(dp),
                                             e.ctypes.data_as(dp), stream)
    if status != fq.OK:
        raise fq.FQError(status, "fq_expectation_noalloc")
    return float(e[0])


@pytest.mark.parametrize("n,kind", [(6, "int"), (11, "fp"), (12, "int"), (17, "fp"),
                                    (20, "int"), (23, "int")])
def test_noalloc_expectation_matches(ctx, fq, n, kind):
    rng = np.random.default_rng(100 + n)
    W = complete_int(n, rng) if kind == "int" else gnp_fp(n, rng)
    g, b = angles(rng, 2)
    st = ctx.state(n)
    try:
        ctx.qaoa_forward(st, W, g, b, energy=False)
        want = ctx.expectation(st, W)
        for _ in range(2):  # the shared scratch keeps the previous call's contents
            got = noalloc_energy(fq, st, W, ctx.stream)
            assert abs(got - want) <= ENERGY_RTOL * abs(want), (got, want)
    finally:
        st.free()


def test_noalloc_rejects_sizes_beyond_the_scratch(ctx, fq):
    st = ctx.state(12)
    try:
        W = np.zeros((40, 40))
        e = np.zeros(1)
        dp = ctypes.POINTER(ctypes.c_double)
        status = fq.lib().fq_expectation_noalloc(st.ptr, 40, W.ctypes.data_as(dp),
                                                 e.ctypes.data_as(dp), ctx.stream)
        assert status == fq.ERR_INVALID
        assert b"outside" in fq.lib().fq_last_error()
    finally:
        st.free()
