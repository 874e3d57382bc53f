"""The failure path on the GPU without a fault: a kernel's bounded wait on a
barrier that nothing completes gives up, the host reads FQ_ERR_TIMEOUT at
the next synchronising call, and the same context then computes correct
results (fq_ctx_selftest_wait)."""
import time

import numpy as np
import pytest

from conftest import ENERGY_RTOL, assert_state_close, complete_int, angles

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_context_stays_usable(fq, ctx, oracle):
    t0 = time.monotonic()
    assert fq.lib().fq_ctx_selftest_wait(ctx.handle) == fq.OK
    with pytest.raises(fq.FQError) as e:
        ctx.synchronize()
    assert e.value.status == fq.ERR_TIMEOUT
    assert time.monotonic() - t0 < 10.0  # 2^16 polls (0.26 s); the pipelines' bound is 2^18
    ctx.synchronize()  # the flag was cleared with the report
    rng = np.random.default_rng(99)
    W = complete_int(16, rng)
    g, b = angles(rng, 2)
    st = ctx.state(16)
    try:
        e = ctx.qaoa_forward(st, W, g, b)
        psi = st.to_host()
    finally:
        st.free()
    want = oracle.qaoa_logical(W, g, b)
    assert_state_close(psi, want)
    assert abs(e - oracle.expectation(want, W)) <= ENERGY_RTOL * abs(e)
