"""GPU tests of the serving loop (fq_server_*): a request gives the same
bits alone (fq_qaoa_energy_grad on a context of its own) and in a mix of
many requests of different sizes, batched and overlapped; sessions keep
their step order, stay under the HBM budget (idle ones evicted least
recently used first) and survive eviction; bad requests are refused."""
import numpy as np
import pytest

from conftest import ENERGY_RTOL, complete_int, gnp_fp, gnp_int, angles

pytestmark = pytest.mark.gpu


def session_bytes(n):
    return 2 * 16 * (1 << n)


def make_request(rng, n, P):
    kind = rng.integers(0, 3)
    W = (complete_int(n, rng), gnp_fp(n, rng), gnp_int(n, rng, 0.5))[kind]
    g, b = angles(rng, P)
    return W, g, b


def assert_same(res, alone):
    e, gg, gb = alone
    assert res.status == 0
    assert res.energy == e
    assert np.array_equal(res.grad_gamma, gg)
    assert np.array_equal(res.grad_beta, gb)


def test_mix_matches_alone(fq, ctx, oracle):
    rng = np.random.default_rng(2024)
    ns = [4, 6, 8, 10, 11, 12, 12, 13, 14, 15, 16, 18, 20, 3, 9, 12, 17, 5]
    reqs = [(i, n, *make_request(rng, n, int(rng.integers(1, 9)))) for i, n in
            enumerate(ns * 3)]
    alone = {i: ctx.energy_grad(n, W, g, b) for i, n, W, g, b in reqs}
    with fq.Server(0, 4e9, lanes=3) as srv:
        tickets = {srv.submit(i, W, g, b): i for i, n, W, g, b in reqs}
        done = srv.wait(tickets)
        st = srv.stats()
    assert st["pending"] == 0
    assert st["batched_requests"] + st["lane_requests"] == len(reqs)
    for t, i in tickets.items():
        assert done[t].session == i
        assert_same(done[t], alone[i])
    # And the mix agrees with the FP64 oracle on a few of them.
    for i, n, W, g, b in reqs[:6]:
        eo, _, _ = oracle.energy_grad(W, g, b)
        r = next(done[t] for t, j in tickets.items() if j == i)
        assert abs(r.energy - eo) <= ENERGY_RTOL * max(1.0, abs(eo))


def test_small_requests_share_launches(fq, ctx):
    """Requests of 2..15 qubits (one CTA up to 12, a cluster of 2, 4 or 8
    CTAs above) are batched, one launch per size class and batch."""
    rng = np.random.default_rng(11)
    reqs = [(i, *make_request(rng, int(rng.integers(2, fq.SMALL_MAX_QUBITS + 1)),
                              int(rng.integers(1, 9))))
            for i in range(600)]
    with fq.Server(0, 1e9, lanes=1) as srv:
        tickets = {srv.submit(i, W, g, b): i for i, W, g, b in reqs}
        done = srv.wait(tickets)
        st = srv.stats()
    assert st["batched_requests"] == len(reqs)
    assert st["kernel_launches"] < len(reqs)
    for t, i in list(tickets.items())[::7]:
        _, W, g, b = reqs[i]
        assert_same(done[t], ctx.energy_grad(W.shape[0], W, g, b))


def test_sessions_under_budget_with_eviction(fq, ctx):
    """Four 16-qubit sessions, a budget for two: each step is a gradient step
    on the previous one's angles; the results match the plain calls."""
    rng = np.random.default_rng(16)
    n, P, steps = 16, 3, 4
    graphs = [complete_int(n, rng) for _ in range(4)]
    ang = [list(angles(rng, P)) for _ in range(4)]
    budget = 2 * session_bytes(n) + 1024
    with fq.Server(0, budget, lanes=2) as srv:
        for _ in range(steps):
            tickets = {srv.submit(s, graphs[s], *ang[s]): s for s in range(4)}
            done = srv.wait(tickets)
            st = srv.stats()
            assert st["resident_bytes"] <= budget
            assert st["resident_sessions"] <= 2
            for t, s in tickets.items():
                assert_same(done[t], ctx.energy_grad(n, graphs[s], *ang[s]))
                ang[s][0] = ang[s][0] - 0.01 * done[t].grad_gamma
                ang[s][1] = ang[s][1] - 0.01 * done[t].grad_beta
        for s in range(4):
            srv.close_session(s)
        assert srv.stats()["resident_sessions"] == 0


def test_session_steps_keep_order(fq):
    rng = np.random.default_rng(3)
    W, g, b = make_request(rng, 14, 2)
    with fq.Server(0, 1e9, lanes=4) as srv:
        tickets = [srv.submit(7, W, g + 0.01 * k, b) for k in range(6)]
        done = srv.wait(tickets)
    runs = [done[t] for t in tickets]
    for a, b_ in zip(runs, runs[1:]):
        assert b_.t_start >= a.t_done - 1e-3  # host bookkeeping after the event
        assert a.t_submit <= a.t_start <= a.t_done


def test_bad_requests_are_refused(fq):
    rng = np.random.default_rng(0)
    with fq.Server(0, session_bytes(16), lanes=1) as srv:
        W, g, b = make_request(rng, 18, 2)
        with pytest.raises(fq.FQError) as e:
            srv.submit(1, W, g, b)
        assert e.value.status == fq.ERR_OOM
        W, g, b = make_request(rng, 10, fq.SERVE_MAX_LAYERS + 1)
        with pytest.raises(fq.FQError):
            srv.submit(1, W, g, b)
        W, g, b = make_request(rng, 10, 2)
        g[0] = np.nan
        with pytest.raises(fq.FQError):
            srv.submit(1, W, g, b)
        # The server still serves after refusals.
        W, g, b = make_request(rng, 16, 2)
        t = srv.submit(2, W, g, b)
        assert srv.wait([t])[t].status == 0


def test_native_replay_served_equals_one_at_a_time():
    """The stream driven natively (serve_replay, no Python in the request
    loop): every served result is bit-identical to the same evaluation run
    one at a time, with buffers reused per session and with a plain call per
    evaluation; every session's steps come back in order."""
    import serve_stream as ss
    sessions, steps = ss.make_stream(240, seed=9, steps=6, n_min=4, n_max=19, p_max=6,
                                     mean_gap_ms=0.2)
    served, wall, info = ss.run_native("served", sessions, steps, lanes=3, budget=8e9)
    seq, wall_q, _ = ss.run_native("sequential", sessions, steps)
    plain, wall_p, _ = ss.run_native("plain", sessions, steps)
    assert len(served) == len(seq) == len(plain) == len(sessions) * steps
    assert info["batched_requests"] + info["lane_requests"] == len(served)
    assert info["batched_requests"] > 0 and info["lane_requests"] > 0
    assert ss.compare(served, seq) == 0
    assert ss.compare(served, plain) == 0
    last = {}
    for r in served:
        assert r["step"] == last.get(r["session"], -1) + 1
        last[r["session"]] = r["step"]


def test_native_replay_large_sizes_on_concurrent_lanes():
    """Sessions of N = 21..24 on four lanes at once (each lane's context
    builds its own per-tile cut tables while the others run): every served
    result is bit-identical to the same evaluation run one at a time."""
    import serve_stream as ss
    sessions, steps = ss.make_stream(48, seed=21, steps=3, n_min=21, n_max=24, p_max=3,
                                     mean_gap_ms=0.05)
    served, wall, info = ss.run_native("served", sessions, steps, lanes=4, budget=20e9)
    seq, wall_q, _ = ss.run_native("sequential", sessions, steps)
    assert len(served) == len(seq) == len(sessions) * steps
    assert info["lane_requests"] == len(served)
    assert ss.compare(served, seq) == 0
