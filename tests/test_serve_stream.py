"""CPU tests of the served-stream driver (serve_stream.py) against fakes of
the server and the context that compute with the oracle and complete
requests out of order: the closed loop submits each session's steps in
order, both runs evaluate the same requests, and the comparison and the
summary count what they should."""
import numpy as np
import pytest

import serve_stream as ss


class _R:
    def __init__(self, ticket, session, N, P, e, gg, gb, t):
        self.ticket, self.session, self.N, self.P = ticket, session, N, P
        self.status, self.energy, self.grad_gamma, self.grad_beta = 0, e, gg, gb
        self.t_submit, self.t_start, self.t_done = t, t + 1e-4, t + 2e-4


class FakeFQ:
    SMALL_MAX_QUBITS = 15  # the library's FQ_SMALL_MAX_QUBITS

    def __init__(self, oracle, seed=0):
        self.rng = np.random.default_rng(seed)
        self.submitted = []
        cache = {}

        class Det:
            # The oracle's OpenMP sums may combine thread partials in any
            # order; the fakes return one answer per distinct input.
            @staticmethod
            def energy_grad(graph, g, b):
                key = (graph.tobytes(), np.asarray(g).tobytes(), np.asarray(b).tobytes())
                if key not in cache:
                    cache[key] = oracle.energy_grad(graph, g, b)
                return cache[key]
        self.oracle = Det

    def Server(self, device, budget, lanes):
        fake = self

        class S:
            def __init__(self):
                self.queue, self.t = [], 0

            def submit(self, sid, graph, g, b):
                self.t += 1
                fake.submitted.append((sid, np.array(g), np.array(b)))
                e, gg, gb = fake.oracle.energy_grad(graph, g, b)
                self.queue.append(_R(self.t, sid, graph.shape[0], len(g), e, gg, gb, 0.0))
                return self.t

            def poll(self, n, wait_ms=0):
                fake.rng.shuffle(self.queue)  # completion order differs from submission
                k = int(fake.rng.integers(0, len(self.queue) + 1)) if self.queue else 0
                out, self.queue = self.queue[:max(k, 1)], self.queue[max(k, 1):]
                return out

            def close_session(self, sid):
                pass

            def stats(self):
                return {"pending": len(self.queue)}

            def close(self):
                pass
        return S()

    def Context(self, device):
        fake = self

        class C:
            def state(self, n):
                class St:
                    def free(self):
                        pass
                return St()

            def energy_grad(self, n, graph, g, b, sv=None, costate=None):
                return fake.oracle.energy_grad(graph, g, b)

            def close(self):
                pass
        return C()


def test_stream_distribution():
    sessions, steps = ss.make_stream(2000, seed=1)
    assert steps == 20 and len(sessions) == 100
    ns = [s["N"] for s in sessions]
    assert min(ns) >= 10 and max(ns) <= 28
    assert all(1 <= s["P"] <= 8 for s in sessions)
    for s in sessions[:5]:
        w = s["graph"]
        assert np.all(np.tril(w) == 0)
        nz = w[w != 0]
        assert nz.min() >= 1 and nz.max() <= 10 and np.all(nz == np.rint(nz))
    arr = [s["arrival"] for s in sessions]
    assert arr == sorted(arr)


def test_closed_loop_matches_sequential(oracle):
    sessions, steps = ss.make_stream(24, seed=3, steps=4, n_min=3, n_max=7, p_max=3,
                                     mean_gap_ms=0.0)
    fq = FakeFQ(oracle)
    served, wall, stats = ss.run_served(fq, sessions, steps)
    assert len(served) == len(sessions) * steps
    # Every session's steps were submitted in order, each from the previous gradient.
    for s in sessions:
        subs = [(g, b) for sid, g, b in fq.submitted if sid == s["id"]]
        assert len(subs) == steps
        assert np.array_equal(subs[0][0], s["gammas"])
        steps_of = sorted((r for r in served if r["session"] == s["id"]),
                          key=lambda r: r["step"])
        for k in range(1, steps):
            want = ss.next_angles(*subs[k - 1], steps_of[k - 1]["grad_gamma"],
                                  steps_of[k - 1]["grad_beta"])
            assert np.array_equal(subs[k][0], want[0])
            assert np.array_equal(subs[k][1], want[1])
    seq, wall_q = ss.run_sequential(fq, sessions, steps)
    assert ss.compare(served, seq) == 0
    out = ss.summarize(served, wall, seq, wall_q, stats)
    assert out["requests"] == len(served)
    assert out["mismatches_vs_sequential"] == 0
    assert sum(b["requests"] for b in out["buckets"].values()) == len(served)


def test_compare_counts_a_planted_difference(oracle):
    sessions, steps = ss.make_stream(6, seed=4, steps=2, n_min=3, n_max=5, p_max=2,
                                     mean_gap_ms=0.0)
    fq = FakeFQ(oracle)
    seq, _ = ss.run_sequential(fq, sessions, steps)
    served = [dict(r) for r in seq]
    served[1]["energy"] = np.nextafter(served[1]["energy"], np.inf)
    for r in served:
        r["queue"] = 0.0
    assert ss.compare(served, seq) == 1
