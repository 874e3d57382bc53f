#!/usr/bin/env python3
"""Served request stream: QAOA energy+gradient evaluations of uneven size and
depth, run through the serving loop (fq_server_*) and, for comparison, as
sequential plain calls of fq_qaoa_energy_grad, one evaluation at a time.

Stream: sessions of `steps` energy+gradient evaluations each (an optimiser
loop: every step moves the angles against the previous step's gradient),
sessions arriving as a Poisson process.  Each session draws N uniformly from
[n_min, n_max], p uniformly from [1, p_max] and an Erdos-Renyi G(N, 0.5)
graph with integer weights in 1..10, all from one seed.

Both runs evaluate exactly the same requests: the gradients, and therefore
the angle trajectories, are bit-identical alone and in the mix, which the
comparison checks for every request.

    python serve_stream.py --requests 10000       # the full 10k stream
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

BUCKETS = ((2, 15, "one CTA or cluster each (N<=15)"), (16, 20, "lanes, N 16..20"),
           (21, 33, "lanes, N 21..28"))


def make_stream(n_requests, seed, steps=20, n_min=10, n_max=28, p_max=8, mean_gap_ms=1.0):
    rng = np.random.default_rng(seed)
    n_sessions = max(1, n_requests // steps)
    sessions = []
    t = 0.0
    for s in range(n_sessions):
        n = int(rng.integers(n_min, n_max + 1))
        P = int(rng.integers(1, p_max + 1))
        w = np.triu(rng.integers(1, 11, size=(n, n)).astype(np.float64), 1)
        w *= np.triu(rng.random((n, n)) < 0.5, 1)
        sessions.append({"id": s, "N": n, "P": P, "graph": w,
                         "gammas": rng.uniform(0, np.pi, P), "betas": rng.uniform(0, np.pi / 2, P),
                         "arrival": t})
        t += rng.exponential(mean_gap_ms / 1000.0)
    return sessions, steps


def next_angles(g, b, gg, gb):
    """One optimiser step (deterministic, so both runs follow the same path)."""
    s = 0.05 / max(1.0, float(np.abs(gg).max()), float(np.abs(gb).max()))
    return g - s * gg, b - s * gb


def run_served(fq, sessions, steps, device=0, lanes=4, budget=150e9):
    """Closed-loop sessions through the server; returns (records, wall_s, stats)."""
    srv = fq.Server(device, budget, lanes)
    order = sorted(sessions, key=lambda s: s["arrival"])
    ang = {s["id"]: (s["gammas"].copy(), s["betas"].copy()) for s in sessions}
    left = {s["id"]: steps for s in sessions}
    by_id = {s["id"]: s for s in sessions}
    recs = []
    nxt = 0
    outstanding = 0
    try:
        t0 = time.monotonic()
        while nxt < len(order) or outstanding:
            now = time.monotonic() - t0
            while nxt < len(order) and order[nxt]["arrival"] <= now:
                s = order[nxt]
                srv.submit(s["id"], s["graph"], *ang[s["id"]])
                outstanding += 1
                nxt += 1
            wait = 0 if nxt < len(order) else 20
            for r in srv.poll(4096, wait_ms=wait):
                outstanding -= 1
                if r.status != 0:
                    raise RuntimeError(f"request {r.ticket} failed with status {r.status}")
                sid = r.session
                g, b = ang[sid]
                recs.append({"session": sid, "step": steps - left[sid], "N": r.N, "P": r.P,
                             "energy": r.energy, "grad_gamma": r.grad_gamma,
                             "grad_beta": r.grad_beta, "latency": r.t_done - r.t_submit,
                             "queue": r.t_start - r.t_submit})
                left[sid] -= 1
                ang[sid] = next_angles(g, b, r.grad_gamma, r.grad_beta)
                if left[sid]:
                    srv.submit(sid, by_id[sid]["graph"], *ang[sid])
                    outstanding += 1
                else:
                    srv.close_session(sid)
        wall = time.monotonic() - t0
        stats = srv.stats()
    finally:
        srv.close()
    return recs, wall, stats


def run_sequential(fq, sessions, steps, device=0, reuse=True):
    """The same evaluations one at a time through fq_qaoa_energy_grad.
    reuse: state and costate allocated once per session; otherwise every
    call allocates and frees its own (a plain call of the public API)."""
    ctx = fq.Context(device)
    recs = []
    try:
        t0 = time.monotonic()
        for s in sorted(sessions, key=lambda s: s["arrival"]):
            n = s["N"]
            sv = cs = None
            if n > fq.SMALL_MAX_QUBITS and reuse:
                sv, cs = ctx.state(n), ctx.state(n)
            g, b = s["gammas"].copy(), s["betas"].copy()
            for k in range(steps):
                t1 = time.monotonic()
                e, gg, gb = ctx.energy_grad(n, s["graph"], g, b, sv=sv, costate=cs)
                recs.append({"session": s["id"], "step": k, "N": n, "P": s["P"], "energy": e,
                             "grad_gamma": gg, "grad_beta": gb,
                             "latency": time.monotonic() - t1})
                g, b = next_angles(g, b, gg, gb)
            if sv is not None:
                sv.free()
                cs.free()
        wall = time.monotonic() - t0
    finally:
        ctx.close()
    return recs, wall


REPLAY = os.path.join(HERE, "serve_replay")


def write_stream(sessions, steps, path):
    """The stream in serve_replay's input format."""
    with open(path, "wb") as f:
        f.write(np.array([len(sessions), steps], dtype=np.int32).tobytes())
        for s in sessions:
            f.write(np.array([s["id"], s["N"], s["P"]], dtype=np.int32).tobytes())
            f.write(np.array([s["arrival"]], dtype=np.float64).tobytes())
            f.write(np.ascontiguousarray(s["graph"], dtype=np.float64).tobytes())
            f.write(np.asarray(s["gammas"], dtype=np.float64).tobytes())
            f.write(np.asarray(s["betas"], dtype=np.float64).tobytes())


def read_records(path):
    raw = open(path, "rb").read()
    recs, off = [], 0
    while off < len(raw):
        sid, step, n, P = np.frombuffer(raw, dtype=np.int32, count=4, offset=off)
        off += 16
        d = np.frombuffer(raw, dtype=np.float64, count=3 + 2 * P, offset=off)
        off += 8 * (3 + 2 * P)
        recs.append({"session": int(sid), "step": int(step), "N": int(n), "P": int(P),
                     "energy": float(d[0]), "latency": float(d[1]), "queue": float(d[2]),
                     "grad_gamma": d[3:3 + P].copy(), "grad_beta": d[3 + P:].copy()})
    return recs


def run_native(mode, sessions, steps, lanes=4, budget=150e9):
    """The stream through serve_replay (no Python in the request loop):
    mode 'served', 'sequential' or 'plain'; returns (records, wall_s, info)."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "stream.bin"), os.path.join(td, "out.bin")
        write_stream(sessions, steps, fin)
        r = subprocess.run([REPLAY, fin, mode, fout, str(lanes), str(budget / 1e9)],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("serve_replay %s failed: %s" % (mode, r.stderr[-1000:]))
        info = json.loads(r.stdout.strip().splitlines()[-1])
        recs = read_records(fout)
    return recs, info["wall_s"], info


def pct(xs, q):
    return float(np.percentile(np.asarray(xs), q)) * 1000.0 if len(xs) else None


def compare(served, seq):
    key = lambda r: (r["session"], r["step"])
    a = {key(r): r for r in served}
    bad = 0
    for r in seq:
        s = a.get(key(r))
        if (s is None or s["energy"] != r["energy"]
                or not np.array_equal(s["grad_gamma"], r["grad_gamma"])
                or not np.array_equal(s["grad_beta"], r["grad_beta"])):
            bad += 1
    return bad


def summarize(served, wall_s, seq=None, wall_q=None, stats=None, plain=None, wall_p=None):
    out = {"requests": len(served), "evals_per_s": len(served) / wall_s, "wall_s": wall_s,
           "latency_ms_p50": pct([r["latency"] for r in served], 50),
           "latency_ms_p99": pct([r["latency"] for r in served], 99),
           "queue_ms_p50": pct([r["queue"] for r in served], 50), "buckets": {}}
    if stats:
        out["server"] = stats
    if seq is not None:
        out["sequential_evals_per_s"] = len(seq) / wall_q
        out["sequential_wall_s"] = wall_q
        out["speedup_vs_sequential"] = out["evals_per_s"] / out["sequential_evals_per_s"]
        out["mismatches_vs_sequential"] = compare(served, seq)
    if plain is not None:
        out["plain_evals_per_s"] = len(plain) / wall_p
        out["plain_wall_s"] = wall_p
        out["speedup_vs_plain"] = out["evals_per_s"] / out["plain_evals_per_s"]
        out["mismatches_vs_plain"] = compare(served, plain)
    for lo, hi, name in BUCKETS:
        sr = [r for r in served if lo <= r["N"] <= hi]
        if not sr:
            continue
        b = {"requests": len(sr), "latency_ms_p50": pct([r["latency"] for r in sr], 50),
             "latency_ms_p99": pct([r["latency"] for r in sr], 99)}
        if seq is not None:
            sq = [r for r in seq if lo <= r["N"] <= hi]
            b["sequential_ms_per_eval"] = 1000.0 * float(np.mean([r["latency"] for r in sq]))
            b["sequential_share_of_time"] = float(sum(r["latency"] for r in sq)) / wall_q
        out["buckets"][name] = b
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--steps", type=int, default=20, help="evaluations per session")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--n-min", type=int, default=10)
    ap.add_argument("--n-max", type=int, default=28)
    ap.add_argument("--p-max", type=int, default=8)
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--gap-ms", type=float, default=1.0, help="mean session inter-arrival")
    ap.add_argument("--no-sequential", action="store_true")
    ap.add_argument("--python-client", action="store_true",
                    help="drive the stream from this Python loop instead of serve_replay")
    a = ap.parse_args(argv)
    sessions, steps = make_stream(a.requests, a.seed, a.steps, a.n_min, a.n_max, a.p_max,
                                  a.gap_ms)
    seq = wall_q = plain = wall_p = None
    if a.python_client:
        import forqaoa as fq
        served, wall, stats = run_served(fq, sessions, steps, 0, a.lanes, a.budget_gb * 1e9)
        if not a.no_sequential:
            seq, wall_q = run_sequential(fq, sessions, steps)
            plain, wall_p = run_sequential(fq, sessions, steps, reuse=False)
    else:
        served, wall, stats = run_native("served", sessions, steps, a.lanes, a.budget_gb * 1e9)
        if not a.no_sequential:
            seq, wall_q, _ = run_native("sequential", sessions, steps)
            plain, wall_p, _ = run_native("plain", sessions, steps)
    out = summarize(served, wall, seq, wall_q, stats, plain, wall_p)
    out["stream"] = {"sessions": len(sessions), "steps": steps, "n": [a.n_min, a.n_max],
                     "p": [1, a.p_max], "graph": "G(N,0.5), integer weights 1..10",
                     "arrivals": f"Poisson, mean gap {a.gap_ms} ms", "seed": a.seed,
                     "lanes": a.lanes, "budget_gb": a.budget_gb}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
