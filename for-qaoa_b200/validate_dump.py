#!/usr/bin/env python3
"""Check a state dumped by `weighted ... --dump FILE` against an independent
dense simulation of the same circuit.

The dump is the raw complex128 state (2^N amplitudes, little-endian
{re, im}) in the reference's physical qubit order; FILE.labels gives the
logical qubit held at each physical bit position.  The expected state is
computed here gate by gate from the textbook definitions, with nothing
shared with the library: H on every qubit, RZZ(gamma) = exp(-i gamma/2 Z Z)
on every weighted edge (a phase of exp(+i gamma S/2) with S = sum over edges
of +w if cut, -w if not), RX(beta) = exp(-i beta X/2) on every qubit, per
layer.  By default the circuit is the CLI's own (unit-weight complete graph,
gamma = beta = pi/4), or the one in FILE.circuit when the CLI wrote it
(N P, the gammas, the betas, the N x N graph); --graph takes an N x N weight
matrix (upper triangle read, text as numpy.savetxt writes it) and
--gammas/--betas per-layer angles, overriding both.

    weighted 2 14 0 5 14 --weights int --angles random --dump s.bin
    python validate_dump.py s.bin 14 2

Exit status 0 when max |dump - expected| <= --tol (1e-8 by default, the
tolerance of the reference's own validator).  Dense simulation: N <= 26.
The default circuit's state does not change under a relabelling of the
qubits, so only a weighted graph (--graph) tests the label map.
"""
import argparse
import math
import sys

import numpy as np


def expected_state(N, graph, gammas, betas):
    """Logical-order state of the QAOA circuit (little-endian: index bit q is
    qubit q)."""
    z = np.arange(1 << N, dtype=np.int64)
    bits = [(z >> q) & 1 for q in range(N)]
    S = np.zeros(1 << N)
    for i in range(N):
        for j in range(i + 1, N):
            w = graph[i, j]
            if w != 0:
                S += np.where(bits[i] != bits[j], w, -w)
    psi = np.full(1 << N, 2.0 ** (-N / 2), dtype=np.complex128)
    for g, b in zip(gammas, betas):
        psi *= np.exp(0.5j * g * S)
        c, s = math.cos(b / 2), math.sin(b / 2)
        for q in range(N):
            v = psi.reshape(-1, 2, 1 << q)
            a0, a1 = v[:, 0, :].copy(), v[:, 1, :].copy()
            v[:, 0, :] = c * a0 - 1j * s * a1
            v[:, 1, :] = -1j * s * a0 + c * a1
    return psi


def to_logical(dump, labels):
    """Reorder a physical-order state: physical bit b holds logical qubit
    labels[b]."""
    N = len(labels)
    y = np.arange(1 << N, dtype=np.int64)
    x = np.zeros_like(y)
    for b, q in enumerate(labels):
        x |= ((y >> b) & 1) << q
    out = np.empty_like(dump)
    out[x] = dump
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("dump")
    ap.add_argument("N", type=int)
    ap.add_argument("P", type=int)
    ap.add_argument("--labels", help="label map (default: DUMP.labels; none: identity)")
    ap.add_argument("--graph", help="N x N weight matrix (text); default unit complete graph")
    ap.add_argument("--gammas", help="comma-separated per-layer gammas (default pi/4)")
    ap.add_argument("--betas", help="comma-separated per-layer betas (default pi/4)")
    ap.add_argument("--tol", type=float, default=1e-8)
    a = ap.parse_args(argv)
    if not 1 <= a.N <= 26:
        ap.error("N must be in 1..26 for the dense check")
    dump = np.fromfile(a.dump, dtype=np.complex128)
    if dump.size != 1 << a.N:
        print(f"FAIL: {a.dump} holds {dump.size} amplitudes, expected 2^{a.N}")
        return 1
    try:
        labels = [int(t) for t in open(a.labels or a.dump + ".labels").read().split()]
    except OSError:
        if a.labels:
            raise
        labels = list(range(a.N))
    if sorted(labels) != list(range(a.N)):
        print("FAIL: the label map is not a permutation of 0..N-1")
        return 1
    graph = np.triu(np.ones((a.N, a.N)), 1)
    gammas, betas = [math.pi / 4] * a.P, [math.pi / 4] * a.P
    try:
        rows = [ln.split() for ln in open(a.dump + ".circuit").read().splitlines() if ln.strip()]
        if [int(t) for t in rows[0]] != [a.N, a.P]:
            print(f"FAIL: {a.dump}.circuit describes N={rows[0][0]} P={rows[0][1]}")
            return 1
        gammas = [float(t) for t in rows[1]]
        betas = [float(t) for t in rows[2]]
        graph = np.array([[float(t) for t in r] for r in rows[3:3 + a.N]])
    except OSError:
        pass
    if a.graph:
        graph = np.loadtxt(a.graph)
    if a.gammas:
        gammas = [float(t) for t in a.gammas.split(",")]
    if a.betas:
        betas = [float(t) for t in a.betas.split(",")]
    if len(gammas) != a.P or len(betas) != a.P:
        ap.error("need P gammas and P betas")
    want = expected_state(a.N, graph, gammas, betas)
    got = to_logical(dump, labels)
    err = float(np.abs(got - want).max())
    ok = err <= a.tol
    print(f"{'PASS' if ok else 'FAIL'}: max |dump - expected| = {err:.3e} (tol {a.tol:g}), "
          f"N={a.N} P={a.P}, norm {np.linalg.norm(got):.15f}")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
