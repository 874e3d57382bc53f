"""CPU tests of validate_dump.py (the check of a `weighted --dump` file):
its independent dense simulation agrees with the oracle, a dump written in
the reference's physical order with its label-map sidecar passes, and a
changed amplitude or a wrong label map fails."""
import math

import numpy as np
import pytest

import validate_dump as vd
from conftest import complete_int


def physical_dump(psi_logical, labels):
    """Inverse of vd.to_logical: physical bit b holds logical qubit labels[b]."""
    N = len(labels)
    y = np.arange(1 << N)
    x = np.zeros_like(y)
    for b, q in enumerate(labels):
        x |= ((y >> b) & 1) << q
    return psi_logical[x]


@pytest.mark.parametrize("N,P", [(6, 1), (9, 3)])
def test_expected_state_matches_oracle(oracle, N, P):
    rng = np.random.default_rng(N)
    W = complete_int(N, rng)
    g, b = rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)
    got = vd.expected_state(N, W, g, b)
    want = oracle.qaoa_logical(W, g, b)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_dump_with_labels_passes_and_corruption_fails(fq, oracle, tmp_path):
    """Integer weights: unlike the unit complete graph, whose state does not
    change under a relabelling of the qubits, a wrong label map shows."""
    N, P, C = 10, 2, 4
    rng = np.random.default_rng(3)
    W = complete_int(N, rng)
    g, b = rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)
    labels = list(fq.reference_label_map(N, C, P))
    assert labels != sorted(labels)
    dump = physical_dump(oracle.qaoa_logical(W, g, b), labels)
    f = tmp_path / "s.bin"
    gf = tmp_path / "w.txt"
    np.savetxt(gf, W)
    args = [str(f), str(N), str(P), "--graph", str(gf), "--gammas", ",".join(map(repr, g.tolist())),
            "--betas", ",".join(map(repr, b.tolist()))]
    dump.tofile(f)
    (tmp_path / "s.bin.labels").write_text(" ".join(map(str, labels)) + "\n")
    assert vd.main(args + ["--tol", "1e-12"]) == 0
    bad = dump.copy()
    bad[17] += 1e-6
    bad.tofile(f)
    assert vd.main(args) == 1
    dump.tofile(f)
    (tmp_path / "s.bin.labels").write_text(" ".join(map(str, range(N))) + "\n")
    assert vd.main(args) == 1


def test_unit_complete_graph_is_label_blind(oracle, tmp_path):
    """The CLI's default circuit (unit K_N, pi/4) is symmetric under qubit
    relabelling: its dump passes with any label map."""
    N, P = 8, 2
    W = np.triu(np.ones((N, N)), 1)
    g = b = np.full(P, math.pi / 4)
    psi = oracle.qaoa_logical(W, g, b)
    f = tmp_path / "u.bin"
    physical_dump(psi, [3, 1, 0, 2, 7, 6, 5, 4]).tofile(f)
    assert vd.main([str(f), str(N), str(P), "--tol", "1e-12"]) == 0
