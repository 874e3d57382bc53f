"""CPU tests of the C ABI library: it loads, exports every declared entry
point, and its host-only functions agree with the oracle.  No kernel is
launched here."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, PKG, complete_int, gnp_fp

HEADER = os.path.join(ROOT, "include", "forqaoa.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fq_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_abi():
    names = declared_functions()
    for n in ("fq_ctx_create", "fq_cost_phase", "fq_rx_chunk", "fq_swap_blocks",
              "fq_qaoa_forward", "fq_expectation", "fq_relabel_graph"):
        assert n in names


def test_library_exports_every_declared_symbol(fq):
    lib = fq.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # The Python front-end binds exactly what the header declares.
    assert sorted(fq.SIGNATURES) == declared_functions()


def declared_arity():
    """{name: number of parameters} of every fq_* declaration."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(fq_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_python_bindings_match_declared_arity(fq):
    arity = declared_arity()
    assert sorted(arity) == declared_functions()
    wrong = {n: (len(fq.SIGNATURES[n][1]), k) for n, k in arity.items()
             if len(fq.SIGNATURES[n][1]) != k}
    assert not wrong, wrong


REFAPI_SYMBOLS = [
    "_Z11createStateiiii", "_Z12destroyStateRK5State", "_Z20stateCpyDeviceToHostRK5State",
    "_Z20stateCpyHostToDeviceRK5State", "_Z20stateInitDeviceStateRK5State",
    "_Z10ncclWarnupR5State", "_Z7prepareR5Statei", "_Z11init2DGraphRK5State",
    "_Z16addEdgeTo2DGraphRK5StatePdiid", "_Z11free2DGraphPd", "_Z11init1DGraphRK5State",
    "_Z16addEdgeTo1DGraphRK5StatePyii", "_Z11free1DGraphPy", "_Z5initHRK5State",
    "_Z27rotationCompressionWeightedR5StatedPKdb",
    "_Z29rotationCompressionUnweightedRK5StatedPyb",
    "_Z12multiRotateXR5StateRSt6vectorIiSaIiEEid", "_Z7rotateXRK5Stateid",
    "_Z15swap_gate_contiRK5Stateiii", "_Z9swap_gateRK5Stateii",
    "_Z24mapping_after_swap_contiRK5StatePdiii", "_Z24mapping_after_swap_contiRK5StatePyiii",
]


def test_reference_cpp_api_exported(fq):
    lib = fq.lib()
    missing = [s for s in REFAPI_SYMBOLS if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings(fq):
    lib = fq.lib()
    assert lib.fq_status_string(0) == b"ok"
    assert lib.fq_status_string(fq.ERR_INVALID) == b"invalid argument"
    assert lib.fq_status_string(99) == b"unknown status"
    assert lib.fq_version() >= 100


def test_init_amp_matches_reference_formula(fq, oracle):
    for n in range(1, 34):
        assert fq.init_amp(n) == oracle.init_amp(n) == pow(1 / np.sqrt(2), n)


@pytest.mark.parametrize("N,out,inn,k", [(8, 0, 3, 3), (10, 1, 6, 4), (12, 0, 10, 2),
                                         (7, 2, 4, 1), (13, 0, 6, 6)])
def test_relabel_graph_matches_oracle(fq, oracle, N, out, inn, k):
    rng = np.random.default_rng(N + k)
    W = complete_int(N, rng)
    assert np.array_equal(fq.relabel_graph(W, out, inn, k),
                          oracle.mapping_after_swap_conti(W, out, inn, k))


def test_relabel_graph_rejects_overlap(fq):
    W = np.zeros((8, 8))
    with pytest.raises(fq.FQError) as e:
        fq.relabel_graph(W, 0, 2, 3)
    assert e.value.status == fq.ERR_INVALID


@pytest.mark.parametrize("N,C,P", [(10, 3, 3), (12, 5, 4), (30, 12, 5), (32, 13, 3),
                                   (11, 11, 1), (26, 13, 10)])
def test_reference_label_map_matches_oracle(fq, oracle, N, C, P):
    lab = fq.reference_label_map(N, C, P)
    if N <= 12:
        rng = np.random.default_rng(1)
        W = gnp_fp(N, rng)
        _, _, lab_o = oracle.weighted_run(W, C, np.zeros(P), np.zeros(P))
        assert np.array_equal(lab, lab_o)
    assert sorted(lab.tolist()) == list(range(N))


def test_weighted_cli_usage():
    exe = os.path.join(PKG, "weighted")
    assert os.path.exists(exe)
    r = subprocess.run([exe, "1", "2"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
