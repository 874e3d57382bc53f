"""ctypes front-end of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by the test suite, the smoke check and the
CPU-baseline leg of the bench, as the checker of the CUDA library.  The
product library never imports it.  Every function here calls the C
restatement in oracle.c, which cites the FOR-QAOA source lines it follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_init_amp.restype = ctypes.c_double
        L.orc_init_amp.argtypes = [ctypes.c_int]
        L.orc_upper_tri_to_1d.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_cost_phase.argtypes = [_dp, ctypes.c_int, ctypes.c_double, _dp,
                                     ctypes.c_int, ctypes.c_double]
        L.orc_multi_rotate_x.argtypes = [_dp, ctypes.c_int, _ip, ctypes.c_int,
                                         ctypes.c_double]
        L.orc_swap_gate_conti.argtypes = [_dp] + [ctypes.c_int] * 4
        L.orc_mapping_after_swap_conti.argtypes = [_dp] + [ctypes.c_int] * 4
        L.orc_weighted_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _dp, _dp, _dp, _dp, _dp, _ip]
        L.orc_qaoa_logical.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp,
                                       _dp, _dp]
        L.orc_cost_diag_S.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_cut_values.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_expectation.restype = ctypes.c_double
        L.orc_expectation.argtypes = [_dp, ctypes.c_int, _dp]
        L.orc_energy_grad.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp,
                                      _dp, _dp, _dp]
        L.orc_permute_qubits.argtypes = [_dp, _dp, ctypes.c_int, _ip]
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_state_fill.argtypes = [_dp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.orc_layer_chunk.argtypes = [_dp, ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def num_threads():
    return lib().orc_num_threads()


def init_amp(n):
    return lib().orc_init_amp(n)


def upper_tri_to_1d(graph):
    g = _f64(graph)
    n = g.shape[0]
    out = np.zeros(max(n * (n - 1) // 2, 1))
    lib().orc_upper_tri_to_1d(n, _d(g), _d(out))
    return out[: n * (n - 1) // 2]


def cost_phase(sv, n, angle, graph1d, is_first, amp0=None):
    """In place, like rotationCompressionWeighted (rzz.cu:173-206)."""
    assert sv.dtype == np.complex128 and sv.flags.c_contiguous
    g = _f64(graph1d) if len(graph1d) else np.zeros(1)
    amp0 = init_amp(n) if amp0 is None else amp0
    lib().orc_cost_phase(sv.view(np.float64).ctypes.data_as(_dp), n, angle,
                         _d(g), int(bool(is_first)), amp0)
    return sv


def multi_rotate_x(sv, n, targets, angle):
    t = np.ascontiguousarray(targets, dtype=np.int32)
    lib().orc_multi_rotate_x(sv.view(np.float64).ctypes.data_as(_dp), n, _i(t),
                             len(t), angle)
    return sv


def swap_gate_conti(sv, n, swap_out, swap_in, k):
    lib().orc_swap_gate_conti(sv.view(np.float64).ctypes.data_as(_dp), n,
                              swap_out, swap_in, k)
    return sv


def mapping_after_swap_conti(graph, swap_out, swap_in, k):
    g = _f64(graph).copy()
    lib().orc_mapping_after_swap_conti(_d(g), g.shape[0], swap_out, swap_in, k)
    return g


def weighted_run(graph, C, gammas, betas):
    """The reference schedule (Weighted.cpp:97-138): returns (state in the
    reference's physical order, final relabelled graph, label map)."""
    g = _f64(graph)
    n = g.shape[0]
    P = len(gammas)
    sv = np.zeros(1 << n, dtype=np.complex128)
    gf = np.zeros_like(g)
    lab = np.zeros(n, dtype=np.int32)
    lib().orc_weighted_run(n, C, P, _d(g), _d(_f64(gammas)), _d(_f64(betas)),
                           sv.view(np.float64).ctypes.data_as(_dp), _d(gf), _i(lab))
    return sv, gf, lab


def qaoa_logical(graph, gammas, betas):
    g = _f64(graph)
    n = g.shape[0]
    sv = np.zeros(1 << n, dtype=np.complex128)
    lib().orc_qaoa_logical(n, len(gammas), _d(g), _d(_f64(gammas)),
                           _d(_f64(betas)), sv.view(np.float64).ctypes.data_as(_dp))
    return sv


def cost_diag_S(graph):
    g = _f64(graph)
    n = g.shape[0]
    S = np.zeros(1 << n)
    lib().orc_cost_diag_S(n, _d(g), _d(S))
    return S


def cut_values(graph):
    g = _f64(graph)
    n = g.shape[0]
    Cz = np.zeros(1 << n)
    lib().orc_cut_values(n, _d(g), _d(Cz))
    return Cz


def expectation(sv, graph):
    g = _f64(graph)
    sv = _c128(sv)
    return lib().orc_expectation(sv.view(np.float64).ctypes.data_as(_dp),
                                 g.shape[0], _d(g))


def energy_grad(graph, gammas, betas):
    g = _f64(graph)
    n = g.shape[0]
    P = len(gammas)
    e = np.zeros(1)
    gg = np.zeros(P)
    gb = np.zeros(P)
    lib().orc_energy_grad(n, P, _d(g), _d(_f64(gammas)), _d(_f64(betas)), _d(e),
                          _d(gg), _d(gb))
    return float(e[0]), gg, gb


def permute_qubits(sv, perm):
    sv = _c128(sv)
    n = len(perm)
    out = np.zeros_like(sv)
    p = np.ascontiguousarray(perm, dtype=np.int32)
    lib().orc_permute_qubits(sv.view(np.float64).ctypes.data_as(_dp),
                             out.view(np.float64).ctypes.data_as(_dp), n, _i(p))
    return out


def to_logical(sv_phys, label_map):
    """Physical-order state (reference layout) -> logical order."""
    return permute_qubits(sv_phys, label_map)


class CpuLayer:
    """One QAOA layer of the reference algorithm on a full 2^N host state,
    timed in equal parts (orc_layer_chunk): the CPU baseline of the bench.
    The state is allocated and first-touched once (16 GiB at N = 30)."""

    def __init__(self, graph, nchunks=32):
        g = _f64(graph)
        self.n = g.shape[0]
        g1d = upper_tri_to_1d(g)
        self.g1d = g1d if len(g1d) else np.zeros(1)
        self.nchunks = nchunks
        self.sv = np.empty(1 << self.n, dtype=np.complex128)
        lib().orc_state_fill(self._p(), self.n, 2.0 ** (-self.n / 2), 0.0)

    def _p(self):
        return self.sv.view(np.float64).ctypes.data_as(_dp)

    def chunk(self, k, gamma, beta):
        """Part k of a layer (not the first: the cost phase reads and
        multiplies); returns its seconds."""
        tc, tr = np.zeros(1), np.zeros(1)
        lib().orc_layer_chunk(self._p(), self.n, _d(self.g1d), gamma, beta, 0,
                              k % self.nchunks, self.nchunks, _d(tc), _d(tr))
        return float(tc[0] + tr[0])

    def full_layer(self, gamma, beta):
        """One whole layer in the reference's order (the read-multiply cost
        phase of rzz.cu:152-154 on every amplitude, then RX on qubits 0..N-1,
        rx.cu:32-53); returns its seconds."""
        import time
        t0 = time.perf_counter()
        lib().orc_cost_phase(self._p(), self.n, gamma, _d(self.g1d), 0, init_amp(self.n))
        tg = np.arange(self.n, dtype=np.int32)
        lib().orc_multi_rotate_x(self._p(), self.n, _i(tg), self.n, beta)
        return time.perf_counter() - t0

    def free(self):
        self.sv = None
