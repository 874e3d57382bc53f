"""Python front-end of libforqaoa.so (ctypes over the C ABI in
include/forqaoa.h).

Only the C ABI is used: device memory comes from fq_state_alloc, copies go
through fq_state_to_host / fq_state_from_host, and every call checks the
returned status and raises FQError with the library's message.  There is no
fallback: if libforqaoa.so is missing or fails to load, importing this module
raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libforqaoa.so")
# FQ_SMALL_MAX_QUBITS of include/forqaoa.h: energy+gradient instances up to
# this size run wholly in shared memory and need no state buffers.
SMALL_MAX_QUBITS = 15

OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_BUSY = range(7)

# Kernel kinds of fq_ctx_profile (include/forqaoa.h)
KINDS = {"phase_pass": 0, "mixer_pass": 1, "cost": 2, "rx": 3, "swap": 4, "expect": 5,
         "other": 6, "adjoint": 7, "init_pass": 8}

if not os.path.exists(LIB_PATH):
    raise ImportError("libforqaoa.so not built: run `make -C for-qaoa_b200` "
                      "(or __graft_entry__.build())")
_lib = ctypes.CDLL(LIB_PATH)

_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i = ctypes.c_int
_d = ctypes.c_double

# name -> (restype, argtypes), mirroring include/forqaoa.h
SIGNATURES = {
    "fq_status_string": (ctypes.c_char_p, [_i]),
    "fq_last_error": (ctypes.c_char_p, []),
    "fq_version": (_i, []),
    "fq_ctx_create": (_i, [_i, _vp, ctypes.POINTER(_vp)]),
    "fq_ctx_destroy": (_i, [_vp]),
    "fq_ctx_synchronize": (_i, [_vp]),
    "fq_ctx_selftest_wait": (_i, [_vp]),
    "fq_ctx_stream": (_vp, [_vp]),
    "fq_ctx_kernel_launches": (_i, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "fq_ctx_device_info": (_i, [_vp, _ip, _ip]),
    "fq_ctx_set_profiling": (_i, [_vp, _i]),
    "fq_ctx_profile": (_i, [_vp, _i, _dp, ctypes.POINTER(ctypes.c_longlong), _dp]),
    "fq_ctx_profile_reset": (_i, [_vp]),
    "fq_state_alloc": (_i, [_vp, _i, ctypes.POINTER(_vp)]),
    "fq_state_free": (_i, [_vp, _vp]),
    "fq_state_init_basis0": (_i, [_vp, _vp, _i]),
    "fq_state_to_host": (_i, [_vp, _vp, _i, _vp]),
    "fq_state_from_host": (_i, [_vp, _vp, _i, _vp]),
    "fq_init_amp": (_d, [_i]),
    "fq_cost_phase": (_i, [_vp, _vp, _i, _d, _dp, _i, _d]),
    "fq_rx_chunk": (_i, [_vp, _vp, _i, _i, _ip, _i, _d]),
    "fq_rx_targets": (_i, [_vp, _vp, _i, _ip, _i, _d]),
    "fq_swap_blocks": (_i, [_vp, _vp, _i, _i, _i, _i]),
    "fq_relabel_graph": (_i, [_dp, _i, _i, _i, _i]),
    "fq_shard_layer": (_i, [_vp, _vp, _i, _i, _i, _dp, _d, _d, _i]),
    "fq_shard_layer_after_swap": (_i, [_vp, _vp, _i, _i, _i, _dp, _d, _d, _d]),
    "fq_shard_expectation": (_i, [_vp, _vp, _i, _i, _i, _dp, _dp]),
    "fq_qaoa_forward": (_i, [_vp, _vp, _i, _i, _dp, _dp, _dp, _dp]),
    "fq_expectation": (_i, [_vp, _vp, _i, _dp, _dp]),
    "fq_qaoa_energy_grad": (_i, [_vp, _vp, _vp, _i, _i, _dp, _dp, _dp, _dp, _dp, _dp]),
    "fq_cut_diagonal": (_i, [_vp, _vp, _i, _dp]),
    "fq_permute_qubits": (_i, [_vp, _vp, _vp, _i, _ip]),
    "fq_state_diff": (_i, [_vp, _vp, _vp, _i, _dp]),
    "fq_reference_label_map": (_i, [_i, _i, _i, _ip]),
    "fq_expectation_noalloc": (_i, [_vp, _i, _dp, _dp, _vp]),
    "fq_server_create": (_i, [_i, _d, _i, ctypes.POINTER(_vp)]),
    "fq_server_destroy": (_i, [_vp]),
    "fq_server_submit": (_i, [_vp, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "fq_server_poll": (_i, [_vp, ctypes.c_void_p, _i, _ip, _i]),
    "fq_server_close_session": (_i, [_vp, ctypes.c_uint64]),
    "fq_server_stats": (_i, [_vp, ctypes.c_void_p]),
}

SERVE_MAX_LAYERS = 16  # FQ_SERVE_MAX_LAYERS


class _Request(ctypes.Structure):
    _fields_ = [("session", ctypes.c_uint64), ("N", _i), ("P", _i), ("graph_upper", _dp),
                ("gammas", _dp), ("betas", _dp)]


class _Result(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("session", ctypes.c_uint64), ("N", _i),
                ("P", _i), ("status", _i), ("pad", _i), ("energy", _d),
                ("grad_gamma", _d * SERVE_MAX_LAYERS), ("grad_beta", _d * SERVE_MAX_LAYERS),
                ("t_submit", _d), ("t_start", _d), ("t_done", _d)]


class _Counters(ctypes.Structure):
    _fields_ = [("pending", ctypes.c_longlong), ("kernel_launches", ctypes.c_longlong),
                ("batched_requests", ctypes.c_longlong), ("lane_requests", ctypes.c_longlong),
                ("resident_sessions", ctypes.c_longlong), ("resident_bytes", _d)]
for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class FQError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = _lib.fq_last_error().decode(errors="replace")
        name = _lib.fq_status_string(status).decode()
        super().__init__("%s: %s (%d): %s" % (where, name, status, msg))


def _check(status, where):
    if status != OK:
        raise FQError(status, where)


def lib():
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


def init_amp(n):
    return _lib.fq_init_amp(n)


def relabel_graph(graph, swap_out, swap_in, k):
    """mapping_after_swap_conti (src/swap.cu:27-50) on a copy of graph."""
    g = _f64(graph).copy()
    _check(_lib.fq_relabel_graph(_dptr(g), g.shape[0], swap_out, swap_in, k),
           "fq_relabel_graph")
    return g


def reference_label_map(n, C, P):
    lab = np.zeros(n, dtype=np.int32)
    _check(_lib.fq_reference_label_map(n, C, P, _iptr(lab)), "fq_reference_label_map")
    return lab


class DeviceState:
    """2^n complex128 amplitudes in device memory owned by a Context."""

    def __init__(self, ctx, n):
        self.ctx = ctx
        self.n = n
        p = _vp()
        _check(_lib.fq_state_alloc(ctx.handle, n, ctypes.byref(p)), "fq_state_alloc")
        self.ptr = p

    @property
    def nbytes(self):
        return 16 << self.n

    def free(self):
        if self.ptr:
            _check(_lib.fq_state_free(self.ctx.handle, self.ptr), "fq_state_free")
            self.ptr = None

    def to_host(self, out=None):
        if out is None:
            out = np.empty(1 << self.n, dtype=np.complex128)
        assert out.dtype == np.complex128 and out.flags.c_contiguous and out.size == 1 << self.n
        _check(_lib.fq_state_to_host(self.ctx.handle, self.ptr, self.n, out.ctypes.data),
               "fq_state_to_host")
        return out

    def from_host(self, arr):
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        assert a.size == 1 << self.n
        _check(_lib.fq_state_from_host(self.ctx.handle, self.ptr, self.n, a.ctypes.data),
               "fq_state_from_host")
        return self

    def init_basis0(self):
        _check(_lib.fq_state_init_basis0(self.ctx.handle, self.ptr, self.n),
               "fq_state_init_basis0")
        return self


class Context:
    """fq_ctx: one device, one stream, the kernels' scratch."""

    def __init__(self, device=0, stream=None):
        h = _vp()
        _check(_lib.fq_ctx_create(device, stream, ctypes.byref(h)), "fq_ctx_create")
        self.handle = h

    def close(self):
        if self.handle:
            _check(_lib.fq_ctx_destroy(self.handle), "fq_ctx_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def synchronize(self):
        _check(_lib.fq_ctx_synchronize(self.handle), "fq_ctx_synchronize")

    @property
    def stream(self):
        return _lib.fq_ctx_stream(self.handle)

    def launches(self):
        c = ctypes.c_longlong()
        _check(_lib.fq_ctx_kernel_launches(self.handle, ctypes.byref(c)),
               "fq_ctx_kernel_launches")
        return c.value

    def set_profiling(self, on=True):
        _check(_lib.fq_ctx_set_profiling(self.handle, int(bool(on))), "fq_ctx_set_profiling")

    def profile_reset(self):
        _check(_lib.fq_ctx_profile_reset(self.handle), "fq_ctx_profile_reset")

    def profile(self):
        """{kind: (device ms, launches, algorithmic bytes)} since the last reset."""
        out = {}
        for name, k in KINDS.items():
            ms, n, b = _d(), ctypes.c_longlong(), _d()
            _check(_lib.fq_ctx_profile(self.handle, k, ctypes.byref(ms), ctypes.byref(n),
                                       ctypes.byref(b)), "fq_ctx_profile")
            if n.value:
                out[name] = (ms.value, n.value, b.value)
        return out

    def device_info(self):
        a, b = _i(), _i()
        _check(_lib.fq_ctx_device_info(self.handle, ctypes.byref(a), ctypes.byref(b)),
               "fq_ctx_device_info")
        return a.value, b.value

    def state(self, n):
        return DeviceState(self, n)

    # -- reference-path kernels -------------------------------------------
    def cost_phase(self, st, angle, graph, is_first, amp0=None):
        g = _f64(graph)
        amp0 = init_amp(st.n) if amp0 is None else amp0
        _check(_lib.fq_cost_phase(self.handle, st.ptr, st.n, angle, _dptr(g),
                                  int(bool(is_first)), amp0), "fq_cost_phase")

    def rx_chunk(self, st, chunk_qubits, targets, angle):
        t = np.ascontiguousarray(targets, dtype=np.int32)
        _check(_lib.fq_rx_chunk(self.handle, st.ptr, st.n, chunk_qubits, _iptr(t), len(t),
                                angle), "fq_rx_chunk")

    def rx_targets(self, st, targets, angle):
        t = np.ascontiguousarray(targets, dtype=np.int32)
        _check(_lib.fq_rx_targets(self.handle, st.ptr, st.n, _iptr(t), len(t), angle),
               "fq_rx_targets")

    # -- shards of a state split over 2^D devices (raw device pointers) ------
    def shard_layer(self, ptr, N, D, rank, graph, gamma, beta, first_layer):
        """Cost phase + RX(beta) on the local qubits of shard `rank`
        (fq_shard_layer); graph in the shards' current physical order."""
        g = _f64(graph)
        _check(_lib.fq_shard_layer(self.handle, _vp(ptr), N, D, rank, _dptr(g), gamma, beta,
                                   int(bool(first_layer))), "fq_shard_layer")

    def shard_layer_after_swap(self, ptr, N, D, rank, graph, gamma, beta, beta_prev):
        """RX(beta_prev) on the qubits the last all-to-all swapped in
        (local qubits N-2D..N-D-1), then a later layer on shard `rank`
        (fq_shard_layer_after_swap: the rotation inside the layer's first
        pass where its tile allows)."""
        g = _f64(graph)
        _check(_lib.fq_shard_layer_after_swap(self.handle, _vp(ptr), N, D, rank, _dptr(g), gamma,
                                              beta, beta_prev), "fq_shard_layer_after_swap")

    def shard_expectation(self, ptr, N, D, rank, graph):
        """This shard's part of <C> (fq_shard_expectation)."""
        g = _f64(graph)
        e = np.zeros(1)
        _check(_lib.fq_shard_expectation(self.handle, _vp(ptr), N, D, rank, _dptr(g), _dptr(e)),
               "fq_shard_expectation")
        return float(e[0])

    def rx_targets_ptr(self, ptr, n, targets, angle):
        """fq_rx_targets on the 2^n amplitudes at device address ptr."""
        t = np.ascontiguousarray(targets, dtype=np.int32)
        _check(_lib.fq_rx_targets(self.handle, _vp(ptr), n, _iptr(t), len(t), angle),
               "fq_rx_targets")

    def swap_blocks(self, st, swap_out, swap_in, k):
        _check(_lib.fq_swap_blocks(self.handle, st.ptr, st.n, swap_out, swap_in, k),
               "fq_swap_blocks")

    # -- fused engine --------------------------------------------------------
    def qaoa_forward(self, st, graph, gammas, betas, energy=True):
        g = _f64(graph)
        ga, be = _f64(gammas), _f64(betas)
        assert len(ga) == len(be)
        e = np.zeros(1)
        _check(_lib.fq_qaoa_forward(self.handle, st.ptr, st.n, len(ga), _dptr(g), _dptr(ga),
                                    _dptr(be), _dptr(e) if energy else None),
               "fq_qaoa_forward")
        return float(e[0]) if energy else None

    def energy_grad(self, n, graph, gammas, betas, sv=None, costate=None):
        """(<C>, dE/dgamma[P], dE/dbeta[P]) by the adjoint method.  sv and
        costate are DeviceState workspaces of n qubits (allocated here when
        omitted and n > SMALL_MAX_QUBITS)."""
        g = _f64(graph)
        ga, be = _f64(gammas), _f64(betas)
        P = len(ga)
        e, gg, gb = np.zeros(1), np.zeros(P), np.zeros(P)
        own = []
        if n > SMALL_MAX_QUBITS:
            if sv is None:
                sv = DeviceState(self, n)
                own.append(sv)
            if costate is None:
                costate = DeviceState(self, n)
                own.append(costate)
        try:
            _check(_lib.fq_qaoa_energy_grad(self.handle, sv.ptr if sv else None,
                                            costate.ptr if costate else None, n, P, _dptr(g),
                                            _dptr(ga), _dptr(be), _dptr(e), _dptr(gg),
                                            _dptr(gb)), "fq_qaoa_energy_grad")
        finally:
            for s in own:
                s.free()
        return float(e[0]), gg, gb

    def expectation(self, st, graph):
        g = _f64(graph)
        e = np.zeros(1)
        _check(_lib.fq_expectation(self.handle, st.ptr, st.n, _dptr(g), _dptr(e)),
               "fq_expectation")
        return float(e[0])

    def cut_diagonal(self, n, graph):
        """C(z) for every z (float64), computed on the device."""
        g = _f64(graph)
        tmp = DeviceState(self, n - 1) if n > 1 else DeviceState(self, 1)
        try:
            _check(_lib.fq_cut_diagonal(self.handle, tmp.ptr, n, _dptr(g)), "fq_cut_diagonal")
            raw = tmp.to_host()
        finally:
            tmp.free()
        return raw.view(np.float64)[: 1 << n].copy()

    def permute_qubits(self, src, dst, perm):
        p = np.ascontiguousarray(perm, dtype=np.int32)
        _check(_lib.fq_permute_qubits(self.handle, src.ptr, dst.ptr, src.n, _iptr(p)),
               "fq_permute_qubits")

    def state_diff(self, a, b):
        """{max_abs_diff, max_abs_b, l2_diff, l2_b} of two device states."""
        out = np.zeros(4)
        _check(_lib.fq_state_diff(self.handle, a.ptr, b.ptr, a.n, _dptr(out)), "fq_state_diff")
        return dict(zip(("max_abs_diff", "max_abs_b", "l2_diff", "l2_b"), out.tolist()))

    def reference_schedule(self, st, graph, C, gammas, betas):
        """The reference's layer loop (src/Weighted.cpp:97-138) through the
        per-launcher entry points; returns the relabelled graph.  The state is
        left in the reference's physical order."""
        g = _f64(graph).copy()
        n = st.n
        sizes = [min(C, n - i) for i in range(0, n, C)]
        sub0 = list(range(min(C, n)))
        amp0 = init_amp(n)
        for p, (ga, be) in enumerate(zip(gammas, betas)):
            self.cost_phase(st, ga, g, p == 0, amp0)
            swap_in = 0
            for i, sz in enumerate(sizes):
                self.rx_chunk(st, min(13, n), sub0[:sz], be)
                if i < len(sizes) - 1:
                    swap_in += sz
                    self.swap_blocks(st, 0, swap_in, sizes[i + 1])
                    _check(_lib.fq_relabel_graph(_dptr(g), n, 0, swap_in, sizes[i + 1]),
                           "fq_relabel_graph")
        return g


class ServeResult:
    """One finished request of a Server."""
    __slots__ = ("ticket", "session", "N", "P", "status", "energy", "grad_gamma", "grad_beta",
                 "t_submit", "t_start", "t_done")

    def __init__(self, r):
        self.ticket, self.session = int(r.ticket), int(r.session)
        self.N, self.P, self.status = r.N, r.P, r.status
        self.energy = r.energy
        self.grad_gamma = np.array(r.grad_gamma[:r.P])
        self.grad_beta = np.array(r.grad_beta[:r.P])
        self.t_submit, self.t_start, self.t_done = r.t_submit, r.t_start, r.t_done

    @property
    def latency(self):
        return self.t_done - self.t_submit


class Server:
    """Continuous batching of energy+gradient requests on one device
    (fq_server_* in include/forqaoa.h).  submit() returns a ticket; poll()
    returns finished ServeResults in completion order."""

    def __init__(self, device=0, hbm_budget_bytes=150e9, lanes=4):
        h = _vp()
        _check(_lib.fq_server_create(device, float(hbm_budget_bytes), lanes, ctypes.byref(h)),
               "fq_server_create")
        self.handle = h
        self._stash = []  # results polled by wait() for other tickets

    def close(self):
        if self.handle:
            _check(_lib.fq_server_destroy(self.handle), "fq_server_destroy")
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, session, graph, gammas, betas):
        g, ga, be = _f64(graph), _f64(gammas), _f64(betas)
        assert ga.shape == be.shape and g.shape[0] == g.shape[1]
        q = _Request(session, g.shape[0], len(ga), _dptr(g), _dptr(ga), _dptr(be))
        t = ctypes.c_uint64()
        _check(_lib.fq_server_submit(self.handle, ctypes.byref(q), ctypes.byref(t)),
               "fq_server_submit")
        return int(t.value)

    def _poll_lib(self, max_results, wait_ms):
        buf = (_Result * max_results)()
        n = _i()
        _check(_lib.fq_server_poll(self.handle, buf, max_results, ctypes.byref(n), wait_ms),
               "fq_server_poll")
        return [ServeResult(buf[i]) for i in range(n.value)]

    def poll(self, max_results=1024, wait_ms=0):
        if self._stash:
            out, self._stash = self._stash[:max_results], self._stash[max_results:]
            return out
        return self._poll_lib(max_results, wait_ms)

    def wait(self, tickets, timeout_s=600.0):
        """Polls until every ticket in `tickets` is done; returns {ticket: result}.
        Results of other tickets stay queued for poll()."""
        import time
        want, got, keep = set(tickets), {}, []
        for r in self._stash:
            if r.ticket in want:
                got[r.ticket] = r
            else:
                keep.append(r)
        self._stash = keep
        t_end = time.monotonic() + timeout_s
        while want - got.keys():
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - got.keys())} requests not done")
            for r in self._poll_lib(1024, 50):
                if r.ticket in want:
                    got[r.ticket] = r
                else:
                    self._stash.append(r)
        return got

    def close_session(self, session):
        _check(_lib.fq_server_close_session(self.handle, session), "fq_server_close_session")

    def stats(self):
        c = _Counters()
        _check(_lib.fq_server_stats(self.handle, ctypes.byref(c)), "fq_server_stats")
        return {k: getattr(c, k) for k, _ in _Counters._fields_}
