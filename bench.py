#!/usr/bin/env python3
"""Headline benchmark: QAOA Max-Cut, N=30 qubits, p=5 layers, on B200.

Workload (benchmark config 2): complete graph K_30 (435 edges) with seeded
integer weights in 1..10, gamma_k ~ U[0,pi), beta_k ~ U[0,pi/2), complex128
state of 2^30 amplitudes (16 GiB, far larger than the 126 MB L2, so no L2
flush is needed between steps).  One step = the whole p=5 circuit from
|+>^30 through the fused engine (fq_qaoa_forward).  value = layers/s over all
ranks; every rank runs its own replica (the path has no exchange step on one
device, so there is no data-path collective).

Also reported on the same JSON line:
  e2e          the same circuit through the public C ABI with host inputs:
               the graph is uploaded from pinned host memory every step and
               <C> is read back to the host every step;
  roofline     the dominant kernel kind (the one with the largest share of
               device time: at N=30 the fused passes and the mixer passes
               take nearly equal shares, so either can lead): algorithmic
               bytes per launch / average launch time (CUDA events on the
               library's stream), against the measured HBM copy bandwidth;
               per_kind gives every kind, per_layer the same over every pass
               of a layer;
  cpu_baseline the oracle (plain FP64 OpenMP restatement of the reference's
               algorithm) timed on the host cores on one whole N=30 layer of
               a full 16 GiB host state, beside the estimate from timed
               equal parts of a layer (scale_check = full / estimate);
  reference_schedule  the reference's own per-layer schedule (cost sweep, RX
               chunks of C=12, block swaps) through this library's per-kernel
               entry points, with per-kernel HBM GB/s;
  gradient     <C> and its 2p derivatives (adjoint) for K_26, p=10;
  config3      the N=32 p=3 circuit on a 3-regular graph with FP64 weights
               (64 GiB state): layers/s and per-layer HBM fraction;
  serving      a sample of the served request stream (sessions of 20
               energy+gradient steps, N in 10..28, p in 1..8) through the
               server against the same evaluations as sequential calls, plus
               the same stream per size class (by_size);
  clocks       SM clock / throttle reasons sampled during the timed region.

`--impl reference` times the reference algorithm on the host cores (the
reference ships no CPU implementation; the oracle port stands in) on the same
workload and metric: each step is one of 32 equal parts of a layer on the
full-size state (value = parts' share of a layer / their time), and one
whole layer is timed once at the end as a check of the parts.
"""
import argparse
import json
import os
import re
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "for-qaoa_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
for _p in (PKG, ORACLE_DIR):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "N=30 p=5 layers/s & HBM GB/s vs roofline; served energy+grad evals/s, p50/p99"
UNIT = "layers/s"
# Reference (H100, its own ncu report of `weighted 5 30 0 11 24`): 615.7 ms of
# kernel time per layer.
BASELINE_LAYERS_PER_S = 1.62
FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", "--qubits", dest="n", type=int, default=30)
    ap.add_argument("--p", type=int, default=5)
    ap.add_argument("--chunk", type=int, default=12)
    ap.add_argument("--seed", type=int, default=30)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-ref-schedule", action="store_true")
    ap.add_argument("--cpu-parts", type=int, default=8,
                    help="parts (of 32 per layer) timed for the CPU estimate")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's own CUDA build")
    ap.add_argument("--no-cpu-full", action="store_true",
                    help="skip the whole-layer CPU measurement (parts only)")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests of the served-stream leg (0: skip it)")
    ap.add_argument("--serve-sustained-requests", type=int, default=1200,
                    help="requests of the served leg's sustainable-rate latency run")
    ap.add_argument("--serve-lanes", type=int, default=4)
    ap.add_argument("--no-grad", action="store_true", help="skip the adjoint-gradient leg")
    ap.add_argument("--no-config3", action="store_true",
                    help="skip the N=32 p=3 (3-regular, FP64 weights) circuit leg")
    return ap.parse_args(argv)


def workload(n, P, seed):
    rng = np.random.default_rng(seed)
    graphs = [np.triu(rng.integers(1, 11, size=(n, n)).astype(np.float64), 1) for _ in range(2)]
    gammas = rng.uniform(0, np.pi, P)
    betas = rng.uniform(0, np.pi / 2, P)
    return graphs, gammas, betas


def workload_config(args):
    return {
        "workload": "QAOA Max-Cut N=%d p=%d, K_%d integer weights 1..10, complex128 state "
                    "(%d GiB)" % (args.n, args.p, args.n, (16 << args.n) >> 30),
        "N": args.n, "p": args.p, "graph": "K%d" % args.n, "weights": "int U{1..10}",
        "angles": "gamma~U[0,pi), beta~U[0,pi/2)", "seed": args.seed,
        "l2": "state larger than L2 (no flush needed)",
    }


# ------------------------------------------------------------ distributed --

class Dist:
    """Rank bookkeeping; every rank is an independent replica.  Host-side
    gloo collectives carry only the barrier and the timing reductions."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        return self._reduce(x, "max")

    def sum(self, x):
        return self._reduce(x, "sum")

    def _reduce(self, x, op):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX if op == "max" else self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------ clocks --

REASON_BITS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
               0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
               0x100: "display_clock_setting"}


class ClockSampler:
    """Samples SM clock, power and clock-event reasons every 200 ms (read-only
    NVML queries) while the timed region runs."""

    def __init__(self, device_index):
        self.samples = []
        self.max_mhz = None
        self.err = None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            h = None
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(device_index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid).encode())
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.h = h
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report why
            self.nv = None
            self.err = repr(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                try:
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except AttributeError:
                    rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((sm, pw, rs))
            except Exception as e:
                self.err = repr(e)
            self._stop.wait(0.2)

    def start(self):
        if self.nv:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [],
                    "samples": 0, "error": self.err}
        busy = [s for s in self.samples if not (s[2] & 0x1)] or self.samples
        reasons = set()
        for s in busy:
            for bit, name in REASON_BITS.items():
                if s[2] & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(s[0] for s in busy), "sm_max_mhz": self.max_mhz,
                "power_w_max": max(s[1] for s in busy), "reasons": sorted(reasons),
                "samples": len(busy)}


# ------------------------------------------------------------ roofline --

def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def is_headline(args):
    """Whether the run is the configuration the reference's figure and the
    committed ncu traffic are quoted on (N=30, p=5)."""
    return args.n == 30 and args.p == 5


# The kernels behind each pass kind of the engine at N=30 (tiles of 4096
# amplitudes; strided tiles of 128-byte rows run paired, 512 threads).
KIND_KERNELS = {
    "init_pass": "fq::k_pass, PH_INIT (layer 0: launch-control init + phase + RX, write-only, "
                 "strided tile, paired)",
    "phase_pass": "fq::k_pass with GM2 (fused two-layer pass: RX, next layer's phase, RX; "
                  "strided tiles, paired)",
    "mixer_pass": "fq::k_pass, PH_NONE (RX only: the contiguous pass over qubits 0..11, and "
                  "the circuit's last pass)",
}


def ncu_traffic_per_launch(kind, args):
    """DRAM bytes (read + write) per launch of a pass kind at N=30 from the
    committed ncu summary (profiles/engine_passes_n30_p5.md), or None (other
    sizes have no committed figure)."""
    if not is_headline(args):
        return None
    p = os.path.join(ROOT, "profiles", "engine_passes_n30_p5.md")
    try:
        m = re.search(r"traffic_bytes_per_launch\[%s\]:\s*([0-9.eE+]+)" % kind, open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


# ------------------------------------------------------------ CPU leg --

CPU_CHUNKS = 32


def cpu_layer_parts(cl, gammas, betas, parts, start=0):
    """Seconds of `parts` consecutive parts (1/CPU_CHUNKS of a layer each)."""
    return [cl.chunk(start + k, gammas[(start + k) % len(gammas)],
                     betas[(start + k) % len(betas)]) for k in range(parts)]


def cpu_baseline_obj(args, graph, gammas, betas):
    """The oracle on the host cores at the benchmark's size: one whole layer
    of a full 2^N host state (the value), and the estimate from `cpu_parts`
    timed parts of a layer (scale_check = whole / estimate)."""
    import oracle
    cl = oracle.CpuLayer(graph, CPU_CHUNKS)
    try:
        cpu_layer_parts(cl, gammas, betas, 1)  # warm-up part
        t_parts = cpu_layer_parts(cl, gammas, betas, args.cpu_parts, start=1)
        est = sum(t_parts) * CPU_CHUNKS / len(t_parts)
        full = None if args.no_cpu_full else cl.full_layer(gammas[1], betas[1])
    finally:
        cl.free()
    cores = oracle.num_threads()
    out = {"unit": UNIT, "cores": cores, "kind": "port",
           "parts_estimate_s": est, "parts_timed": len(t_parts), "parts_per_layer": CPU_CHUNKS}
    if full is not None:
        out.update(value=1.0 / full, full_layer_s=full, scale_check=full / est,
                   sample="oracle (FP64 OpenMP restatement of src/rzz.cu:121-156 and "
                          "src/rx.cu:32-53) on one whole N=%d layer of a full 2^%d-amplitude "
                          "host state: the read-multiply cost phase with the K_%d pair loop on "
                          "every amplitude, then RX on every qubit; value = 1 / its time "
                          "(measured, not scaled); parts_estimate_s = %d timed parts of 1/%d "
                          "layer scaled by %d/%d"
                          % (args.n, args.n, args.n, len(t_parts), CPU_CHUNKS, CPU_CHUNKS,
                             len(t_parts)))
    else:
        out.update(value=1.0 / est,
                   sample="oracle on %d timed parts of 1/%d of an N=%d layer of a full "
                          "host state, scaled to a layer" % (len(t_parts), CPU_CHUNKS, args.n))
    return out


def reference_gpu_leg(args, graph, gammas, betas, chunk=11):
    """The reference's own single-device CUDA path (its unmodified sources,
    built by oracle/Makefile.ref with CHUNK_QUBIT = 11, the chunk of its
    committed ncu report) on this box's GPU: the layer loop of
    src/Weighted.cpp:115-138 timed with CUDA events on its compute stream."""
    import subprocess
    import tempfile
    exe = os.path.join(ORACLE_DIR, "_ref", "ref_harness_c%d" % chunk)
    if not os.path.exists(exe):
        return {"unavailable": "reference build oracle/_ref/ref_harness_c%d not present" % chunk}
    with tempfile.TemporaryDirectory() as td:
        fin, fout, fidx = (os.path.join(td, x) for x in ("in.bin", "out.bin", "idx.bin"))
        with open(fin, "wb") as f:
            f.write(np.array([args.n, chunk, len(gammas)], dtype=np.int32).tobytes())
            f.write(np.ascontiguousarray(graph, dtype=np.float64).tobytes())
            f.write(np.asarray(gammas, dtype=np.float64).tobytes())
            f.write(np.asarray(betas, dtype=np.float64).tobytes())
        np.array([0], dtype=np.int64).tofile(fidx)
        r = subprocess.run([exe, fin, fout, "sample", fidx], capture_output=True, text=True,
                           timeout=900)
        if r.returncode != 0:
            return {"unavailable": "reference harness exited %d: %s"
                    % (r.returncode, (r.stderr or r.stdout)[-300:])}
        raw = np.fromfile(fout, dtype=np.float64)
    loop_ms, norm, energy = (float(x) for x in raw[:3])
    return {"layers_per_s": len(gammas) / (loop_ms / 1000.0), "loop_ms": loop_ms,
            "chunk_qubit": chunk, "layers": len(gammas), "energy": energy, "norm": norm,
            "how": "FOR-QAOA's unmodified single-device CUDA path (oracle/Makefile.ref, "
                   "CHUNK_QUBIT=%d) run through oracle/ref_harness.cpp on this GPU; CUDA events "
                   "on its compute stream around the layer loop (its host-side launch work, "
                   "graph packing and swap tables included)" % chunk}


def run_reference_impl(args):
    """The reference algorithm on the host cores (oracle port), same metric
    and workload: each step is one part (1/32) of a layer on the full-size
    host state; one whole layer is timed once after the steps."""
    d = Dist()
    if d.rank != 0:
        d.close()
        return
    import oracle
    graphs, gammas, betas = workload(args.n, args.p, args.seed)
    wall0 = time.perf_counter()
    cl = oracle.CpuLayer(graphs[0], CPU_CHUNKS)
    try:
        cpu_layer_parts(cl, gammas, betas, args.warmup)
        t_steps = cpu_layer_parts(cl, gammas, betas, args.steps, start=args.warmup)
        full = None if args.no_cpu_full else cl.full_layer(gammas[1], betas[1])
    finally:
        cl.free()
    wall = time.perf_counter() - wall0
    ms_step = 1000.0 * statistics.mean(t_steps)
    value = (1.0 / CPU_CHUNKS) / (ms_step / 1000.0)
    cores = oracle.num_threads()
    cpu = {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": "each step: part k (of %d) of one N=%d layer on a full 2^%d-amplitude "
                     "host state -- the read-multiply cost phase with the K_%d pair loop on "
                     "1/%d of the amplitudes, RX on every qubit for 1/%d of its pairs; value "
                     "= (1/%d layer) / mean step time; wall %.1f s for the whole run"
                     % (CPU_CHUNKS, args.n, args.n, args.n, CPU_CHUNKS, CPU_CHUNKS,
                        CPU_CHUNKS, wall)}
    if full is not None:
        cpu.update(full_layer_s=full, scale_check=full / (CPU_CHUNKS * ms_step / 1000.0))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": (value / BASELINE_LAYERS_PER_S) if is_headline(args) else None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(args),
        "engine": "oracle port on the host cores (FP64, OpenMP): the reference ships no CPU "
                  "implementation",
        "layers_per_step": 1.0 / CPU_CHUNKS,
        "impl": "reference", "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu_leg(args, graphs[0], gammas, betas)
    print(json.dumps(line), flush=True)
    d.close()


# ------------------------------------------------------------ GPU leg --

def run_ours(args):
    import torch
    import forqaoa

    d = Dist()
    dev = d.local_rank
    torch.cuda.set_device(dev)
    graphs, gammas, betas = workload(args.n, args.p, args.seed)
    ctx = forqaoa.Context(dev)
    st = ctx.state(args.n)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    for _ in range(args.warmup):
        ctx.qaoa_forward(st, graphs[0], gammas, betas, energy=False)
    ctx.synchronize()

    # ---- timed region: device-resident inputs, CUDA events on ctx's stream
    clocks = ClockSampler(dev)
    ctx.profile_reset()
    ctx.set_profiling(True)
    launches0 = ctx.launches()
    d.barrier()
    ctx.synchronize()
    clocks.start()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.qaoa_forward(st, graphs[0], gammas, betas, energy=False)
    e1.record(stream)
    ctx.synchronize()
    clocks.stop()
    d.barrier()
    launches = ctx.launches() - launches0
    ms = e0.elapsed_time(e1)
    prof = ctx.profile()
    ctx.set_profiling(False)
    ms_max = d.max(ms)
    ms_per_step = ms_max / args.steps
    value = d.world * args.p * args.steps / (ms_max / 1000.0)

    # ---- e2e: public API with host inputs (graph re-uploaded every step from
    # pinned staging: alternate two K_30 graphs so no upload is skipped) and
    # <C> read back to the host every step.
    for k in range(args.warmup):
        ctx.qaoa_forward(st, graphs[k % 2], gammas, betas, energy=True)
    d.barrier()
    t0 = time.perf_counter()
    energy = None
    for k in range(args.steps):
        energy = ctx.qaoa_forward(st, graphs[k % 2], gammas, betas, energy=True)
    e2e_s = time.perf_counter() - t0
    e2e_s = d.max(e2e_s)
    e2e = {"value": d.world * args.p * args.steps / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": 4 * args.n * args.n, "d2h_bytes_per_step": 8,
           "ms_per_step": 1000.0 * e2e_s / args.steps, "energy_last": energy}

    # ---- roofline.  The engine's tile passes by kind: the layer-0 pass
    # (launch-control init, write-only), the phase passes (fused two-layer
    # passes) and the mixer passes (RX only).  The dominant kernel is the kind
    # with the largest share of device time; per_layer covers every pass.
    peak, peak_src = hbm_peak()
    kern = {}
    tot_ms = tot_b = tot_n = 0
    for kind in ("init_pass", "phase_pass", "mixer_pass"):
        if kind in prof:
            kms, kn, kb = prof[kind]
            kern[kind] = {"launches": kn, "ms_avg": kms / kn, "ms_total": kms,
                          "alg_bytes_per_launch": kb / kn, "gbs": kb / (kms / 1000.0) / 1e9,
                          "frac": kb / (kms / 1000.0) / 1e9 / peak,
                          "traffic": ncu_traffic_per_launch(kind, args)}
            tot_ms += kms
            tot_b += kb
            tot_n += kn
    dom_kind = max(kern, key=lambda k: kern[k]["ms_total"]) if kern else None
    dom = kern.get(dom_kind, {})
    layer_gbs = tot_b / (tot_ms / 1000.0) / 1e9 if tot_ms else None
    roofline = {"bound": "hbm", "achieved": dom.get("gbs"), "peak": peak, "unit": "GB/s",
                "frac": dom.get("frac"),
                "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)" if
                peak_src == "measured" else "fallback 6.65 TB/s",
                "traffic": dom.get("traffic"),
                "kernel": KIND_KERNELS.get(dom_kind),
                "kind": dom_kind,
                "alg_bytes_per_launch": dom.get("alg_bytes_per_launch"),
                "per_layer": {"gbs": layer_gbs, "frac": layer_gbs / peak if layer_gbs else None,
                              "launches": tot_n,
                              "kernels": "every tile pass of the circuit (fq::k_pass, "
                                         "fq::k_pass_tma)",
                              "sweeps_per_layer": tot_n / (args.steps * args.p),
                              "alg_bytes_per_layer": tot_b / (args.steps * args.p),
                              "share_of_step": (tot_ms / ms) if ms else None},
                "per_kind": kern}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": (value / BASELINE_LAYERS_PER_S) if is_headline(args) else None,
        "dtype": "f64", "data": "synthetic", "config": workload_config(args),
        "engine": "fused tile passes (fq_qaoa_forward)", "layers_per_step": args.p,
        "parallelism": "replicas" if d.world > 1 else "single",
        "amp_updates_per_s": value * (1 << args.n) * (args.n + 1),
        "e2e": e2e, "roofline": roofline, "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    st.free()

    # ---- the reference's own schedule through the per-kernel entry points
    if not args.no_ref_schedule:
        line["reference_schedule"] = reference_schedule_leg(ctx, args, graphs[0], gammas, betas,
                                                            peak)
    # ---- adjoint gradient of the N=26 p=10 circuit (one GPU)
    if not args.no_grad and d.world == 1:
        line["gradient"] = gradient_leg(ctx, peak)
    # ---- served energy+gradient stream vs sequential plain calls (one GPU)
    if args.serve_requests > 0 and d.world == 1:
        line["serving"] = serving_leg(args)
    # ---- config 3: N=32 p=3, 3-regular graph with FP64 weights (one GPU),
    # after the serving leg, whose processes then have the device's memory
    if not args.no_config3 and d.world == 1:
        line["config3"] = config3_leg(ctx, peak)
    # ---- CPU baseline (rank 0, one GPU only)
    if not args.no_cpu and d.world == 1 and d.rank == 0:
        line["cpu_baseline"] = cpu_baseline_obj(args, graphs[0], gammas, betas)
    ctx.close()
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.close()


def gradient_leg(ctx, peak, n=26, P=10, reps=5):
    """<C> and its 2p partial derivatives (adjoint method) for K_26 with
    integer weights 1..10 and p=10: ms per evaluation and the adjoint
    kernel's HBM GB/s (64 B per amplitude per launch: both vectors read and
    written)."""
    rng = np.random.default_rng(2610)
    W = np.triu(rng.integers(1, 11, size=(n, n)).astype(np.float64), 1)
    g, b = rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)
    sv, cs = ctx.state(n), ctx.state(n)
    try:
        ctx.energy_grad(n, W, g, b, sv=sv, costate=cs)  # warm-up
        ctx.profile_reset()
        ctx.set_profiling(True)
        t0 = time.perf_counter()
        for _ in range(reps):
            e, gg, gb = ctx.energy_grad(n, W, g, b, sv=sv, costate=cs)
        wall = (time.perf_counter() - t0) / reps
        prof = ctx.profile()
        ctx.set_profiling(False)
    finally:
        sv.free()
        cs.free()
    out = {"workload": f"K_{n} integer weights 1..10, p={P}, <C> + {2 * P} derivatives",
           "ms_per_eval": 1000.0 * wall, "energy": e, "kernels": {}}
    for kind, (kms, kn, kb) in prof.items():
        gbs = kb / (kms / 1000.0) / 1e9 if kb else None
        out["kernels"][kind] = {"launches": kn // reps, "ms_per_eval": kms / reps, "gbs": gbs,
                                "frac": gbs / peak if gbs else None}
    return out


def regular3(n, rng):
    """A random 3-regular graph on n vertices by seeded pairing of 3n
    half-edges, redrawn while a pairing has a loop or a double edge."""
    while True:
        pts = rng.permutation(np.repeat(np.arange(n), 3))
        edges = set()
        for i in range(0, 3 * n, 2):
            u, v = int(min(pts[i], pts[i + 1])), int(max(pts[i], pts[i + 1]))
            if u == v or (u, v) in edges:
                break
            edges.add((u, v))
        else:
            return sorted(edges)


def config3_leg(ctx, peak, n=32, P=3, reps=3):
    """Benchmark config 3: N=32 (a 64 GiB state), p=3, a random 3-regular
    graph (48 edges) with FP64 weights in [0, 1), seeded.  The fused engine
    at three passes per layer (the contiguous one and two strided passes of
    10 qubits each over rows of 4 amplitudes); FP64 phases take the product
    tree where the weights' sum times |gamma| allows it, else one sincos of
    the reference's argument per amplitude.  layers/s from CUDA events on the
    library's stream, and the per-layer HBM fraction over every pass."""
    import torch
    rng = np.random.default_rng(32)
    W = np.zeros((n, n))
    for u, v in regular3(n, rng):
        W[u, v] = rng.uniform(0.0, 1.0)
    g, b = rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = ctx.state(n)
    try:
        ctx.qaoa_forward(st, W, g, b, energy=False)  # warm-up
        ctx.synchronize()
        ctx.profile_reset()
        ctx.set_profiling(True)
        e0.record(stream)
        for _ in range(reps):
            ctx.qaoa_forward(st, W, g, b, energy=False)
        e1.record(stream)
        ctx.synchronize()
        prof = ctx.profile()
        ctx.set_profiling(False)
        energy = ctx.qaoa_forward(st, W, g, b, energy=True)
    finally:
        st.free()
    ms = e0.elapsed_time(e1)
    kb = sum(v[2] for k, v in prof.items() if k in ("init_pass", "phase_pass", "mixer_pass"))
    kms = sum(v[0] for k, v in prof.items() if k in ("init_pass", "phase_pass", "mixer_pass"))
    gbs = kb / (kms / 1000.0) / 1e9 if kms else None
    return {"workload": f"N={n} p={P}, random 3-regular graph (48 edges), FP64 weights "
                        "U[0,1), complex128 state (64 GiB), seed 32",
            "layers_per_s": P * reps / (ms / 1000.0), "ms_per_circuit": ms / reps,
            "energy": energy,
            "per_layer": {"gbs": gbs, "frac": gbs / peak if gbs else None,
                          "sweeps_per_layer": sum(v[1] for k, v in prof.items()
                                                  if k in ("init_pass", "phase_pass",
                                                           "mixer_pass")) / (P * reps)},
            "kernels": {k: {"launches": v[1] // reps, "ms_per_circuit": v[0] / reps}
                        for k, v in prof.items()}}


def eval_bytes(ctx, n, P, cache):
    """Algorithmic HBM bytes of one energy+gradient evaluation (the library's
    per-launch accounting, summed over one evaluation), cached per (n, P)."""
    key = (n, P)
    if key not in cache:
        rng = np.random.default_rng(n * 100 + P)
        W = np.triu(rng.integers(1, 11, size=(n, n)).astype(np.float64), 1)
        ctx.profile_reset()
        ctx.set_profiling(True)
        ctx.energy_grad(n, W, rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P))
        prof = ctx.profile()
        ctx.set_profiling(False)
        cache[key] = sum(v[2] for v in prof.values())
    return cache[key]


def serving_ceiling(seq, peak_gbs, sms):
    """Best speed-up over sequential calls this stream allows: every request
    at least its HBM roofline time (algorithmic bytes / measured copy
    bandwidth; requests share one HBM), a request held in shared memory
    (N <= 15: one CTA up to 12 qubits, a cluster of 2^(N-12) CTAs above) at
    least its sequential time times its share of the SMs.  ceiling = sum of
    sequential times / sum of those bounds."""
    import forqaoa
    cache = {}
    t_seq = t_bound = 0.0
    with forqaoa.Context(0) as ctx:
        for r in seq:
            t_seq += r["latency"]
            if r["N"] <= forqaoa.SMALL_MAX_QUBITS:
                t_bound += r["latency"] * (1 << max(0, r["N"] - 12)) / sms
            else:
                t_bound += eval_bytes(ctx, r["N"], r["P"], cache) / (peak_gbs * 1e9)
    return t_seq / t_bound, t_seq, t_bound


def serving_leg(args):
    """The served stream (config 5: sessions of 20 energy+gradient steps,
    N ~ U{10..28}, p ~ U{1..8}, G(N,0.5) integer weights, Poisson session
    arrivals, 150 GB budget), every request loop driven natively
    (serve_replay): evals/s and p50/p99 latency through the server against
    the same evaluations as sequential calls, the speed-up ceiling this
    stream allows, latency at a sustainable arrival rate, and the stream per
    size class (by_size) against sequential and plain calls."""
    import serve_stream as ss
    peak, _ = hbm_peak()
    sessions, steps = ss.make_stream(args.serve_requests, seed=5)
    ss.run_native("served", sessions[:4], 2, lanes=args.serve_lanes)  # warm-up
    served, wall, info = ss.run_native("served", sessions, steps, lanes=args.serve_lanes)
    seq, wall_q, _ = ss.run_native("sequential", sessions, steps)
    out = ss.summarize(served, wall, seq, wall_q, None)
    out["server"] = info
    ceil, t_seq, t_bound = serving_ceiling(seq, peak, 148)
    out["ceiling_speedup_vs_sequential"] = ceil
    out["ceiling_note"] = ("sum of sequential times %.1f s / sum of per-request bounds %.1f s "
                           "(HBM roofline of each request's algorithmic bytes at %.0f GB/s; "
                           "shared-memory requests, N <= 15: sequential time x their CTAs / "
                           "148 SMs)" % (t_seq, t_bound, peak))
    out["stream"] = {"sessions": len(sessions), "steps": steps, "n": [10, 28], "p": [1, 8],
                     "graph": "G(N,0.5), integer weights 1..10", "seed": 5,
                     "arrivals": "Poisson, mean gap 1 ms (arrivals outpace the device: "
                                 "latency includes queueing)",
                     "lanes": args.serve_lanes, "budget_gb": 150,
                     "client": "serve_replay (native closed loop)"}
    # Latency where the server keeps up: sessions arriving at 80% of the
    # session rate just measured.
    cap_sessions_per_s = out["evals_per_s"] / steps
    gap_ms = 1000.0 / (0.8 * cap_sessions_per_s)
    sus, _ = ss.make_stream(args.serve_sustained_requests, seed=6, mean_gap_ms=gap_ms)
    sv, w, _ = ss.run_native("served", sus, steps, lanes=args.serve_lanes)
    r = ss.summarize(sv, w)
    out["sustained"] = {"requests": r["requests"], "arrival_gap_ms": gap_ms,
                        "load": "80% of the session rate measured above",
                        "evals_per_s": r["evals_per_s"], "latency_ms_p50": r["latency_ms_p50"],
                        "latency_ms_p99": r["latency_ms_p99"], "queue_ms_p50": r["queue_ms_p50"]}
    # The same stream restricted to one size class at a time: the mixed
    # stream's time is dominated by N = 27..28 (HBM-bound one at a time),
    # these show what batching and overlap do where a request is not.  All
    # sessions of a class arrive within the first few milliseconds (mean gap
    # 0.01 ms), so the served rate is the server's capacity, not the rate at
    # which 1 ms-spaced arrivals offer work (a session of small requests ends
    # in a few milliseconds).
    out["by_size"] = {}
    for lo, hi, n_req, lanes in ((10, 12, 4000, args.serve_lanes), (13, 15, 2000, args.serve_lanes),
                                 (16, 20, 2000, 16), (21, 28, 200, args.serve_lanes)):
        sess, steps = ss.make_stream(n_req, seed=lo, n_min=lo, n_max=hi, mean_gap_ms=0.01)
        sv, w, _ = ss.run_native("served", sess, steps, lanes=lanes)
        sq, wq, _ = ss.run_native("sequential", sess, steps)
        pl, wp, _ = ss.run_native("plain", sess, steps)
        r = ss.summarize(sv, w, sq, wq, None, pl, wp)
        out["by_size"][f"N {lo}..{hi}"] = {
            k: r[k] for k in ("requests", "evals_per_s", "latency_ms_p50", "latency_ms_p99",
                              "sequential_evals_per_s", "speedup_vs_sequential",
                              "plain_evals_per_s", "speedup_vs_plain",
                              "mismatches_vs_sequential", "mismatches_vs_plain")}
        out["by_size"][f"N {lo}..{hi}"]["lanes"] = lanes
        out["by_size"][f"N {lo}..{hi}"]["arrivals"] = "all sessions at once (mean gap 0.01 ms)"
    return out


def reference_schedule_leg(ctx, args, graph, gammas, betas, peak, steps=2):
    st = ctx.state(args.n)
    try:
        ctx.reference_schedule(st, graph, args.chunk, gammas, betas)  # warm-up
        ctx.synchronize()
        ctx.profile_reset()
        ctx.set_profiling(True)
        t0 = time.perf_counter()
        for _ in range(steps):
            ctx.reference_schedule(st, graph, args.chunk, gammas, betas)
        ctx.synchronize()
        wall = time.perf_counter() - t0
        prof = ctx.profile()
        ctx.set_profiling(False)
    finally:
        st.free()
    kern_ms = sum(v[0] for v in prof.values())
    out = {"chunk": args.chunk, "layers_per_s": args.p * steps / (kern_ms / 1000.0),
           "wall_layers_per_s": args.p * steps / wall, "kernels": {}}
    for kind, (kms, kn, kb) in prof.items():
        gbs = kb / (kms / 1000.0) / 1e9 if kb else None
        out["kernels"][kind] = {"launches": kn, "ms_avg": kms / kn, "gbs": gbs,
                                "frac": gbs / peak if gbs else None}
    return out


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference_impl(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
