"""CPU tests of bench.py's multi-rank plumbing (gloo, world size 2) and of
its reference arm (the oracle timed on host cores).  Every rank is an
independent replica; the only collectives are the barrier and the
max/sum reductions of timings."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT

BENCH = os.path.join(ROOT, "bench.py")


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    q.put((rank, d.max(10.0 + rank), d.sum(1.0 + rank)))
    d.barrier()
    d.close()


def test_dist_reductions_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 11.0, 3.0), (1, 11.0, 3.0)]


def _json_lines(text):
    return [json.loads(l) for l in text.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    """The reference arm on a 2^20-amplitude state (the default is the
    benchmark's N=30, 16 GiB of host memory): its line carries the GPU arm's
    workload config, the parts' timing and the whole-layer check."""
    r = subprocess.run([sys.executable, BENCH, "--impl", "reference", "--steps", "2",
                        "--warmup", "1", "--n", "20", "--no-ref-gpu"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    (line,) = _json_lines(r.stdout)
    assert line["impl"] == "reference" and line["unit"] == "layers/s"
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["N"] == 20 and "engine" not in line["config"]
    assert line["cpu_baseline"]["full_layer_s"] > 0 and line["cpu_baseline"]["scale_check"] > 0
    assert line["layers_per_step"] == 1 / 32
    assert abs(line["value"] * line["ms_per_step"] / 1000 - 1 / 32) < 1e-9


def test_reference_arm_under_torchrun_prints_once():
    port = free_port()
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port",
                        str(port), BENCH, "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "1", "--qubits", "18", "--no-ref-gpu"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _json_lines(r.stdout)
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2


def test_config3_graph_is_seeded_3_regular():
    """The config-3 leg's graph: 48 distinct edges on 32 vertices, each vertex
    of degree 3, the same for the same seed."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    e1 = bench.regular3(32, np.random.default_rng(32))
    e2 = bench.regular3(32, np.random.default_rng(32))
    assert e1 == e2 and len(e1) == 48 and len(set(e1)) == 48
    deg = np.zeros(32, dtype=int)
    for u, v in e1:
        assert 0 <= u < v < 32
        deg[u] += 1
        deg[v] += 1
    assert (deg == 3).all()
