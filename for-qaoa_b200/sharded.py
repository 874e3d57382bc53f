#!/usr/bin/env python3
"""QAOA on a state split over 2^D GPUs (the reference's D > 0 path), one
process per GPU over torch.distributed (NCCL).

The state of N qubits is split by its top D index bits: rank r holds the
2^(N-D) amplitudes whose physical qubits N-D..N-1 read r.  One layer:

  1. every rank: cost phase + RX(beta) on its N-D local qubits
     (fq_shard_layer: the tile passes of the single-GPU engine, with the
     rank's bits entering the cut values);
  2. one all-to-all of equal chunks: chunk d of every shard (the amplitudes
     whose local qubits N-2D..N-D-1 read d) goes to rank d, stored at the
     position of its source rank.  This swaps qubit blocks [N-2D, N-D) and
     [N-D, N) -- the reference's global/local swap (src/swap.cu:223-345),
     here with no packing kernel because the chunks are contiguous;
  3. every rank: RX(beta) on qubits N-2D..N-D-1, which now hold the qubits
     that were global: inside the next layer's first pass
     (fq_shard_layer_after_swap, one sweep fewer per layer), after the last
     layer as a pass of its own (fq_rx_targets);
  4. the graph is relabelled for the new physical order (fq_relabel_graph,
     as mapping_after_swap_conti, src/swap.cu:27-50) and the label map
     records which logical qubit each physical position holds.

The schedule (`forward`) is written against a small interface (`ShardOps`
methods and an exchange callable), so it runs with one shard per process
(`dist_exchange`) or with every shard in one process (`local_exchange`).

    torchrun --nproc-per-node 2 --master-addr 127.0.0.1 for-qaoa_b200/sharded.py --n 31 --p 3
    python for-qaoa_b200/sharded.py --n 30 --emulate 1     # both shards on one GPU, timed
"""
import argparse
import datetime
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


class ShardOps:
    """One shard on one GPU: a buffer of 2^(N-D) amplitudes, a spare buffer
    of the same size for the all-to-all, and the CUDA passes of the C ABI.
    `ctx` must run on the current torch stream, where the exchanges run (a
    stream of its own, not the legacy default stream, whose handle 0 would
    give the context a private stream: `shard_context`)."""

    def __init__(self, ctx, N, D, rank, device):
        import torch
        cur = torch.cuda.current_stream().cuda_stream
        if not cur or (ctx.stream or 0) != cur:
            raise ValueError("the context must run on the current torch stream (shard_context)")
        self.ctx, self.N, self.D, self.rank = ctx, N, D, rank
        self.n = N - D
        self.buf = torch.empty(1 << self.n, dtype=torch.complex128, device=device)
        self.spare = torch.empty_like(self.buf)

    def layer(self, graph, gamma, beta, first_layer):
        self.ctx.shard_layer(self.buf.data_ptr(), self.N, self.D, self.rank, graph, gamma, beta,
                             first_layer)

    def layer_after_swap(self, graph, gamma, beta, beta_prev):
        self.ctx.shard_layer_after_swap(self.buf.data_ptr(), self.N, self.D, self.rank, graph,
                                        gamma, beta, beta_prev)

    def rx_top(self, beta):
        n, D = self.n, self.D
        self.ctx.rx_targets_ptr(self.buf.data_ptr(), n, list(range(n - D, n)), beta)

    def expectation(self, graph):
        return self.ctx.shard_expectation(self.buf.data_ptr(), self.N, self.D, self.rank, graph)

    def swap(self):
        self.buf, self.spare = self.spare, self.buf


def shard_context(device):
    """A torch stream made current on `device` and a library context on it,
    so the passes and the exchanges share one stream order.  Returns
    (stream, context); the caller closes the context."""
    import torch
    import forqaoa
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    return stream, forqaoa.Context(device, stream.cuda_stream)


def local_exchange(shards):
    """The all-to-all with every shard in this process (shards[r] is rank
    r's): shard d receives chunk d of every shard r at chunk position r."""
    R = len(shards)
    m = shards[0].buf.numel() // R
    for d, sd in enumerate(shards):
        for r, sr in enumerate(shards):
            sd.spare[r * m:(r + 1) * m].copy_(sr.buf[d * m:(d + 1) * m])
    for s in shards:
        s.swap()


def dist_exchange(shards):
    """The all-to-all with one shard per process over torch.distributed
    (NCCL on GPUs, in the current stream's order; gloo on CPU tensors),
    equal splits."""
    import torch
    import torch.distributed as dist
    (s,) = shards
    dist.all_to_all_single(torch.view_as_real(s.spare), torch.view_as_real(s.buf))
    s.swap()


def relabel(graph, swap_out, swap_in, k):
    import forqaoa
    return forqaoa.relabel_graph(graph, swap_out, swap_in, k)


def forward(shards, exchange, N, D, graph, gammas, betas, relabel_fn=relabel, fuse=True):
    """The P-layer circuit from |+>^N on the given shards.  Returns the
    label map (physical position -> logical qubit) and the graph in the
    final physical order.  fuse: rotate the qubits each all-to-all swaps in
    inside the next layer's first pass (`layer_after_swap`) instead of in a
    pass of their own (`rx_top`) after every exchange."""
    n = N - D
    labels = np.arange(N)
    g = np.ascontiguousarray(graph, dtype=np.float64)
    for p, (gamma, beta) in enumerate(zip(gammas, betas)):
        for s in shards:
            if p > 0 and fuse:
                s.layer_after_swap(g, gamma, beta, betas[p - 1])
            else:
                s.layer(g, gamma, beta, p == 0)
        exchange(shards)
        if not fuse or p == len(gammas) - 1:
            for s in shards:
                s.rx_top(beta)
        g = relabel_fn(g, n - D, n, D)
        labels[n - D:n], labels[n:N] = labels[n:N].copy(), labels[n - D:n].copy()
    return labels, g


def to_logical(state_phys, labels):
    """Reorder a gathered physical-order state: position b holds logical
    qubit labels[b]."""
    N = len(labels)
    y = np.arange(1 << N, dtype=np.int64)
    x = np.zeros_like(y)
    for b, q in enumerate(labels):
        x |= ((y >> b) & 1) << int(q)
    out = np.empty_like(state_phys)
    out[x] = state_phys
    return out


def emulate(n_qubits, D, P, seed, fuse=True):
    """Every shard on GPU 0 (the exchange as chunk copies): device time per
    layer of the shard passes, the exchange and the separate RX passes of
    the swapped-in qubits, by CUDA events (one layer runs untimed first as
    warm-up).  With `fuse` the swapped-in qubits are rotated inside the
    next layer's first pass, and only the last layer's are a pass of their
    own."""
    import torch
    rng = np.random.default_rng(seed)
    N = n_qubits
    W = np.triu(rng.integers(1, 11, (N, N)).astype(np.float64), 1)
    g, b = rng.uniform(0, np.pi, P), rng.uniform(0, np.pi / 2, P)
    stream, ctx = shard_context(0)
    try:
        shards = [ShardOps(ctx, N, D, r, "cuda") for r in range(1 << D)]
        forward(shards, local_exchange, N, D, W, g[:1], b[:1])
        torch.cuda.synchronize()
        n = N - D
        gphys = np.ascontiguousarray(W)
        t = {"shard_passes": 0.0, "exchange": 0.0, "rx_swapped_in": 0.0}
        for p in range(P):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            e[0].record(stream)
            for s in shards:
                if p > 0 and fuse:
                    s.layer_after_swap(gphys, g[p], b[p], b[p - 1])
                else:
                    s.layer(gphys, g[p], b[p], p == 0)
            e[1].record(stream)
            local_exchange(shards)
            e[2].record(stream)
            if not fuse or p == P - 1:
                for s in shards:
                    s.rx_top(b[p])
            e[3].record(stream)
            torch.cuda.synchronize()
            for k, (i, j) in zip(t, ((0, 1), (1, 2), (2, 3))):
                t[k] += e[i].elapsed_time(e[j])
            gphys = relabel(gphys, n - D, n, D)
        ms = {k: v / P for k, v in t.items()}
        return {"N": N, "D": D, "p": P, "shards_on_one_gpu": 1 << D,
                "schedule": "swapped-in RX in the next layer's first pass" if fuse
                else "swapped-in RX as a pass of its own",
                "ms_per_layer": ms, "ms_per_layer_total": sum(ms.values())}
    finally:
        ctx.close()


def main(argv=None):
    import torch
    import torch.distributed as dist
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--n", type=int, default=31)
    ap.add_argument("--p", type=int, default=3)
    ap.add_argument("--seed", type=int, default=30)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--emulate", type=int, default=0, metavar="D",
                    help="run all 2^D shards on GPU 0 (no torch.distributed) and time the parts")
    ap.add_argument("--no-fuse", action="store_true",
                    help="rotate the swapped-in qubits in a pass of their own after every exchange")
    a = ap.parse_args(argv)
    if a.emulate:
        print(json.dumps(emulate(a.n, a.emulate, a.p, a.seed, fuse=not a.no_fuse)))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    D = world.bit_length() - 1
    if world < 2 or (1 << D) != world:
        raise SystemExit("needs a power-of-two world size >= 2 (one rank per GPU)")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    stream, ctx = shard_context(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    rng = np.random.default_rng(a.seed)
    W = np.triu(rng.integers(1, 11, (a.n, a.n)).astype(np.float64), 1)
    gammas, betas = rng.uniform(0, np.pi, a.p), rng.uniform(0, np.pi / 2, a.p)
    s = ShardOps(ctx, a.n, D, rank, "cuda")
    # Device time on the ranks' streams (CUDA events), the max over ranks.
    times = []
    for _ in range(a.steps):
        dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        _, g = forward([s], dist_exchange, a.n, D, W, gammas, betas, fuse=not a.no_fuse)
        t1.record(stream)
        torch.cuda.synchronize()
        times.append(t0.elapsed_time(t1) / 1000.0)
    e = torch.tensor([s.expectation(g)], dtype=torch.float64, device="cuda")
    dist.all_reduce(e)
    t = torch.tensor([min(times)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        print(json.dumps({"N": a.n, "D": D, "p": a.p, "ranks": world,
                          "layers_per_s": a.p / float(t.item()), "energy": float(e.item())}))
    ctx.close()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
