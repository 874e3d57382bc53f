"""The sharded schedule of for-qaoa_b200/sharded.py (the D > 0 path) over
torch.distributed with the gloo backend on CPU, world sizes 2 and 4 (D = 1,
2): each rank holds one shard, the all-to-all is the product's
`dist_exchange`, the graph relabelling the library's fq_relabel_graph, and
the passes on a shard a numpy stand-in written here from the textbook gate
definitions (the CUDA passes are checked in test_gpu_shard.py).  The
gathered state, reordered by the label map, and the summed <C> are checked
against the oracle."""
import os
import socket
import sys
import tempfile

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import PKG, ENERGY_RTOL, assert_state_close, complete_int, gnp_fp, angles

sys.path.insert(0, PKG)


class NumpyShard:
    """Rank r's 2^(N-D) amplitudes (global index = r << (N-D) | local) and
    the passes of one layer on them."""

    def __init__(self, N, D, rank):
        self.N, self.D, self.rank, self.n = N, D, rank, N - D
        self.buf = torch.zeros(1 << self.n, dtype=torch.complex128)
        self.spare = torch.empty_like(self.buf)

    def _cut(self, graph):
        z = (self.rank << self.n) | np.arange(1 << self.n, dtype=np.int64)
        C = np.zeros(1 << self.n)
        for i in range(self.N):
            for j in range(i + 1, self.N):
                if graph[i, j] != 0:
                    C += graph[i, j] * (((z >> i) ^ (z >> j)) & 1)
        return C

    @staticmethod
    def _rx(psi, q, beta):
        c, s = np.cos(beta / 2), np.sin(beta / 2)
        v = psi.reshape(-1, 2, 1 << q)
        a0, a1 = v[:, 0, :].copy(), v[:, 1, :].copy()
        v[:, 0, :] = c * a0 - 1j * s * a1
        v[:, 1, :] = -1j * s * a0 + c * a1

    def layer(self, graph, gamma, beta, first_layer):
        W = np.triu(graph, 1).sum()
        ph = np.exp(0.5j * gamma * (2 * self._cut(graph) - W))
        psi = self.buf.numpy()
        if first_layer:
            psi[:] = 2.0 ** (-self.N / 2) * ph
        else:
            psi *= ph
        for q in range(self.n):
            self._rx(psi, q, beta)

    def layer_after_swap(self, graph, gamma, beta, beta_prev):
        self.rx_top(beta_prev)
        self.layer(graph, gamma, beta, False)

    def rx_top(self, beta):
        psi = self.buf.numpy()
        for q in range(self.n - self.D, self.n):
            self._rx(psi, q, beta)

    def expectation(self, graph):
        return float(np.sum(np.abs(self.buf.numpy()) ** 2 * self._cut(graph)))

    def swap(self):
        self.buf, self.spare = self.spare, self.buf


def _rank_main(rank, world, port, N, W, g, b, outdir):
    import sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        D = world.bit_length() - 1
        s = NumpyShard(N, D, rank)
        labels, gfin = sharded.forward([s], sharded.dist_exchange, N, D, W, g, b)
        e = torch.tensor([s.expectation(gfin)], dtype=torch.float64)
        dist.all_reduce(e)
        parts = [torch.empty_like(s.buf) for _ in range(world)]
        dist.all_gather(parts, s.buf)
        if rank == 0:
            np.save(os.path.join(outdir, "state.npy"), torch.cat(parts).numpy())
            np.save(os.path.join(outdir, "labels.npy"), labels)
            np.save(os.path.join(outdir, "energy.npy"), e.numpy())
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


@pytest.mark.parametrize("world,N,P,kind", [(2, 9, 3, "int"), (4, 10, 2, "fp"), (2, 11, 1, "int"),
                                            (4, 12, 3, "int")])
def test_sharded_schedule_matches_oracle(oracle, world, N, P, kind):
    import sharded
    rng = np.random.default_rng(100 * world + N)
    W = complete_int(N, rng) if kind == "int" else gnp_fp(N, rng)
    g, b = angles(rng, P)
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank_main, args=(world, _free_port(), N, W, g, b, d), nprocs=world, join=True)
        psi = np.load(os.path.join(d, "state.npy"))
        labels = np.load(os.path.join(d, "labels.npy"))
        e = float(np.load(os.path.join(d, "energy.npy"))[0])
    want = oracle.qaoa_logical(W, g, b)
    assert_state_close(sharded.to_logical(psi, labels), want, what=f"sharded N={N} x{world}")
    eo = oracle.expectation(want, W)
    assert abs(e - eo) <= ENERGY_RTOL * max(1.0, abs(eo))
    # Every layer moves D qubits out of and back into the device bits.
    assert sorted(labels.tolist()) == list(range(N))


@pytest.mark.parametrize("fuse", [True, False])
@pytest.mark.parametrize("D,N,P", [(1, 8, 2), (2, 9, 3), (3, 10, 2)])
def test_local_exchange_schedule_matches_oracle(oracle, D, N, P, fuse):
    """Every shard in this process: `local_exchange` (the chunk copies the
    one-GPU emulation uses) in place of the collective; the swapped-in
    qubits rotated in the next layer's first pass or after each exchange."""
    import sharded
    rng = np.random.default_rng(7 * N + D)
    W = complete_int(N, rng)
    g, b = angles(rng, P)
    shards = [NumpyShard(N, D, r) for r in range(1 << D)]
    labels, gfin = sharded.forward(shards, sharded.local_exchange, N, D, W, g, b, fuse=fuse)
    psi = torch.cat([s.buf for s in shards]).numpy()
    want = oracle.qaoa_logical(W, g, b)
    assert_state_close(sharded.to_logical(psi, labels), want, what=f"local N={N} D={D}")
    e = sum(s.expectation(gfin) for s in shards)
    eo = oracle.expectation(want, W)
    assert abs(e - eo) <= ENERGY_RTOL * max(1.0, abs(eo))
