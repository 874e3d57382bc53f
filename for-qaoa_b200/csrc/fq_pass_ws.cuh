// fq_pass_ws.cuh -- the strided RX pass as a warp-specialised TMA pipeline
// with TMA stores.
//
// Same tile, thread layouts and RX rounds as k_pass_tma (fq_pass_tma.cuh),
// for passes without a cost phase or <C> (the strided passes of a layer).
// The difference is the way out and who drives the pipeline:
//   - one producer warp (warp 8; one elected thread) issues every TMA load
//     and store and is the only thread that ever waits for the copy engine;
//   - 8 consumer warps (256 threads) wait for a landed tile, rotate it in
//     registers (exchanging through the tile's own stage buffer), write the
//     result back into that buffer in the TMA layout and signal the stage;
//   - the producer then stores the stage with one cp.async.bulk.tensor
//     store, waits until the copy engine has read it and refills it with the
//     tile three ahead.
// So the consumers issue no global stores at all (the strided pass with
// per-thread stores stalled on its store queue), and loading, computing and
// storing of different tiles overlap.  No multicast.  Every mbarrier wait
// is bounded; on expiry the error flag is set (FQ_ERR_TIMEOUT on the host),
// the copies in flight are drained (bounded) and the kernel returns.
#pragma once

#include "fq_pass_tma.cuh"

namespace fq {

constexpr int kWsConsumers = kPassThreads;           // 8 consumer warps
constexpr int kWsThreads = kWsConsumers + 32;        // + the producer warp

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0,
                                             int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
            (unsigned long long)map),
        "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, const void* src, int c0,
                                             int c1, int c2, int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5, %6}], "
        "[%1];" ::"l"((unsigned long long)map),
        "r"(smem_addr(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Every committed bulk store has finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Barrier of the 256 consumer threads (named barrier 1).
__device__ __forceinline__ void consumer_sync() {
    asm volatile("bar.sync 1, %0;" ::"r"(kWsConsumers) : "memory");
}

// The same barrier, returning whether any consumer passed p = true: every
// consumer gets the same answer, so a decision to stop stays uniform.
__device__ __forceinline__ bool consumer_sync_or(bool p) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((unsigned)p), "r"(kWsConsumers)
        : "memory");
    return r != 0;
}

// Layout change through buf; the caller has already synchronised the
// consumers since their last reads of buf.
template <int LF, int LT>
__device__ __forceinline__ void exchange_ws(double2 (&v)[kRegs], double2* buf, int tid) {
#pragma unroll
    for (int r = 0; r < kRegs; r++) buf[xslot(lay_index<LF>(tid, r))] = v[r];
    consumer_sync();
#pragma unroll
    for (int r = 0; r < kRegs; r++) v[r] = buf[xslot(lay_index<LT>(tid, r))];
}

__host__ __device__ inline size_t ws_pass_smem_bytes() {
    return 1024 + (size_t)kStages * kTileBytes + 2 * kStages * sizeof(unsigned long long) + 16;
}

// RX on the tile bits of A.tmask (reduced form GM, round schedule SC); no
// phase, no <C>.
template <int GM, int SC>
__global__ void __launch_bounds__(kWsThreads, 1)
    k_pass_ws(const PassArgs A, const __grid_constant__ CUtensorMap tmap, const TmaGeom G) {
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    double2* stage = reinterpret_cast<double2*>(sm);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + kStages * kTileBytes);
    unsigned long long* done = full + kStages;
    const int tid = threadIdx.x;
    const int nmid = A.a - A.l;
    const i64 my_tiles =
        blockIdx.x < A.ntiles ? (A.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // Box coordinates of this CTA's tile j (the same box for load and store).
    auto coords = [&](i64 j, int* c) {
        const i64 T = blockIdx.x + j * (i64)gridDim.x;
        c[0] = c[1] = c[2] = c[3] = c[4] = 0;
        if (G.kind == TG_CONTIG) {
            c[2] = (int)(2 * T);
        } else if (G.kind == TG_ROWS) {
            c[2] = (int)(T & ((1ll << nmid) - 1));
            c[4] = (int)(T >> nmid);
        } else {
            c[1] = (int)(T & ((1ll << nmid) - 1));
            c[4] = (int)(T >> nmid);
        }
    };
    auto load = [&](i64 j) {
        const int s = (int)(j % kStages);
        int c[5];
        coords(j, c);
        mbar_expect_tx(&full[s], kTileBytes);
        if (G.kind == TG_CONTIG)
            tma_load_3d(stage + (size_t)s * kTile, &tmap, &full[s], c[0], c[1], c[2]);
        else
            tma_load_5d(stage + (size_t)s * kTile, &tmap, &full[s], c[0], c[1], c[2], c[3], c[4]);
    };
    auto store = [&](i64 j) {
        const int s = (int)(j % kStages);
        int c[5];
        coords(j, c);
        if (G.kind == TG_CONTIG)
            tma_store_3d(&tmap, stage + (size_t)s * kTile, c[0], c[1], c[2]);
        else
            tma_store_5d(&tmap, stage + (size_t)s * kTile, c[0], c[1], c[2], c[3], c[4]);
        bulk_commit();
    };

    if (tid == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&done[s], kWsConsumers);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();

    if (tid >= kWsConsumers) {
        // ---- producer: one elected thread drives the copy engine
        if (tid == kWsConsumers) {
            i64 issued = 0;
            for (; issued < kStages && issued < my_tiles; issued++) load(issued);
            bool ok = true;
            for (i64 j = 0; j < my_tiles; j++) {
                const int s = (int)(j % kStages);
                if (!mbar_wait_bounded(&done[s], (unsigned)((j / kStages) & 1))) {
                    ok = false;  // consumers gave up (or stalled): stop issuing
                    break;
                }
                store(j);
                if (j + kStages < my_tiles) {
                    bulk_wait_read_all();  // stage s is read out: refill it
                    load(j + kStages);
                    issued = j + kStages + 1;
                }
            }
            if (!ok) {
                if (A.err) atomicExch(A.err, 2);
                // Drain loads still in flight into this CTA's stages (bounded).
                for (i64 k = issued - kStages; k < issued; k++)
                    if (k >= 0) mbar_wait_bounded(&full[k % kStages], (unsigned)((k / kStages) & 1));
            }
            bulk_wait_all();  // stores complete before the CTA's memory goes away
        }
        return;
    }

    // ---- consumers
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    for (i64 j = 0; j < my_tiles; j++) {
        const int s = (int)(j % kStages);
        double2* buf = stage + (size_t)s * kTile;
        const bool ok = mbar_wait_bounded(&full[s], (unsigned)((j / kStages) & 1));
        double2 v[kRegs];
#pragma unroll
        for (int r = 0; r < kRegs; r++)
            v[r] = ok ? buf[tslot(lay_index<0>(tid, r))] : make_double2(0.0, 0.0);
        rx_regs<GM>(v, m_hi, A.gx, A.c, A.s);
        if (lo_lane >= 0) rx_lane<GM>(v, lo_lane, A.gx, A.c, A.s);
        // Every consumer has read the landed tile (buf may be overwritten),
        // and all agree whether the tile landed at all.
        if (consumer_sync_or(!ok)) {
            if (tid == 0 && A.err) atomicExch(A.err, 1);
            break;  // the producer's bounded wait on `done` then gives up too
        }
        if (SC == SC_L021) {
            exchange_ws<0, 2>(v, buf, tid);
            rx_regs<GM>(v, m_lo, A.gx, A.c, A.s);
            consumer_sync();
            exchange_ws<2, 1>(v, buf, tid);
        } else if (SC == SC_L01) {
            exchange_ws<0, 1>(v, buf, tid);
        }
        constexpr int LAY = SC != SC_L0 ? 1 : 0;
        if (SC != SC_L0) {
            rx_regs<GM>(v, m_mid, A.gx, A.c, A.s);
            consumer_sync();  // every consumer is done reading the exchange
        }
#pragma unroll
        for (int r = 0; r < kRegs; r++) buf[tslot(lay_index<LAY>(tid, r))] = v[r];
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(&done[s]);
    }
}

}  // namespace fq
