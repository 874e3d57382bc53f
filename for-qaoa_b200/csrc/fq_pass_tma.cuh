// fq_pass_tma.cuh -- the streaming tile pass as a persistent TMA pipeline.
//
// Same tile, thread layouts, cut decomposition and RX rounds as k_pass
// (fq_pass.cuh), but tiles reach shared memory through the Tensor Memory
// Accelerator instead of per-thread loads, so HBM keeps streaming while the
// CTA computes:
//   - one CTA per SM loops over its tiles; a ring of three 64 KB stage
//     buffers holds the tile being computed and the next two in flight;
//   - thread 0 issues one cp.async.bulk.tensor copy per tile (a 3-D or 5-D
//     box over the state seen as rows of 8 amplitudes = 128 bytes, 128-byte
//     swizzle, no multicast), completion counted on a per-stage mbarrier;
//   - the 256 threads read the landed tile into registers (layout L0),
//     rotate, exchange through the same buffer, and store with 16-byte
//     streaming stores straight from registers (layout L1), so no second
//     copy of the tile is staged for the way out.
// Every mbarrier wait is bounded: on expiry the CTA records an error flag
// the host reports as FQ_ERR_TIMEOUT, drains the copies it issued (again
// bounded) and returns.
#pragma once

#include <cuda.h>

#include "fq_pass.cuh"

namespace fq {

constexpr int kStages = 3;
constexpr unsigned kTileBytes = kTile * sizeof(double2);  // 64 KB
// Bound on mbarrier polls: a poll that finds the phase incomplete suspends
// the thread for ~4 us on B200 (2^16 polls measured 0.26 s), so 2^18 polls
// give up after about a second; a landing copy ends the wait at once.
constexpr long long kWaitSpins = 1ll << 18;

// Box geometry of a pass (host-chosen, see make_pass_tmap):
//   TG_CONTIG  l = 12: rank 3, box {16 doubles, 256 rows, 2}
//   TG_ROWS    4 <= l <= 11: rank 5, box {16, 2^(l-3), 1, 2^(12-l), 1}
//   TG_ROWS8   l = 3: rank 5, box {16, 1, 32, 16, 1}
enum { TG_CONTIG = 0, TG_ROWS = 1, TG_ROWS8 = 2 };

struct TmaGeom {
    int kind;
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier: at most max_polls polls
// (each may suspend the thread for a while); false if it gave up.  A
// %globaltimer bound in the loop cost the strided pass 10% (7.05 vs 6.41 ms
// at N=30), so the bound is a poll count.
__device__ __forceinline__ bool mbar_wait_polls(unsigned long long* bar, unsigned parity,
                                                long long max_polls) {
    for (long long i = 0; i < max_polls; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
    return mbar_wait_polls(bar, parity, kWaitSpins);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map,
                                            unsigned long long* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"((unsigned long long)map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map,
                                            unsigned long long* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
        "l"((unsigned long long)map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(c4)
        : "memory");
}

// Slot of tile index t in a buffer written by TMA with the 128-byte swizzle:
// 16-byte chunk bits 0..2 are XORed with the 128-byte row bits 0..2.
__device__ __forceinline__ int tslot(int t) { return t ^ ((t >> 3) & 7); }

// Bytes of the cut tables of a TMA pass: PassSmem without its exchange
// buffer (the landed stage serves as one); FP64 weights need no phase table
// (sincos), which keeps the ring plus tables within 227 KB.
template <typename WT>
__host__ __device__ constexpr size_t cut_table_bytes() {
    return sizeof(WT) == sizeof(int) ? PassSmem<WT>::bytes : PassSmem<WT>::smtab;
}

// Shared-memory bytes of the TMA pass (1 KB of alignment slack included):
// the ring, the mbarriers, 32 register-slot offsets, the cut tables.
template <typename WT>
__host__ __device__ constexpr size_t tma_pass_smem_bytes(int = 0) {
    return 1024 + (size_t)kStages * kTileBytes + 64 + 32 * sizeof(i64) + cut_table_bytes<WT>();
}
static_assert(tma_pass_smem_bytes<int>() <= 227 * 1024, "ring + tables fit one SM (int)");
static_assert(tma_pass_smem_bytes<double>() <= 227 * 1024, "ring + tables fit one SM (FP64)");
static_assert(kMaxQubits * kMaxQubits * sizeof(double) <= kTileBytes, "weights fit one stage");

template <typename WT, int PH, int GM, int EX, int SC>
__global__ void __launch_bounds__(kPassThreads, 1)
    k_pass_tma(const PassArgs A, const __grid_constant__ CUtensorMap tmap, const TmaGeom G) {
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    double2* stage = reinterpret_cast<double2*>(sm);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + kStages * kTileBytes);
    int* s_abort = reinterpret_cast<int*>(full + kStages);
    i64* offtab = reinterpret_cast<i64*>(sm + kStages * kTileBytes + 64);
    unsigned char* tsm = sm + kStages * kTileBytes + 64 + 32 * sizeof(i64);
    const CutTables<WT> ct(tsm);
    double* red = reinterpret_cast<double*>(tsm + PassSmem<WT>::red);
    double2* smtab = reinterpret_cast<double2*>(tsm + PassSmem<WT>::smtab);
    constexpr bool CUT = (PH != PH_NONE) || (EX == EX_ENERGY);
    constexpr bool INTW = sizeof(WT) == sizeof(int);
    // <C> of a pass whose rounds end in layout L1 is taken there (the cut
    // constants of L1), so the tile leaves from L1 without a change back.
    constexpr bool E1 = EX == EX_ENERGY && GM != GM_NONE && SC != SC_L0;
    const int N = A.N, l = A.l, a = A.a;
    const int nF = N - kTileBits;
    const int nmid = a - l;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const i64 my_tiles =
        blockIdx.x < A.ntiles ? (A.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    // Issue the copy of this CTA's tile j into stage j % kStages.
    auto issue = [&](i64 j) {
        const i64 T = blockIdx.x + j * (i64)gridDim.x;
        const int s = (int)(j % kStages);
        void* dst = stage + (size_t)s * kTile;
        mbar_expect_tx(&full[s], kTileBytes);
        if (G.kind == TG_CONTIG) {
            tma_load_3d(dst, &tmap, &full[s], 0, 0, (int)(2 * T));
        } else if (G.kind == TG_ROWS) {
            tma_load_5d(dst, &tmap, &full[s], 0, 0, (int)(T & ((1ll << nmid) - 1)), 0,
                        (int)(T >> nmid));
        } else {
            tma_load_5d(dst, &tmap, &full[s], 0, (int)(T & ((1ll << nmid) - 1)), 0, 0,
                        (int)(T >> nmid));
        }
    };

    // ---- set-up.  The weights are staged in the last stage, which no copy
    // fills before the loop's first barrier.
    if (tid == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&full[s], 1);
        *s_abort = 0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (tid < 2 * kRegs) {
        const int r = tid & 15, lo = tid < kRegs ? 8 : 4;
        i64 o = 0;
        for (int k = 0; k < 4; k++)
            if ((r >> k) & 1) o += 1ll << tile_phys(lo + k, l, a);
        offtab[tid] = o;
    }
    WT* sw = reinterpret_cast<WT*>(stage + (size_t)(kStages - 1) * kTile);
    if (CUT) {
        const WT* gw = reinterpret_cast<const WT*>(A.w);
        for (int i = tid; i < N * N; i += kPassThreads) sw[i] = gw[i];
    }
    if (PH != PH_NONE && INTW) load_phase_tables(A, smtab, tid, kPassThreads);
    __syncthreads();
    if (tid == 0)
        for (i64 j = 0; j < kStages - 1 && j < my_tiles; j++) issue(j);
    if (CUT) ct.template setup<false>(sw, N, l, a, tid, A.gamma);

    i64 thr_off = 0, thr_off1 = 0;
    for (int jj = 0; jj < 8; jj++) thr_off |= (i64)((tid >> jj) & 1) << tile_phys(jj, l, a);
    {
        const int t1 = lay_index<1>(tid, 0);
        for (int jj = 0; jj < kTileBits; jj++)
            if ((t1 >> jj) & 1) thr_off1 |= 1ll << tile_phys(jj, l, a);
    }
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    WT* const kp = ct.ke;  // written after a tile's first barrier, read after its second
    double acc = 0, comp = 0;
    i64 j = 0;

    for (; j < my_tiles; j++) {
        const i64 T = blockIdx.x + j * (i64)gridDim.x;
        const i64 base = ((T & ((1ll << nmid) - 1)) << l) | ((T >> nmid) << (a + kTileBits - l));
        const int s = (int)(j % kStages);
        double2* buf = stage + (size_t)s * kTile;
        __syncthreads();  // tile j-1 (or the set-up) is finished: its stage may be refilled
        if (tid == 0 && j + kStages - 1 < my_tiles) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(j + kStages - 1);
        }
        if (CUT) ct.tile(kp, base | A.goff, nF, l, a, warp, lane);  // warps 0 and 1, while the copy lands
        if (!mbar_wait_bounded(&full[s], (unsigned)((j / kStages) & 1))) {
            *s_abort = 1;
            if (A.err) atomicExch(A.err, 1);
        }
        __syncthreads();  // tile landed (or abort), kp visible
        if (*s_abort) break;

        double2 v[kRegs];
#pragma unroll
        for (int r = 0; r < kRegs; r++) v[r] = buf[tslot(lay_index<0>(tid, r))];
        if (PH != PH_NONE) {
            WT cbase, g0, g1, g2, g3;
            ct.consts(kp, tid, cbase, g0, g1, g2, g3);
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + ct.creg[r] + ((r & 1) ? g0 : WT(0)) +
                              ((r & 2) ? g1 : WT(0)) + ((r & 4) ? g2 : WT(0)) +
                              ((r & 8) ? g3 : WT(0));
                double2 ph;
                if (INTW) {
                    ph = int_phase(A, smtab, (int)cr);
                } else {
                    const double S = 2.0 * (double)cr - A.W;
                    double sn, cs;
                    sincos(S * A.gamma / 2, &sn, &cs);
                    ph.x = cs;
                    ph.y = sn;
                }
                if (PH == PH_INIT) {
                    v[r].x = ph.x * A.scale;
                    v[r].y = ph.y * A.scale;
                } else {
                    if (!INTW) {
                        ph.x *= A.scale;
                        ph.y *= A.scale;
                    }
                    const double2 in = v[r];
                    v[r].x = in.x * ph.x - in.y * ph.y;
                    v[r].y = in.x * ph.y + in.y * ph.x;
                }
            }
        }
        constexpr int LAY = (GM != GM_NONE && SC != SC_L0 && (EX == EX_NONE || E1)) ? 1 : 0;
        if (GM != GM_NONE) {
            rx_regs<GM>(v, m_hi, A.gx, A.c, A.s);
            if (lo_lane >= 0) rx_lane<GM>(v, lo_lane, A.gx, A.c, A.s);
            if (SC == SC_L021) {
                exchange<0, 2, false, false>(v, buf, tid);
                rx_regs<GM>(v, m_lo, A.gx, A.c, A.s);
                exchange<2, 1, false, false>(v, buf, tid);
            } else if (SC == SC_L01) {
                exchange<0, 1, false, false>(v, buf, tid);
            }
            if (SC != SC_L0) {
                rx_regs<GM>(v, m_mid, A.gx, A.c, A.s);
                if (LAY == 0) exchange<1, 0, false, false>(v, buf, tid);
            }
        }
        if (EX == EX_ENERGY) {
            constexpr int LE = E1 ? 1 : 0;  // layout of the registers here
            WT cbase, g0, g1, g2, g3;
            ct.template consts<LE>(kp, tid, cbase, g0, g1, g2, g3);
            const WT* crg = ct.creg + 16 * LE;
            double ts = 0;
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                ts = fma(fma(v[r].x, v[r].x, v[r].y * v[r].y), (double)cr, ts);
            }
            const double y = ts - comp;
            const double t2 = acc + y;
            comp = (t2 - acc) - y;
            acc = t2;
        }
        if (LAY == 0) {
            double2* const p = A.sv + base + thr_off;
#pragma unroll
            for (int r = 0; r < kRegs; r++) __stcs(p + offtab[r], v[r]);
        } else {
            double2* const p1 = A.sv + base + thr_off1;
#pragma unroll
            for (int r = 0; r < kRegs; r++) __stcs(p1 + offtab[kRegs + r], v[r]);
        }
    }
    if (*s_abort) {
        // Drain the copies still in flight into this CTA's stages (bounded).
        if (tid == 0)
            for (i64 k = j; k < j + kStages && k < my_tiles; k++)
                mbar_wait_bounded(&full[k % kStages], (unsigned)((k / kStages) & 1));
        return;
    }
    if (EX == EX_ENERGY) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        __syncthreads();
        if (lane == 0) red[warp] = acc;
        __syncthreads();
        if (tid == 0) {
            double sum = 0;
            for (int w = 0; w < kPassThreads / 32; w++) sum += red[w];
            A.partial[blockIdx.x] = sum;
        }
    }
}

}  // namespace fq
