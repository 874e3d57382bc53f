// fq_pass_tmaf.cuh -- the fused two-layer pass as a persistent TMA pipeline.
//
// Same work as k_pass with GM2 (RX of layer p on the tile's targets, the
// cost phase of layer p+1, RX of layer p+1 on the same targets), with the
// tiles streamed by the ring of k_pass_tma: one CTA per SM, three 64 KB
// stages, one bulk tensor copy per tile issued two tiles ahead, completion
// on a per-stage mbarrier (bounded waits; on expiry the CTA records the
// error flag, drains its copies and returns).  The landed stage is also the
// exchange buffer of the layout changes, and the tile leaves from registers
// (layout L0) with streaming stores.  The cut decomposition is CutTables
// (constants for layouts L0 and L1), so the phase is applied in L1 between
// the two layers' rounds as in k_pass.
#pragma once

#include "fq_pass_tma.cuh"

namespace fq {

// Shared memory: 1 KB of alignment slack, the ring, the mbarriers, the cut
// tables (cut_table_bytes).
template <typename WT>
__host__ __device__ constexpr size_t tmaf_smem_bytes() {
    return 1024 + (size_t)kStages * kTileBytes + 64 + cut_table_bytes<WT>();
}

template <typename WT, int GM, int GM2, int SC>
__global__ void __launch_bounds__(kPassThreads, 1)
    k_pass_tmaf(const PassArgs A, const __grid_constant__ CUtensorMap tmap, const TmaGeom G) {
    extern __shared__ unsigned char smraw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smraw) + 1023) & ~(uintptr_t)1023);
    double2* stage = reinterpret_cast<double2*>(sm);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + kStages * kTileBytes);
    int* s_abort = reinterpret_cast<int*>(full + kStages);
    unsigned char* tsm = sm + kStages * kTileBytes + 64;
    const CutTables<WT> ct(tsm);
    double2* smtab = reinterpret_cast<double2*>(tsm + PassSmem<WT>::smtab);
    constexpr bool INTW = sizeof(WT) == sizeof(int);
    constexpr int LP = SC == SC_L0 ? 0 : 1;  // layout of the phase
    const int N = A.N, l = A.l, a = A.a;
    const int nF = N - kTileBits;
    const int nmid = a - l;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const i64 my_tiles =
        blockIdx.x < A.ntiles ? (A.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const bool tree = INTW ? A.nhi > 0 : A.tree != 0;

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
    WT* sw = reinterpret_cast<WT*>(stage + (size_t)(kStages - 1) * kTile);
    {
        const WT* gw = reinterpret_cast<const WT*>(A.w);
        for (int i = tid; i < N * N; i += kPassThreads) sw[i] = gw[i];
    }
    if (INTW) load_phase_tables(A, smtab, tid, kPassThreads);
    __syncthreads();
    if (tid == 0)
        for (i64 j = 0; j < kStages - 1 && j < my_tiles; j++) issue(j);
    ct.template setup<true>(sw, N, l, a, tid, A.gamma);

    const i64 thr_off = tile_off(tid, l, a);
    const i64 s8 = 1ll << tile_phys(8, l, a), s9 = 1ll << tile_phys(9, l, a);
    const i64 s10 = 1ll << tile_phys(10, l, a), s11 = 1ll << tile_phys(11, l, a);
    auto off0 = [&](int r) -> i64 {
        return ((r & 1) ? s8 : 0) + ((r & 2) ? s9 : 0) + ((r & 4) ? s10 : 0) + ((r & 8) ? s11 : 0);
    };
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    WT* const kp = ct.ke;  // written after a tile's first barrier, read after its second
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
        ct.tile(kp, base | A.goff, nF, l, a, warp, lane);  // warps 0 and 1, while the copy lands
        if (!mbar_wait_bounded(&full[s], (unsigned)((j / kStages) & 1))) {
            *s_abort = 1;
            if (A.err) atomicExch(A.err, 1);
        }
        __syncthreads();  // tile landed (or abort), kp visible
        if (*s_abort) break;

        double2 v[kRegs];
#pragma unroll
        for (int r = 0; r < kRegs; r++) v[r] = buf[tslot(lay_index<0>(tid, r))];

        // RX of layer p: L0 -> (L2 ->) L1 (L0 only with SC_L0).  The first
        // exchange's leading barrier orders the reads of the landed tile
        // before the buffer is overwritten.
        rx_regs<GM>(v, m_hi, A.gx, A.c, A.s);
        if (lo_lane >= 0) rx_lane<GM>(v, lo_lane, A.gx, A.c, A.s);
        if (SC == SC_L021) {
            exchange<0, 2>(v, buf, tid, true);
            rx_regs<GM>(v, m_lo, A.gx, A.c, A.s);
            exchange<2, 1>(v, buf, tid, true);
        } else if (SC == SC_L01) {
            exchange<0, 1>(v, buf, tid, true);
        }
        if (SC != SC_L0) rx_regs<GM>(v, m_mid, A.gx, A.c, A.s);

        // Phase of layer p+1 in layout LP (see k_pass).
        {
            WT cb, h0, h1, h2, h3;
            ct.template consts<LP>(kp, tid, cb, h0, h1, h2, h3);
            const double2* qt = ct.qtab + 16 * LP;
            const WT* crg = ct.creg + 16 * LP;
            if (tree) {
                const double2 P = phase_of<WT>(A, smtab, cb);
                phase_base<PH_MUL>(v, P, qt);
                phase_bit(v, 0, zpow<WT>(A, smtab, h0));
                phase_bit(v, 1, zpow<WT>(A, smtab, h1));
                phase_bit(v, 2, zpow<WT>(A, smtab, h2));
                phase_bit(v, 3, zpow<WT>(A, smtab, h3));
            } else {
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    const WT cr = cb + crg[r] + ((r & 1) ? h0 : WT(0)) + ((r & 2) ? h1 : WT(0)) +
                                  ((r & 4) ? h2 : WT(0)) + ((r & 8) ? h3 : WT(0));
                    double2 ph;
                    if (INTW) {
                        ph = int_phase(A, smtab, (int)cr);
                    } else {  // the reference's own argument (src/rzz.cu:146-150)
                        const double S = 2.0 * (double)cr - A.W;
                        double sn, cs;
                        sincos(S * A.gamma / 2, &sn, &cs);
                        ph = make_double2(cs * A.scale, sn * A.scale);
                    }
                    v[r] = cmul(v[r], ph);
                }
            }
        }

        // RX of layer p+1 in the opposite order, back to L0.
        if (SC == SC_L0) {
            rx_regs<GM2>(v, m_hi, A.gx2, A.c, A.s);
            if (lo_lane >= 0) rx_lane<GM2>(v, lo_lane, A.gx2, A.c, A.s);
        } else {
            rx_regs<GM2>(v, m_mid, A.gx2, A.c, A.s);
            if (lo_lane >= 0) rx_lane<GM2>(v, lo_lane, A.gx2, A.c, A.s);
            if (SC == SC_L021) {
                exchange<1, 2>(v, buf, tid, true);
                rx_regs<GM2>(v, m_lo, A.gx2, A.c, A.s);
                exchange<2, 0>(v, buf, tid, true);
            } else {
                exchange<1, 0>(v, buf, tid, true);
            }
            rx_regs<GM2>(v, m_hi, A.gx2, A.c, A.s);
        }
        double2* const p = A.sv + base + thr_off;
#pragma unroll
        for (int r = 0; r < kRegs; r++) __stcs(p + off0(r), v[r]);
    }
    if (*s_abort) {
        // Drain the copies still in flight into this CTA's stages (bounded).
        if (tid == 0)
            for (i64 k = j; k < j + kStages && k < my_tiles; k++)
                mbar_wait_bounded(&full[k % kStages], (unsigned)((k / kStages) & 1));
    }
}

}  // namespace fq
