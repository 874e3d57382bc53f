// fq_pass_dual.cuh -- the tile pass over two vectors at once, for the
// adjoint (reverse) sweep of the gradient.
//
// The adjoint of E = <psi|C|psi> with respect to the layer angles walks the
// layers backwards carrying psi and the costate lambda (lambda = C psi at
// the end of the circuit), moving both back through the exact inverse of
// each layer (a recompute: no stored intermediate states).  At layer k
//   dE/dbeta_k  =  Im <lambda| sum_q X_q |psi>   (anywhere inside mixer k,
//                                                 since X_q commutes with
//                                                 every RX)
//   dE/dgamma_k = -Im <lambda| S |psi>           (after mixer k is undone;
//                                                 S commutes with the phase)
// A backward layer is the forward layer's passes over (psi, lambda): the
// strided passes undo RX on their qubits, then the contiguous pass undoes RX
// on qubits 0..11, accumulates dE/dgamma_k and applies the inverse phase.
// RX(-beta) runs in the reduced form of the forward engine; the kernel
// tracks the scale that gives the vectors and corrects every inner product
// for it, and the inverse phase restores the true scale.
//
// 256 threads x 16 amplitudes x 2 vectors in registers, one CTA per SM; the
// layouts, exchanges (one 64 KB buffer per vector) and cut decomposition are
// those of k_pass.
#pragma once

#include "fq_pass.cuh"

namespace fq {

// Reduced RX (GM_TAN / GM_COT: the gate divided by its factor f) on the
// register bits of m4 for both vectors.  Before each qubit q is rotated,
// Im<w|X_q|v> is added to acc times sc, the scale that undoes the factors
// 1/f the vectors picked up from the reduced rotations so far (X_q commutes
// with every RX, so the true inner product is the same at any point of the
// mixer); sc gains f^2 with every rotation.
template <int GM>
__device__ __forceinline__ void rx_regs_dual(double2 (&v)[kRegs], double2 (&w)[kRegs], unsigned m4,
                                             double g, double f2, double& sc, double& acc) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if ((m4 >> k) & 1u) {
            double ta = 0, tb = 0;  // two FMA chains
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                if (!((r >> k) & 1)) {
                    const int q = r | (1 << k);
                    ta = fma(w[r].x, v[q].y, ta);
                    ta = fma(-w[r].y, v[q].x, ta);
                    tb = fma(w[q].x, v[r].y, tb);
                    tb = fma(-w[q].y, v[r].x, tb);
                    rx_pair<GM>(v[r], v[q], g, 0.0, 0.0);
                    rx_pair<GM>(w[r], w[q], g, 0.0, 0.0);
                }
            }
            acc = fma(sc, ta + tb, acc);
            sc *= f2;
        }
    }
}

// The same for a qubit held in lane bit j (each lane adds its own term).
template <int GM>
__device__ __forceinline__ void rx_lane_dual(double2 (&v)[kRegs], double2 (&w)[kRegs], int j,
                                             double g, double f2, double& sc, double& acc) {
    const unsigned lm = 1u << j;
    double t = 0;
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        double2 pv, pw;
        pv.x = __shfl_xor_sync(0xffffffffu, v[r].x, lm);
        pv.y = __shfl_xor_sync(0xffffffffu, v[r].y, lm);
        pw.x = __shfl_xor_sync(0xffffffffu, w[r].x, lm);
        pw.y = __shfl_xor_sync(0xffffffffu, w[r].y, lm);
        t = fma(w[r].x, pv.y, t);
        t = fma(-w[r].y, pv.x, t);
        const double2 mv = v[r], mw = w[r];
        if (GM == GM_TAN) {
            v[r].x = fma(g, pv.y, mv.x);
            v[r].y = fma(-g, pv.x, mv.y);
            w[r].x = fma(g, pw.y, mw.x);
            w[r].y = fma(-g, pw.x, mw.y);
        } else {
            v[r].x = fma(g, mv.x, pv.y);
            v[r].y = fma(g, mv.y, -pv.x);
            w[r].x = fma(g, mw.x, pw.y);
            w[r].y = fma(g, mw.y, -pw.x);
        }
    }
    acc = fma(sc, t, acc);
    sc *= f2;
}

template <int LF, int LT>
__device__ __forceinline__ void exchange_dual(double2 (&v)[kRegs], double2 (&w)[kRegs],
                                              double2* buf, int tid, bool wait_readers = true) {
    if (wait_readers) buf_sync<LF, LT>();  // previous readers of buf are done
    {
        double2* const wb = buf + pbase<LF>(tid);
#pragma unroll
        for (int r = 0; r < kRegs; r++) {
            const int sl = pslot(lay_index<LF>(0, r));
            wb[sl] = v[r];
            wb[kXTile + sl] = w[r];
        }
    }
    buf_sync<LF, LT>();
    {
        const double2* const rb = buf + pbase<LT>(tid);
#pragma unroll
        for (int r = 0; r < kRegs; r++) {
            const int sl = pslot(lay_index<LT>(0, r));
            v[r] = rb[sl];
            w[r] = rb[kXTile + sl];
        }
    }
}

// Shared memory: two padded exchange buffers (the weights are staged in
// them while the kernel sets up), then the tables of k_pass.
template <typename WT>
__host__ __device__ inline size_t dual_smem_bytes(int) {
    return 2 * sizeof(double2) * kXTile + PassSmem<WT>::bytes + 24 * sizeof(double);
}

// RX(-beta) in reduced form GM (A.gx = t or u, A.f2 = f^2, A.sc0 = scale of
// the vectors at the pass's start, see rx_regs_dual) on the pass's targets,
// dE/dbeta partials to gb.  PHI: the pass completes its layer's mixer, so it
// also accumulates dE/dgamma (-Im<w|S|v>, negated on the host) into gg and,
// if A.scale != 0, multiplies both vectors by the conjugate phase times
// A.scale = f^N, which returns them to their true scale.  GM2 != GM_NONE (a
// fused pass, PHI only): then RX(-beta) of the layer before (GM2, A.gx2,
// A.f2b) on the same targets, from scale 1, its dE/dbeta partials to gb2.
// With the reverse pass order alternating from layer to layer, the last
// pass of one layer and the first of the next share a tile geometry, so two
// sweeps become one.  The phase and dE/dgamma are taken in the layout the
// first rounds end in (L1, or L0 with SC_L0).  ST: write the vectors back.
// The next tile of both vectors is prefetched into L2 while the current one
// is computed (one CTA per SM cannot hide the HBM latency of its loads
// otherwise).
//
// TURN: the turnaround of the gradient, three sweeps in one: the forward
// circuit's last pass (RX(+beta) of the last layer, reduced form GM2 with
// A.gx2, on the tile's targets), the costate lambda = C psi of the final
// state with <C> (Kahan sums to gg), and the reverse sweep's first pass
// (RX(-beta), GM with A.gx, from scale A.sc0, dE/dbeta partials to gb).
// Only psi is read (the state before the last forward pass); both vectors
// are written as the reverse sweep's first pass would write them: 32 B
// per amplitude instead of 32 + 48 + 64.
template <typename WT, bool PHI, int SC, bool ST, int GM, int GM2 = GM_NONE, bool TURN = false>
__global__ void __launch_bounds__(kPassThreads, 1)
    k_pass_dual(const PassArgs A, double* gb, double* gg, double* gb2) {
    extern __shared__ __align__(16) unsigned char smraw[];
    using SM = PassSmem<WT>;
    double2* buf = reinterpret_cast<double2*>(smraw);
    unsigned char* const sm = smraw + 2 * sizeof(double2) * kXTile;
    const CutTables<WT> ct(sm);
    double2* smtab = reinterpret_cast<double2*>(sm + SM::smtab);
    double* red = reinterpret_cast<double*>(sm + SM::bytes);  // 24: the three partials
    const int N = A.N, l = A.l, a = A.a;
    const int nF = N - kTileBits;
    const int nmid = a - l;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr bool CUT = PHI || TURN;
    constexpr bool INTW = sizeof(WT) == sizeof(int);
    constexpr bool FUSED = !TURN && GM2 != GM_NONE;
    static_assert(PHI || !FUSED, "a fused adjoint pass carries its layer's phase");
    static_assert(!(PHI && TURN), "the turnaround pass carries no phase");
    constexpr int LP = SC == SC_L0 ? 0 : 1;  // layout after the first rounds
    constexpr int LAY = (FUSED || TURN) ? 0 : LP;  // layout of the stores

    WT* sw = reinterpret_cast<WT*>(buf);  // N*N weights while setting up
    if (CUT) {
        const WT* gw = reinterpret_cast<const WT*>(A.w);
        for (int i = tid; i < N * N; i += kPassThreads) sw[i] = gw[i];
        if (INTW) load_phase_tables(A, smtab, tid, kPassThreads);
    }
    __syncthreads();
    if (CUT) ct.template setup<true>(sw, N, l, a, tid, A.gamma);
    __syncthreads();  // the weights in buf are dead from here on

    const i64 thr_off = tile_off(tid, l, a);
    const i64 thr_off1 = tile_off(lay_index<1>(tid, 0), l, a);
    const i64 s8 = 1ll << tile_phys(8, l, a), s9 = 1ll << tile_phys(9, l, a);
    const i64 s10 = 1ll << tile_phys(10, l, a), s11 = 1ll << tile_phys(11, l, a);
    const i64 s4 = 1ll << tile_phys(4, l, a), s5 = 1ll << tile_phys(5, l, a);
    const i64 s6 = 1ll << tile_phys(6, l, a), s7 = 1ll << tile_phys(7, l, a);
    auto tile_base = [&](i64 T) -> i64 {
        return ((T & ((1ll << nmid) - 1)) << l) | ((T >> nmid) << (a + kTileBits - l));
    };
    const bool contiguous = (l == kTileBits);
    const int pf_step = l < 3 ? l : 3;
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    double accb = 0, accg = 0, accb2 = 0;
    double ecomp = 0;  // Kahan compensation of <C> (TURN, in accg)
    // Fused passes end in layout L0 and copy the next tile of both vectors
    // into the buffer early, as k_pass's fused passes do (on B200 for K_26,
    // p=10: 22.25-22.27 against 22.45-22.56 ms of adjoint passes per
    // evaluation, A/B in one call).
    constexpr bool CPF = FUSED && ST && (SC != SC_L0);
    bool have_next = false;
    const double g = A.gx, f2 = A.f2;

    int par = 0;
    for (i64 T = blockIdx.x; T < A.ntiles; T += gridDim.x, par ^= 1) {
        const i64 base = tile_base(T);
        double2 v[kRegs], w[kRegs];
        if (CPF && have_next) {  // copied in during the previous tile (see below)
            asm volatile("cp.async.wait_group 0;" ::: "memory");
            const double2* const own = buf + pbase<0>(tid);
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                v[r] = own[pslot(lay_index<0>(0, r))];
                w[r] = own[kXTile + pslot(lay_index<0>(0, r))];
            }
        } else {
            const i64 o = opaque(base + thr_off);
            const i64 b8 = opaque(s8), b9 = opaque(s9), b10 = opaque(s10), b11 = opaque(s11);
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                v[r] = __ldcs(A.sv + o + offr(r, b8, b9, b10, b11));
                if (!TURN) w[r] = __ldcs(A.sv2 + o + offr(r, b8, b9, b10, b11));
            }
        }
        if (T + gridDim.x < A.ntiles) {
            const i64 b2 = tile_base(T + gridDim.x);
            if (contiguous) {
                if (tid < (TURN ? 1 : 2))
                    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                                     (tid ? A.sv2 : A.sv) + b2),
                                 "r"((unsigned)(kTile * sizeof(double2)))
                                 : "memory");
            } else {
                for (int j = tid; j < (1 << (kTileBits - pf_step)); j += kPassThreads) {
                    const i64 o = b2 + tile_off(j << pf_step, l, a);
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(A.sv + o) : "memory");
                    if (!TURN) asm volatile("prefetch.global.L2 [%0];" ::"l"(A.sv2 + o) : "memory");
                }
            }
        }
        WT* const kp = ct.ke + 32 * par;
        if (CUT) ct.tile(kp, base | A.goff, nF, l, a, warp, lane);  // read after the exchanges' barriers
        // The thread index re-read in every tile: the exchange addresses
        // derived from it are recomputed (a few integer ops) instead of being
        // hoisted out of the loop, where they would take registers.
        int xt;
        asm volatile("mov.u32 %0, %%tid.x;" : "=r"(xt));
        // First rounds: L0 -> (L2 ->) L1, or L0 only with SC_L0.  The
        // previous tile's readers of buf are done once every thread is past
        // this tile's first barrier (the leading barrier of its first
        // exchange, a block barrier).
        double sc = A.sc0;
        if constexpr (TURN) {
            // The forward's last pass on psi alone: L0 -> (L2 ->) L1.
            const double gf = A.gx2;
            rx_regs<GM2>(v, m_hi, gf, 0.0, 0.0);
            if (lo_lane >= 0) rx_lane<GM2>(v, lo_lane, gf, 0.0, 0.0);
            if (SC == SC_L021) {
                exchange<0, 2>(v, buf, xt, true);
                rx_regs<GM2>(v, m_lo, gf, 0.0, 0.0);
                exchange<2, 1>(v, buf, xt, true);
            } else if (SC == SC_L01) {
                exchange<0, 1>(v, buf, xt, true);
            }
            if (SC != SC_L0) rx_regs<GM2>(v, m_mid, gf, 0.0, 0.0);
            // The final state: <C> and lambda = C psi (cut constants of layout LP).
            if (SC == SC_L0) __syncthreads();  // kp written by warps 0 and 1
            WT cbase, g0, g1, g2, g3;
            ct.template consts<LP>(kp, tid, cbase, g0, g1, g2, g3);
            const WT* crg = ct.creg + 16 * LP;
            double te = 0;
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                const double c = (double)cr;
                te = fma(fma(v[r].x, v[r].x, v[r].y * v[r].y), c, te);
                w[r] = make_double2(c * v[r].x, c * v[r].y);
            }
            const double y = te - ecomp;
            const double t2 = accg + y;
            ecomp = (t2 - accg) - y;
            accg = t2;
            // The reverse sweep's first pass, back to L0.
            if (SC != SC_L0) rx_regs_dual<GM>(v, w, m_mid, g, f2, sc, accb);
            if (lo_lane >= 0) rx_lane_dual<GM>(v, w, lo_lane, g, f2, sc, accb);
            // No leading barriers (see exchange): each thread writes the v
            // slots it has just read, and the w slots were last read in the
            // previous tile, before this tile's first barrier.
            if (SC == SC_L021) {
                exchange_dual<1, 2>(v, w, buf, xt, false);
                rx_regs_dual<GM>(v, w, m_lo, g, f2, sc, accb);
                exchange_dual<2, 0>(v, w, buf, xt, false);
            } else if (SC == SC_L01) {
                exchange_dual<1, 0>(v, w, buf, xt, false);
            }
            rx_regs_dual<GM>(v, w, m_hi, g, f2, sc, accb);
        } else {
        rx_regs_dual<GM>(v, w, m_hi, g, f2, sc, accb);
        if (lo_lane >= 0) rx_lane_dual<GM>(v, w, lo_lane, g, f2, sc, accb);
        // A fused pass's previous tile ended by reading the thread's own L0
        // slots, which this exchange writes: no leading barrier (see
        // exchange); other passes ended in L1 and need it.
        if (SC == SC_L021) {
            exchange_dual<0, 2>(v, w, buf, xt, !FUSED);
            rx_regs_dual<GM>(v, w, m_lo, g, f2, sc, accb);
            exchange_dual<2, 1>(v, w, buf, xt, false);
        } else if (SC == SC_L01) {
            exchange_dual<0, 1>(v, w, buf, xt, !FUSED);
        }
        if (SC != SC_L0) rx_regs_dual<GM>(v, w, m_mid, g, f2, sc, accb);
        if constexpr (PHI) {
            if (SC == SC_L0) __syncthreads();  // kp written by warps 0 and 1
            WT cbase, g0, g1, g2, g3;
            ct.template consts<LP>(kp, tid, cbase, g0, g1, g2, g3);
            const WT* crg = ct.creg + 16 * LP;
            const double2* qt = ct.qtab + 16 * LP;
            double tg = 0;
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                const double S = 2.0 * (double)cr - A.W;
                tg = fma(w[r].x * v[r].y - w[r].y * v[r].x, S, tg);
            }
            accg = fma(sc, tg, accg);
            if (A.scale != 0.0) {
                if (INTW ? A.nhi > 0 : A.tree != 0) {  // product tree (see k_pass)
                    double2 P = phase_of<WT>(A, smtab, cbase);
                    if (INTW) P = make_double2(P.x * A.scale, P.y * A.scale);
                    // Two stages, to keep few values live next to the 32
                    // amplitudes: the conjugate of L[r & 3] * Q_r with
                    // L = P * {1, E0, E1, E0 E1} on every slot, then that of
                    // H[r >> 2], H = {1, E2, E3, E2 E3}.
                    {
                        const double2 E0 = zpow<WT>(A, smtab, g0), E1 = zpow<WT>(A, smtab, g1);
                        const double2 L[4] = {P, cmul(P, E0), cmul(P, E1),
                                              cmul(cmul(P, E0), E1)};
#pragma unroll
                        for (int r = 0; r < kRegs; r++) {
                            const double2 ph = cmul(L[r & 3], qt[r]);
                            const double2 c = make_double2(ph.x, -ph.y);
                            v[r] = cmul(v[r], c);
                            w[r] = cmul(w[r], c);
                        }
                    }
                    {
                        const double2 E2 = zpow<WT>(A, smtab, g2), E3 = zpow<WT>(A, smtab, g3);
                        const double2 H[4] = {make_double2(1.0, 0.0), E2, E3, cmul(E2, E3)};
#pragma unroll
                        for (int r = 4; r < kRegs; r++) {
                            const double2 c = make_double2(H[r >> 2].x, -H[r >> 2].y);
                            v[r] = cmul(v[r], c);
                            w[r] = cmul(w[r], c);
                        }
                    }
                } else {  // one phase per amplitude: global table or sincos
#pragma unroll
                    for (int r = 0; r < kRegs; r++) {
                        const WT cr = cbase + crg[r] + ((r & 1) ? g0 : WT(0)) +
                                      ((r & 2) ? g1 : WT(0)) + ((r & 4) ? g2 : WT(0)) +
                                      ((r & 8) ? g3 : WT(0));
                        double2 ph;
                        if (INTW) {
                            ph = int_phase(A, smtab, (int)cr);
                        } else {
                            double sn, cs;
                            sincos((2.0 * (double)cr - A.W) * A.gamma / 2, &sn, &cs);
                            ph = make_double2(cs, sn);
                        }
                        const double2 c = make_double2(ph.x * A.scale, -ph.y * A.scale);
                        v[r] = cmul(v[r], c);
                        w[r] = cmul(w[r], c);
                    }
                }
            }
            if constexpr (FUSED) {
                // The earlier layer's rounds in the opposite order, back to
                // L0 (a single target among tile bits 0..3 is the same lane
                // bit in L1 as in L0).
                double sc2 = 1.0;
                const double g2x = A.gx2, f2b = A.f2b;
                if (SC != SC_L0) rx_regs_dual<GM2>(v, w, m_mid, g2x, f2b, sc2, accb2);
                if (lo_lane >= 0) rx_lane_dual<GM2>(v, w, lo_lane, g2x, f2b, sc2, accb2);
                if (SC == SC_L021) {
                    exchange_dual<1, 2>(v, w, buf, xt, false);
                    rx_regs_dual<GM2>(v, w, m_lo, g2x, f2b, sc2, accb2);
                    exchange_dual<2, 0>(v, w, buf, xt, false);
                } else if (SC == SC_L01) {
                    exchange_dual<1, 0>(v, w, buf, xt, false);
                }
                if (CPF) {
                    // Each thread's L0 slots are its own until the next
                    // tile's first exchange: copy its part of the next tile
                    // of both vectors there now.
                    have_next = T + gridDim.x < A.ntiles;
                    if (have_next) {
                        const i64 o = opaque(tile_base(T + gridDim.x) + thr_off);
                        const i64 b8 = opaque(s8), b9 = opaque(s9), b10 = opaque(s10),
                                  b11 = opaque(s11);
                        const unsigned dst =
                            (unsigned)__cvta_generic_to_shared(buf + pbase<0>(tid));
#pragma unroll
                        for (int r = 0; r < kRegs; r++) {
                            const unsigned d = dst + (unsigned)(16 * pslot(lay_index<0>(0, r)));
                            const i64 off = o + offr(r, b8, b9, b10, b11);
                            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d),
                                         "l"(A.sv + off)
                                         : "memory");
                            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                                             d + (unsigned)(16 * kXTile)),
                                         "l"(A.sv2 + off)
                                         : "memory");
                        }
                        asm volatile("cp.async.commit_group;" ::: "memory");
                    }
                }
                rx_regs_dual<GM2>(v, w, m_hi, g2x, f2b, sc2, accb2);
            }
        }
        }  // !TURN
        if (ST) {
            if (LAY == 0) {
                const i64 o = opaque(base + thr_off);
                const i64 b8 = opaque(s8), b9 = opaque(s9), b10 = opaque(s10), b11 = opaque(s11);
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    __stcs(A.sv + o + offr(r, b8, b9, b10, b11), v[r]);
                    __stcs(A.sv2 + o + offr(r, b8, b9, b10, b11), w[r]);
                }
            } else {
                const i64 o = opaque(base + thr_off1);
                const i64 b4 = opaque(s4), b5 = opaque(s5), b6 = opaque(s6), b7 = opaque(s7);
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    __stcs(A.sv + o + offr(r, b4, b5, b6, b7), v[r]);
                    __stcs(A.sv2 + o + offr(r, b4, b5, b6, b7), w[r]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        accb += __shfl_xor_sync(0xffffffffu, accb, o);
        accg += __shfl_xor_sync(0xffffffffu, accg, o);
        accb2 += __shfl_xor_sync(0xffffffffu, accb2, o);
    }
    __syncthreads();
    if (lane == 0) {
        red[warp] = accb;
        red[8 + warp] = accg;
        red[16 + warp] = accb2;
    }
    __syncthreads();
    if (tid == 0) {
        double sb = 0, sg = 0, sb2 = 0;
        for (int k = 0; k < kPassThreads / 32; k++) {
            sb += red[k];
            sg += red[8 + k];
            sb2 += red[16 + k];
        }
        gb[blockIdx.x] = sb;
        if (PHI || TURN) gg[blockIdx.x] = sg;
        if (FUSED) gb2[blockIdx.x] = sb2;
    }
}

}  // namespace fq
