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
// The pass uses the full RX formula (src/rx.cu:47-50) with -beta, so the
// inner products are taken on exactly scaled vectors.
//
// 256 threads x 16 amplitudes x 2 vectors in registers, one CTA per SM; the
// layouts, exchanges (one 64 KB buffer per vector) and cut decomposition are
// those of k_pass.
#pragma once

#include "fq_pass.cuh"

namespace fq {

// RX on the register bits of m4 for both vectors; adds Im<w|X_q|v> of each
// rotated qubit q to acc (taken before the rotation; it commutes).
__device__ __forceinline__ void rx_regs_dual(double2 (&v)[kRegs], double2 (&w)[kRegs], unsigned m4,
                                             double c, double s, double& acc) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if ((m4 >> k) & 1u) {
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                if (!((r >> k) & 1)) {
                    const int q = r | (1 << k);
                    acc += (w[r].x * v[q].y - w[r].y * v[q].x) + (w[q].x * v[r].y - w[q].y * v[r].x);
                    rx_pair<GM_FULL>(v[r], v[q], 0.0, c, s);
                    rx_pair<GM_FULL>(w[r], w[q], 0.0, c, s);
                }
            }
        }
    }
}

// The same for a qubit held in lane bit j (each lane adds its own term).
__device__ __forceinline__ void rx_lane_dual(double2 (&v)[kRegs], double2 (&w)[kRegs], int j,
                                             double c, double s, double& acc) {
    const unsigned lm = 1u << j;
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        double2 pv, pw;
        pv.x = __shfl_xor_sync(0xffffffffu, v[r].x, lm);
        pv.y = __shfl_xor_sync(0xffffffffu, v[r].y, lm);
        pw.x = __shfl_xor_sync(0xffffffffu, w[r].x, lm);
        pw.y = __shfl_xor_sync(0xffffffffu, w[r].y, lm);
        acc += w[r].x * pv.y - w[r].y * pv.x;
        const double2 mv = v[r], mw = w[r];
        v[r].x = mv.x * c + pv.y * s;
        v[r].y = mv.y * c - pv.x * s;
        w[r].x = mw.x * c + pw.y * s;
        w[r].y = mw.y * c - pw.x * s;
    }
}

template <int LF, int LT>
__device__ __forceinline__ void exchange_dual(double2 (&v)[kRegs], double2 (&w)[kRegs],
                                              double2* buf, int tid) {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        const int sl = xslot(lay_index<LF>(tid, r));
        buf[sl] = v[r];
        buf[kTile + sl] = w[r];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRegs; r++) {
        const int sl = xslot(lay_index<LT>(tid, r));
        v[r] = buf[sl];
        w[r] = buf[kTile + sl];
    }
}

template <typename WT>
__host__ __device__ inline size_t dual_smem_bytes(int N) {
    return 2 * sizeof(double2) * kTile + sizeof(double) * 16 + sizeof(i64) * 32 +
           sizeof(int) * 24 + sizeof(WT) * (N * N + 32 + 16 + 24 + 16) + 16 + phase_smem_bytes();
}

// PHI: this pass also accumulates dE/dgamma (-Im<w|S|v>, negated on the
// host) and, if A.scale != 0, multiplies both vectors by the conjugate
// phase.  ST: write the vectors back.  Partials: gb[blockIdx] (beta) and
// gg[blockIdx] (gamma).
template <typename WT, bool PHI, int SC, bool ST>
__global__ void __launch_bounds__(kPassThreads, 1)
    k_pass_dual(const PassArgs A, double* gb, double* gg) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double2* buf = reinterpret_cast<double2*>(smraw);
    double* red = reinterpret_cast<double*>(buf + 2 * kTile);  // 16
    i64* offtab = reinterpret_cast<i64*>(red + 16);
    int* fpos = reinterpret_cast<int*>(offtab + 32);
    WT* sw = reinterpret_cast<WT*>(fpos + 24);
    WT* ke = sw + A.N * A.N;
    WT* creg = ke + 32;
    WT* Dm = creg + 16;
    WT* Ru = Dm + 24;
    double2* smtab = reinterpret_cast<double2*>(
        (reinterpret_cast<uintptr_t>(Ru + 16) + 15) & ~(uintptr_t)15);
    const int N = A.N, l = A.l, a = A.a;
    const int nF = N - kTileBits;
    const int nmid = a - l;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr bool CUT = PHI;

    if (tid < 2 * kRegs) {
        const int r = tid & 15, lo = tid < kRegs ? 8 : 4;
        i64 o = 0;
        for (int k = 0; k < 4; k++)
            if ((r >> k) & 1) o += 1ll << tile_phys(lo + k, l, a);
        offtab[tid] = o;
    }
    if (CUT) {
        const WT* gw = reinterpret_cast<const WT*>(A.w);
        for (int i = tid; i < N * N; i += kPassThreads) sw[i] = gw[i];
        if (tid < nF) fpos[tid] = tid < nmid ? l + tid : a + (kTileBits - l) + (tid - nmid);
        if (sizeof(WT) == sizeof(int)) load_phase_tables(A, smtab, tid, kPassThreads);
    }
    __syncthreads();
    if (CUT) {
        if (tid < nF) {
            const int m = fpos[tid];
            WT d = 0;
            for (int u = 0; u < kTileBits; u++) d += sw[m * N + tile_phys(u, l, a)];
            Dm[tid] = d;
        } else if (tid >= 32 && tid < 32 + kTileBits) {
            const int u = tile_phys(tid - 32, l, a);
            WT r = 0;
            for (int i = 0; i < nF; i++) r += sw[u * N + fpos[i]];
            Ru[tid - 32] = r;
        } else if (tid >= 64 && tid < 80) {
            const int r = tid - 64;
            WT c = 0;
            for (int k = 0; k < 4; k++)
                for (int k2 = k + 1; k2 < 4; k2++)
                    if (((r >> k) ^ (r >> k2)) & 1)
                        c += sw[tile_phys(8 + k, l, a) * N + tile_phys(8 + k2, l, a)];
            creg[r] = c;
        }
    }
    WT athr = 0, f0 = 0, f1 = 0, f2 = 0, f3 = 0;
    if (CUT) {
        for (int j = 0; j < 8; j++) {
            const int pj = tile_phys(j, l, a);
            const int tj = (tid >> j) & 1;
            for (int j2 = j + 1; j2 < 8; j2++)
                if (tj ^ ((tid >> j2) & 1)) athr += sw[pj * N + tile_phys(j2, l, a)];
            const WT w0 = sw[pj * N + tile_phys(8, l, a)], w1 = sw[pj * N + tile_phys(9, l, a)];
            const WT w2 = sw[pj * N + tile_phys(10, l, a)], w3 = sw[pj * N + tile_phys(11, l, a)];
            if (tj) {
                athr += w0 + w1 + w2 + w3;
                f0 -= w0;
                f1 -= w1;
                f2 -= w2;
                f3 -= w3;
            } else {
                f0 += w0;
                f1 += w1;
                f2 += w2;
                f3 += w3;
            }
        }
    }
    i64 thr_off = 0, thr_off1 = 0;
    for (int j = 0; j < 8; j++) thr_off |= (i64)((tid >> j) & 1) << tile_phys(j, l, a);
    {
        const int t1 = lay_index<1>(tid, 0);
        for (int j = 0; j < kTileBits; j++)
            if ((t1 >> j) & 1) thr_off1 |= 1ll << tile_phys(j, l, a);
    }
    const unsigned m_hi = (A.tmask >> 8) & 15u, m_mid = (A.tmask >> 4) & 15u, m_lo = A.tmask & 15u;
    const int lo_lane = (SC != SC_L021 && m_lo) ? __ffs(m_lo) - 1 : -1;
    double accb = 0, accg = 0;

    for (i64 T = blockIdx.x; T < A.ntiles; T += gridDim.x) {
        const i64 base = ((T & ((1ll << nmid) - 1)) << l) | ((T >> nmid) << (a + kTileBits - l));
        if (CUT) {
            __syncthreads();
            if (warp == 0) {
                WT h = 0;
                if (lane < nF) {
                    const int m = fpos[lane];
                    const int zm = (int)((base >> m) & 1);
                    if (zm) h += Dm[lane];
                    for (int i = lane + 1; i < nF; i++)
                        if (zm ^ (int)((base >> fpos[i]) & 1)) h += sw[m * N + fpos[i]];
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
                if (lane < kTileBits) {
                    const int u = tile_phys(lane, l, a);
                    WT e = Ru[lane];
                    for (int i = 0; i < nF; i++)
                        if ((base >> fpos[i]) & 1) e -= 2 * sw[u * N + fpos[i]];
                    ke[1 + lane] = e;
                }
                if (lane == 0) ke[0] = h;
            }
            __syncthreads();
        }
        double2* const pv = A.sv + base + thr_off;
        double2* const pw = A.sv2 + base + thr_off;
        double2 v[kRegs], w[kRegs];
#pragma unroll
        for (int r = 0; r < kRegs; r++) {
            v[r] = __ldcs(pv + offtab[r]);
            w[r] = __ldcs(pw + offtab[r]);
        }
        rx_regs_dual(v, w, m_hi, A.c, A.s, accb);
        if (lo_lane >= 0) rx_lane_dual(v, w, lo_lane, A.c, A.s, accb);
        if (SC == SC_L021) {
            exchange_dual<0, 2>(v, w, buf, tid);
            rx_regs_dual(v, w, m_lo, A.c, A.s, accb);
            exchange_dual<2, 1>(v, w, buf, tid);
        } else if (SC == SC_L01) {
            exchange_dual<0, 1>(v, w, buf, tid);
        }
        constexpr int LAY = (SC != SC_L0 && !PHI) ? 1 : 0;
        if (SC != SC_L0) {
            rx_regs_dual(v, w, m_mid, A.c, A.s, accb);
            if (LAY == 0) exchange_dual<1, 0>(v, w, buf, tid);
        }
        if (PHI) {
            WT cbase = ke[0] + athr;
#pragma unroll
            for (int jj = 0; jj < 8; jj++)
                if ((tid >> jj) & 1) cbase += ke[1 + jj];
            const WT g0 = f0 + ke[9], g1 = f1 + ke[10], g2 = f2 + ke[11], g3 = f3 + ke[12];
#pragma unroll
            for (int r = 0; r < kRegs; r++) {
                const WT cr = cbase + creg[r] + ((r & 1) ? g0 : WT(0)) + ((r & 2) ? g1 : WT(0)) +
                              ((r & 4) ? g2 : WT(0)) + ((r & 8) ? g3 : WT(0));
                const double S = 2.0 * (double)cr - A.W;
                accg = fma(w[r].x * v[r].y - w[r].y * v[r].x, S, accg);
                if (A.scale != 0.0) {
                    double2 ph;
                    if (sizeof(WT) == sizeof(int)) {
                        ph = int_phase(A, smtab, (int)cr);
                    } else {
                        double sn, cs;
                        sincos(S * A.gamma / 2, &sn, &cs);
                        ph = make_double2(cs, sn);
                    }
                    // multiply by conj(ph)
                    const double2 a0 = v[r], b0 = w[r];
                    v[r].x = a0.x * ph.x + a0.y * ph.y;
                    v[r].y = a0.y * ph.x - a0.x * ph.y;
                    w[r].x = b0.x * ph.x + b0.y * ph.y;
                    w[r].y = b0.y * ph.x - b0.x * ph.y;
                }
            }
        }
        if (ST) {
            if (LAY == 0) {
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    __stcs(pv + offtab[r], v[r]);
                    __stcs(pw + offtab[r], w[r]);
                }
            } else {
                double2* const qv = A.sv + base + thr_off1;
                double2* const qw = A.sv2 + base + thr_off1;
#pragma unroll
                for (int r = 0; r < kRegs; r++) {
                    __stcs(qv + offtab[kRegs + r], v[r]);
                    __stcs(qw + offtab[kRegs + r], w[r]);
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        accb += __shfl_xor_sync(0xffffffffu, accb, o);
        accg += __shfl_xor_sync(0xffffffffu, accg, o);
    }
    __syncthreads();
    if (lane == 0) {
        red[warp] = accb;
        red[8 + warp] = accg;
    }
    __syncthreads();
    if (tid == 0) {
        double sb = 0, sg = 0;
        for (int k = 0; k < kPassThreads / 32; k++) {
            sb += red[k];
            sg += red[8 + k];
        }
        gb[blockIdx.x] = sb;
        if (PHI) gg[blockIdx.x] = sg;
    }
}

}  // namespace fq
