// fq_small.cuh -- whole QAOA instances of up to 12 qubits inside one CTA,
// and of 13..15 qubits inside a cluster of 2, 4 or 8 CTAs.
//
// One CTA per instance holds psi (2^N complex128), the costate lambda and
// the cut values of all 2^N basis states in shared memory (160 KB at N=12)
// and runs the forward circuit, <C> and, on request, the adjoint gradient
// without touching HBM except for its inputs and results.  A launch takes a
// batch of independent instances (one per CTA), which is how small requests
// are served: many of them per launch instead of one launch sequence each.
// Above 12 qubits an instance takes a cluster of 2^CB CTAs (CB = N - 12):
// CTA rank r of the cluster holds the 2^12 amplitudes whose top CB qubits
// read r; the phase and the rotations of qubits 0..11 stay in the CTA, the
// rotations of the top CB qubits read the partner CTA's half through
// distributed shared memory, and the sums are added over the cluster in
// rank order.
// Conventions are the reference's (cost phase exp(+i*gamma*S/2), RX(beta)
// with the formula of src/rx.cu:47-50, launch-control amplitude
// pow(1/sqrt(2), N)); the adjoint is the one of fq_pass_dual.cuh.
#pragma once

#include <cooperative_groups.h>

#include "fq_small.h"

namespace fq {

// Fixed-order block sum (same bits for the same inputs).
__device__ __forceinline__ double small_block_sum(double v, double* sh) {
    __syncthreads();
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = kSmallThreads / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// The block sum, then (CB > 0) the sum of the cluster's block sums in rank
// order, valid in rank 0 (the CTA that writes the job's outputs).
template <int CB>
__device__ __forceinline__ double small_sum(double v, double* sh, double* xch) {
    double s = small_block_sum(v, sh);
    if constexpr (CB > 0) {
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        if (threadIdx.x == 0) cl.map_shared_rank(xch, 0)[cl.block_rank()] = s;
        cl.sync();
        s = 0;
        if (cl.block_rank() == 0)
            for (int r = 0; r < (1 << CB); r++) s += xch[r];
        cl.sync();  // xch is free for the next sum
    }
    return s;
}

// RX (full formula) with cos c, sin s of angle/2 on every qubit of x.
__device__ __forceinline__ void small_mixer(double2* x, int N, double c, double s) {
    const int half = 1 << (N - 1);
    for (int q = 0; q < N; q++) {
        for (int k = threadIdx.x; k < half; k += kSmallThreads) {
            const int up = ((k >> q) << (q + 1)) | (k & ((1 << q) - 1));
            const int lo = up + (1 << q);
            const double2 a = x[up], b = x[lo];
            x[up] = make_double2(a.x * c + b.y * s, a.y * c - b.x * s);
            x[lo] = make_double2(a.y * s + b.x * c, -a.x * s + b.y * c);
        }
        __syncthreads();
    }
}

// The same RX on the cluster's CB qubits (above the CTA's 2^12 amplitudes):
// the pair of amplitude k is amplitude k of the CTA whose rank differs in
// the qubit's bit.  Every CTA reads its partner's values after a cluster
// barrier (all earlier writes done), computes its own new values in
// registers, and writes them after a second one (all partner reads done).
template <int CB>
__device__ __forceinline__ void small_mixer_cluster(double2* x, double c, double s) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    constexpr int kPer = (1 << kSmallMaxQubits) / kSmallThreads;
#pragma unroll 1
    for (int j = 0; j < CB; j++) {
        const bool up = !((rank >> j) & 1);
        const double2* px = cl.map_shared_rank(x, rank ^ (1 << j));
        cl.sync();
        double2 t[kPer];
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const int k = threadIdx.x + i * kSmallThreads;
            const double2 a = up ? x[k] : px[k], b = up ? px[k] : x[k];  // (up, lo)
            t[i] = up ? make_double2(a.x * c + b.y * s, a.y * c - b.x * s)
                      : make_double2(a.y * s + b.x * c, -a.x * s + b.y * c);
        }
        cl.sync();
#pragma unroll
        for (int i = 0; i < kPer; i++) x[threadIdx.x + i * kSmallThreads] = t[i];
    }
    __syncthreads();
}

template <int CB>
__global__ void __launch_bounds__(kSmallThreads) k_small_jobs(const SmallJob* jobs, int njobs) {
    namespace cg = cooperative_groups;
    const int job = (int)blockIdx.x >> CB;
    if (job >= njobs) return;  // uniform across a cluster
    const int rank = CB > 0 ? (int)cg::this_cluster().block_rank() : 0;
    const SmallJob J = jobs[job];
    extern __shared__ __align__(16) unsigned char smraw[];
    // N local qubits; the cluster's CB qubits above them are the rank's bits.
    const int N = J.N, NL = N - CB, P = J.P, n = 1 << NL;
    const int zhi = rank << NL;  // global index of local amplitude 0
    double2* psi = reinterpret_cast<double2*>(smraw);
    double2* lam = psi + n;
    double* cz = reinterpret_cast<double*>(lam + n);
    double* w = cz + n;
    double* sh = w + kSmallJobMaxQubits * kSmallJobMaxQubits;
    double* xch = sh + kSmallThreads;
    for (int i = threadIdx.x; i < N * N; i += kSmallThreads) w[i] = J.w[i];
    __syncthreads();
    double Wtot = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) Wtot += w[i * N + j];
    for (int zl = threadIdx.x; zl < n; zl += kSmallThreads) {
        const int z = zl | zhi;
        double c = 0;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (((z >> i) ^ (z >> j)) & 1) c += w[i * N + j];
        cz[zl] = c;
    }
    __syncthreads();
    const double amp0 = pow(1. / sqrt(2.), N);  // src/rzz.cu:26-28
    for (int p = 0; p < P; p++) {
        const double g = J.gammas[p];
        for (int z = threadIdx.x; z < n; z += kSmallThreads) {
            double sn, cs;
            sincos((2.0 * cz[z] - Wtot) * g / 2, &sn, &cs);
            if (p == 0) {
                psi[z] = make_double2(cs * amp0, sn * amp0);
            } else {
                const double2 v = psi[z];
                psi[z] = make_double2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
            }
        }
        __syncthreads();
        const double c = cos(J.betas[p] / 2), s = sin(J.betas[p] / 2);
        small_mixer(psi, NL, c, s);
        if constexpr (CB > 0) small_mixer_cluster<CB>(psi, c, s);
    }
    if (J.flags & SJ_STATE)
        for (int z = threadIdx.x; z < n; z += kSmallThreads) J.state[z | zhi] = psi[z];
    double e = 0;
    for (int z = threadIdx.x; z < n; z += kSmallThreads)
        e = fma(fma(psi[z].x, psi[z].x, psi[z].y * psi[z].y), cz[z], e);
    e = small_sum<CB>(e, sh, xch);
    if (threadIdx.x == 0 && rank == 0) J.out[0] = e;
    if (J.flags & SJ_GRAD) {
        for (int z = threadIdx.x; z < n; z += kSmallThreads)
            lam[z] = make_double2(cz[z] * psi[z].x, cz[z] * psi[z].y);
        __syncthreads();
        const int half = n >> 1;
        for (int k = P - 1; k >= 0; k--) {
            // dE/dbeta_k = Im <lam| sum_q X_q |psi>; a pair across the cluster
            // is counted by the CTA that holds its upper half.
            double gb = 0;
            for (int q = 0; q < NL; q++)
                for (int t = threadIdx.x; t < half; t += kSmallThreads) {
                    const int up = ((t >> q) << (q + 1)) | (t & ((1 << q) - 1));
                    const int lo = up + (1 << q);
                    gb += (lam[up].x * psi[lo].y - lam[up].y * psi[lo].x) +
                          (lam[lo].x * psi[up].y - lam[lo].y * psi[up].x);
                }
            if constexpr (CB > 0) {
                cg::cluster_group cl = cg::this_cluster();
                cl.sync();  // every CTA's psi and lam are final
                for (int j = 0; j < CB; j++) {
                    if ((rank >> j) & 1) continue;
                    const double2* pp = cl.map_shared_rank(psi, rank ^ (1 << j));
                    const double2* pl = cl.map_shared_rank(lam, rank ^ (1 << j));
                    for (int t = threadIdx.x; t < n; t += kSmallThreads) {
                        const double2 lu = lam[t], pu = psi[t], ll = pl[t], plo = pp[t];
                        gb += (lu.x * plo.y - lu.y * plo.x) + (ll.x * pu.y - ll.y * pu.x);
                    }
                }
            }
            gb = small_sum<CB>(gb, sh, xch);
            if (threadIdx.x == 0 && rank == 0) J.out[1 + P + k] = gb;
            const double c = cos(J.betas[k] / 2), s = -sin(J.betas[k] / 2);
            small_mixer(psi, NL, c, s);
            small_mixer(lam, NL, c, s);
            if constexpr (CB > 0) {
                small_mixer_cluster<CB>(psi, c, s);
                small_mixer_cluster<CB>(lam, c, s);
            }
            // dE/dgamma_k = -Im <lam| S |psi>
            double gg = 0;
            for (int z = threadIdx.x; z < n; z += kSmallThreads)
                gg = fma(lam[z].x * psi[z].y - lam[z].y * psi[z].x, 2.0 * cz[z] - Wtot, gg);
            gg = small_sum<CB>(gg, sh, xch);
            if (threadIdx.x == 0 && rank == 0) J.out[1 + k] = -gg;
            if (k > 0) {
                const double g = J.gammas[k];
                for (int z = threadIdx.x; z < n; z += kSmallThreads) {
                    double sn, cs;
                    sincos((2.0 * cz[z] - Wtot) * g / 2, &sn, &cs);
                    const double2 a = psi[z], b = lam[z];
                    psi[z] = make_double2(a.x * cs + a.y * sn, a.y * cs - a.x * sn);
                    lam[z] = make_double2(b.x * cs + b.y * sn, b.y * cs - b.x * sn);
                }
                __syncthreads();
            }
        }
    }
    // No CTA of a cluster leaves while a partner may still read its memory.
    if constexpr (CB > 0) cg::this_cluster().sync();
}

}  // namespace fq
