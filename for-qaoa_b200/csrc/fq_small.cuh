// fq_small.cuh -- whole QAOA instances of up to 12 qubits inside one CTA.
//
// One CTA per instance holds psi (2^N complex128), the costate lambda and
// the cut values of all 2^N basis states in shared memory (160 KB at N=12)
// and runs the forward circuit, <C> and, on request, the adjoint gradient
// without touching HBM except for its inputs and results.  A launch takes a
// batch of independent instances (one per CTA), which is how small requests
// are served: many of them per launch instead of one launch sequence each.
// Conventions are the reference's (cost phase exp(+i*gamma*S/2), RX(beta)
// with the formula of src/rx.cu:47-50, launch-control amplitude
// pow(1/sqrt(2), N)); the adjoint is the one of fq_pass_dual.cuh.
#pragma once

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

__global__ void __launch_bounds__(kSmallThreads) k_small_jobs(const SmallJob* jobs, int njobs) {
    if ((int)blockIdx.x >= njobs) return;
    const SmallJob J = jobs[blockIdx.x];
    extern __shared__ __align__(16) unsigned char smraw[];
    const int N = J.N, P = J.P, n = 1 << N;
    double2* psi = reinterpret_cast<double2*>(smraw);
    double2* lam = psi + n;
    double* cz = reinterpret_cast<double*>(lam + n);
    double* w = cz + n;
    double* sh = w + kSmallMaxQubits * kSmallMaxQubits;
    for (int i = threadIdx.x; i < N * N; i += kSmallThreads) w[i] = J.w[i];
    __syncthreads();
    double Wtot = 0;
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) Wtot += w[i * N + j];
    for (int z = threadIdx.x; z < n; z += kSmallThreads) {
        double c = 0;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (((z >> i) ^ (z >> j)) & 1) c += w[i * N + j];
        cz[z] = c;
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
        small_mixer(psi, N, cos(J.betas[p] / 2), sin(J.betas[p] / 2));
    }
    if (J.flags & SJ_STATE)
        for (int z = threadIdx.x; z < n; z += kSmallThreads) J.state[z] = psi[z];
    double e = 0;
    for (int z = threadIdx.x; z < n; z += kSmallThreads)
        e = fma(fma(psi[z].x, psi[z].x, psi[z].y * psi[z].y), cz[z], e);
    e = small_block_sum(e, sh);
    if (threadIdx.x == 0) J.out[0] = e;
    if (!(J.flags & SJ_GRAD)) return;
    for (int z = threadIdx.x; z < n; z += kSmallThreads)
        lam[z] = make_double2(cz[z] * psi[z].x, cz[z] * psi[z].y);
    __syncthreads();
    const int half = n >> 1;
    for (int k = P - 1; k >= 0; k--) {
        // dE/dbeta_k = Im <lam| sum_q X_q |psi>
        double gb = 0;
        for (int q = 0; q < N; q++)
            for (int t = threadIdx.x; t < half; t += kSmallThreads) {
                const int up = ((t >> q) << (q + 1)) | (t & ((1 << q) - 1));
                const int lo = up + (1 << q);
                gb += (lam[up].x * psi[lo].y - lam[up].y * psi[lo].x) +
                      (lam[lo].x * psi[up].y - lam[lo].y * psi[up].x);
            }
        gb = small_block_sum(gb, sh);
        if (threadIdx.x == 0) J.out[1 + P + k] = gb;
        const double c = cos(J.betas[k] / 2), s = -sin(J.betas[k] / 2);
        small_mixer(psi, N, c, s);
        small_mixer(lam, N, c, s);
        // dE/dgamma_k = -Im <lam| S |psi>
        double gg = 0;
        for (int z = threadIdx.x; z < n; z += kSmallThreads)
            gg = fma(lam[z].x * psi[z].y - lam[z].y * psi[z].x, 2.0 * cz[z] - Wtot, gg);
        gg = small_block_sum(gg, sh);
        if (threadIdx.x == 0) J.out[1 + k] = -gg;
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

}  // namespace fq
