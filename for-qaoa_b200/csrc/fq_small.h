// fq_small.h -- job descriptor of k_small_jobs (fq_small.cuh): one whole
// QAOA instance of up to 12 qubits per CTA, of 13..15 qubits per cluster of
// 2^(N-12) CTAs.
#pragma once

#include "fq_common.cuh"

namespace fq {

constexpr int kSmallMaxQubits = 12;     // qubits held by one CTA
constexpr int kSmallJobMaxQubits = 15;  // qubits of a job (a cluster of up to 8 CTAs)
constexpr int kSmallThreads = 256;

enum { SJ_ENERGY = 1, SJ_GRAD = 2, SJ_STATE = 4 };

struct SmallJob {
    int N, P, flags, pad;
    const double* w;       // N*N symmetric weights (device)
    const double* gammas;  // P (device)
    const double* betas;   // P (device)
    double* out;           // [0] <C>, [1..P] dE/dgamma, [1+P..2P] dE/dbeta (device)
    double2* state;        // final forward state (SJ_STATE), 2^N (device)
};

// Shared memory of a CTA holding 2^nl amplitudes: psi, lambda, the cut
// values, the weights of a job of up to kSmallJobMaxQubits qubits, the
// block-sum scratch and the cluster's exchange words.
// Size class of an N-qubit job: 0 for one CTA (N <= 12), else the log2 of
// its cluster's CTAs.
constexpr int kSmallClasses = kSmallJobMaxQubits - kSmallMaxQubits + 1;
__host__ __device__ inline int small_class(int N) {
    return N <= kSmallMaxQubits ? 0 : N - kSmallMaxQubits;
}

__host__ __device__ inline size_t small_smem_bytes(int nl) {
    const size_t n = (size_t)1 << nl;
    return 2 * n * sizeof(double2) + n * sizeof(double) +
           sizeof(double) * (kSmallJobMaxQubits * kSmallJobMaxQubits + kSmallThreads + 8);
}

}  // namespace fq
