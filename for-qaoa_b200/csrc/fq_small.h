// fq_small.h -- job descriptor of k_small_jobs (fq_small.cuh): one whole
// QAOA instance of up to 12 qubits per CTA.
#pragma once

#include "fq_common.cuh"

namespace fq {

constexpr int kSmallMaxQubits = 12;
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

__host__ __device__ inline size_t small_smem_bytes(int nmax) {
    const size_t n = (size_t)1 << nmax;
    return 2 * n * sizeof(double2) + n * sizeof(double) +
           sizeof(double) * (kSmallMaxQubits * kSmallMaxQubits + kSmallThreads);
}

}  // namespace fq
