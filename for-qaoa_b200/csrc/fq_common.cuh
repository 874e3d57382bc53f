// fq_common.cuh -- shared definitions of the FOR-QAOA B200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "forqaoa.h"

namespace fq {

typedef long long i64;
typedef unsigned long long u64;

// Thread-local message for the last failing call (fq_last_error()).
void set_error(const char* fmt, ...);

#define FQ_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            ::fq::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                            cudaGetErrorString(e_));                               \
            return FQ_ERR_CUDA;                                                    \
        }                                                                          \
    } while (0)

#define FQ_CHECK(cond, code, ...)                                                  \
    do {                                                                           \
        if (!(cond)) {                                                             \
            ::fq::set_error(__VA_ARGS__);                                          \
            return (code);                                                         \
        }                                                                          \
    } while (0)

#define FQ_TRY(expr)                                                               \
    do {                                                                           \
        int s_ = (expr);                                                           \
        if (s_ != FQ_OK) return s_;                                                \
    } while (0)

// Largest state this build accepts: 2^33 amplitudes (128 GiB) fits HBM.
constexpr int kMaxQubits = 33;
// Integer phase tables are used while the cut range has at most this many
// values; wider ranges fall back to a per-amplitude FP64 sincos.
constexpr int kMaxPhaseTable = 1 << 16;

}  // namespace fq
