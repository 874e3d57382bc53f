// fq_noalloc.cu -- <C> of a device state for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: their device memory is owned by
// another allocator (a framework's caching pool, or a serving engine that
// reserves the whole HBM up front and hands out slices), or they run in a
// latency-critical loop where cudaMalloc's implicit device synchronisation
// is not acceptable.  fq_expectation_noalloc serves them: it takes only the
// state (already in device memory, owned by the caller), the host graph and
// a stream, and keeps all of its scratch -- the graph's weights, per-CTA
// partial sums and the result word -- in one fixed file-scope device array.
// It calls no allocating routine and needs no fq_ctx.
//
// The array is kNoAllocScratchBytes (32 KiB) and every GPU that loads the
// library holds it until the process exits.  Every call on a device shares
// it and it keeps the last call's contents; all of it is rewritten before
// it is read, so nothing needs clearing, but calls that overlap on the GPU
// (different streams, or different host threads on one device) race on it
// and must be serialised by the caller.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "fq_ctx.h"
#include "fq_pass.cuh"

namespace fq {
namespace {

constexpr size_t kNoAllocScratchBytes = 32 * 1024;
constexpr size_t kNaWeightsOff = 0;                       // N*N weights (<= 8712 B)
constexpr size_t kNaPartialOff = 9 * 1024;                // per-CTA partials
constexpr int kNaMaxPartials = (int)((kNoAllocScratchBytes - kNaPartialOff - 256) / 8);
constexpr size_t kNaResultOff = kNoAllocScratchBytes - 256;  // result word

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array, looked up once per device.  In host
// code the array's name is only a stand-in for the symbol, never a device
// address, so the address comes from cudaGetSymbolAddress.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

int scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        FQ_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_addr[dev] = p;
    }
    *out = (unsigned char*)g_scratch_addr[dev];
    return FQ_OK;
}

// <C> of a small state (N < 12): one CTA, fixed-order reduction.
__global__ void k_na_small(const double2* sv, int N, const double* w, double* out) {
    __shared__ double sh[256];
    double acc = 0;
    for (int b = threadIdx.x; b < (1 << N); b += 256) {
        double cz = 0;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (((b >> i) ^ (b >> j)) & 1) cz += w[i * N + j];
        const double2 v = sv[b];
        acc = fma(fma(v.x, v.x, v.y * v.y), cz, acc);
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

// Fixed-order sum of the per-CTA partials.
__global__ void k_na_reduce(const double* partial, int n, double* out) {
    __shared__ double sh[256];
    double s = 0;
    for (int i = threadIdx.x; i < n; i += 256) s += partial[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

template <typename WT>
int launch_na_pass(const PassArgs& A, int grid, cudaStream_t st) {
    auto fn = k_pass<WT, PH_NONE, GM_NONE, EX_ENERGY, false, SC_L0>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pass_smem_bytes<WT>(kMaxQubits)));
    fn<<<grid, kPassThreads, pass_smem_bytes<WT>(A.N), st>>>(A);
    FQ_CUDA(cudaGetLastError());
    return FQ_OK;
}

}  // namespace
}  // namespace fq

using namespace fq;

extern "C" int fq_expectation_noalloc(const void* sv, int N, const double* graph_upper,
                                      double* energy, void* stream) {
    FQ_CHECK(sv != nullptr && ((uintptr_t)sv & 15) == 0, FQ_ERR_INVALID,
             "state pointer null or not 16-byte aligned");
    FQ_CHECK(graph_upper != nullptr && energy != nullptr, FQ_ERR_INVALID, "null argument");
    FQ_CHECK(N >= 2 && N <= kMaxQubits, FQ_ERR_INVALID,
             "N=%d outside [2, %d]: the fixed scratch holds at most %d x %d weights", N,
             kMaxQubits, kMaxQubits, kMaxQubits);
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    FQ_CUDA(cudaGetDevice(&dev));
    FQ_CHECK(dev >= 0 && dev < kMaxDevices, FQ_ERR_UNSUPPORTED, "device %d beyond %d", dev,
             kMaxDevices);
    unsigned char* scratch = nullptr;
    FQ_TRY(scratch_address(dev, &scratch));

    // Weights on the stack (no heap): integer path when every weight is an
    // integer of modest size (exact cut values), FP64 otherwise.
    double wd[kMaxQubits * kMaxQubits];
    int wi[kMaxQubits * kMaxQubits];
    bool integral = N >= kTileBits;
    long long absum = 0;
    for (int i = 0; i < N * N; i++) {
        wd[i] = 0;
        wi[i] = 0;
    }
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++) {
            const double w = graph_upper[i * N + j];
            FQ_CHECK(isfinite(w), FQ_ERR_INVALID, "non-finite weight at (%d,%d)", i, j);
            wd[i * N + j] = wd[j * N + i] = w;
            if (w != rint(w) || fabs(w) > (double)(1 << 20)) {
                integral = false;
            } else {
                wi[i * N + j] = wi[j * N + i] = (int)w;
                absum += (long long)fabs(w);
            }
        }
    integral = integral && absum < (1ll << 30);
    const size_t wbytes = (size_t)N * N * (integral ? sizeof(int) : sizeof(double));
    FQ_CUDA(cudaMemcpyAsync(scratch + kNaWeightsOff, integral ? (const void*)wi : (const void*)wd,
                            wbytes, cudaMemcpyHostToDevice, st));
    double* result = (double*)(scratch + kNaResultOff);
    if (N < kTileBits) {
        k_na_small<<<1, 256, 0, st>>>((const double2*)sv, N,
                                      (const double*)(scratch + kNaWeightsOff), result);
        FQ_CUDA(cudaGetLastError());
    } else {
        int nsm = 0;
        FQ_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        PassArgs A;
        memset(&A, 0, sizeof(A));
        A.sv = (double2*)sv;
        A.w = scratch + kNaWeightsOff;
        A.partial = (double*)(scratch + kNaPartialOff);
        A.ntiles = 1ll << (N - kTileBits);
        A.N = N;
        A.l = kTileBits;
        A.a = kTileBits;
        A.ntab = 1;
        A.scale = 1.0;
        const int grid = (int)std::min<i64>(A.ntiles, std::min(2 * nsm, kNaMaxPartials));
        if (integral)
            FQ_TRY(launch_na_pass<int>(A, grid, st));
        else
            FQ_TRY(launch_na_pass<double>(A, grid, st));
        k_na_reduce<<<1, 256, 0, st>>>(A.partial, grid, result);
        FQ_CUDA(cudaGetLastError());
    }
    FQ_CUDA(cudaMemcpyAsync(energy, result, sizeof(double), cudaMemcpyDeviceToHost, st));
    FQ_CUDA(cudaStreamSynchronize(st));
    return FQ_OK;
}
