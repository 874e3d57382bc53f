// fq_disp_misc.cu -- the reference-path RX passes (full RX formula of
// src/rx.cu:47-50), the read-only sweeps (<C> partials, cut diagonal) and
// the self-test of the bounded-wait failure path.
#include "fq_launch.cuh"

namespace fq {

int dispatch_rx_full(fq_ctx* ctx, const PassArgs& A) {
    return launch_pass<int, PH_NONE, GM_FULL, EX_NONE, true>(ctx, A);
}

int dispatch_readonly(fq_ctx* ctx, bool integer, bool diag, const PassArgs& A) {
    if (diag) {
        if (integer) return launch_pass<int, PH_NONE, GM_NONE, EX_DIAG, false>(ctx, A);
        return launch_pass<double, PH_NONE, GM_NONE, EX_DIAG, false>(ctx, A);
    }
    if (integer) return launch_pass<int, PH_NONE, GM_NONE, EX_ENERGY, false>(ctx, A);
    return launch_pass<double, PH_NONE, GM_NONE, EX_ENERGY, false>(ctx, A);
}

int dispatch_costate(fq_ctx* ctx, bool integer, const PassArgs& A) {
    if (integer) return launch_pass<int, PH_NONE, GM_NONE, EX_COSTATE, false>(ctx, A);
    return launch_pass<double, PH_NONE, GM_NONE, EX_COSTATE, false>(ctx, A);
}

// One warp waits, with the bounded wait of the TMA pipelines (a shorter
// poll bound: max_polls), on an mbarrier that nothing arrives at: the wait
// gives up, the kernel records flag 2 and returns (fq_ctx_selftest_wait).
__global__ void k_selftest_wait(int* err, long long max_polls) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    const bool done = mbar_wait_polls(&bar, 0, max_polls);
    if (!done && threadIdx.x == 0) atomicExch(err, 2);
}

}  // namespace fq

extern "C" int fq_ctx_selftest_wait(fq_ctx* ctx) {
    using namespace fq;
    FQ_TRY(validate_ctx(ctx));
    k_selftest_wait<<<1, 32, 0, ctx->stream>>>(ctx->d_err, 1ll << 16);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}
