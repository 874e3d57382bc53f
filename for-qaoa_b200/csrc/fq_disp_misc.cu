// fq_disp_misc.cu -- the reference-path RX passes (full RX formula of
// src/rx.cu:47-50) and the read-only sweeps (<C> partials, cut diagonal).
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

}  // namespace fq
