// fq_disp_dual.cuh -- launches of the adjoint pass k_pass_dual (both vectors
// of the reverse sweep in one sweep).
#pragma once

#include <algorithm>

#include "fq_launch.cuh"
#include "fq_pass_dual.cuh"

namespace fq {

template <typename WT, bool PHI, int SC, int GM, int GM2, bool TURN = false, bool ST = true>
inline int dual_launch(fq_ctx* ctx, const PassArgs& A, double* gb, double* gg, double* gb2) {
    auto fn = k_pass_dual<WT, PHI, SC, ST, GM, GM2, TURN>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dual_smem_bytes<WT>(kMaxQubits)));
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->num_sms);
    const int tok = prof_begin(ctx);
    fn<<<(unsigned)grid, kPassThreads, dual_smem_bytes<WT>(A.N), ctx->stream>>>(A, gb, gg, gb2);
    FQ_CUDA(cudaGetLastError());
    // The turnaround reads one vector and writes two; ST = false reads two.
    prof_end(ctx, tok, FQ_KIND_ADJOINT, (TURN ? 48.0 : ST ? 64.0 : 32.0) * (double)(1ull << A.N));
    ctx->launches++;
    return FQ_OK;
}

template <typename WT, bool PHI, int GM, int GM2, bool ST = true>
inline int dual_sc(fq_ctx* ctx, const PassArgs& A, double* gb, double* gg, double* gb2) {
    switch (schedule_for(A.tmask)) {
        case SC_L021: return dual_launch<WT, PHI, SC_L021, GM, GM2, false, ST>(ctx, A, gb, gg, gb2);
        case SC_L01: return dual_launch<WT, PHI, SC_L01, GM, GM2, false, ST>(ctx, A, gb, gg, gb2);
        default: return dual_launch<WT, PHI, SC_L0, GM, GM2, false, ST>(ctx, A, gb, gg, gb2);
    }
}

// The pass that completes layer k's mixer: dE/dgamma_k and the inverse
// phase, then (gm2 != GM_NONE) layer k-1's RX(-beta) on the same targets.
// store = false (layer 0's completing pass, gm2 == GM_NONE: the sweep's
// last pass, whose vectors nothing reads) leaves the vectors unwritten.
template <typename WT>
inline int dual_phase_dispatch(fq_ctx* ctx, int gm, int gm2, const PassArgs& A, double* gb,
                               double* gg, double* gb2, bool store) {
    FQ_CHECK((gm == GM_TAN || gm == GM_COT) &&
                 (gm2 == GM_NONE || gm2 == GM_TAN || gm2 == GM_COT),
             FQ_ERR_INVALID, "adjoint pass needs reduced gates (%d, %d)", gm, gm2);
    FQ_CHECK(store || gm2 == GM_NONE, FQ_ERR_INVALID, "a fused adjoint pass stores its vectors");
    if (!store)
        return gm == GM_TAN ? dual_sc<WT, true, GM_TAN, GM_NONE, false>(ctx, A, gb, gg, gb2)
                            : dual_sc<WT, true, GM_COT, GM_NONE, false>(ctx, A, gb, gg, gb2);
    if (gm == GM_TAN) {
        if (gm2 == GM_NONE) return dual_sc<WT, true, GM_TAN, GM_NONE>(ctx, A, gb, gg, gb2);
        if (gm2 == GM_TAN) return dual_sc<WT, true, GM_TAN, GM_TAN>(ctx, A, gb, gg, gb2);
        return dual_sc<WT, true, GM_TAN, GM_COT>(ctx, A, gb, gg, gb2);
    }
    if (gm2 == GM_NONE) return dual_sc<WT, true, GM_COT, GM_NONE>(ctx, A, gb, gg, gb2);
    if (gm2 == GM_TAN) return dual_sc<WT, true, GM_COT, GM_TAN>(ctx, A, gb, gg, gb2);
    return dual_sc<WT, true, GM_COT, GM_COT>(ctx, A, gb, gg, gb2);
}

// The turnaround pass (k_pass_dual with TURN): the forward's last pass
// (gmf, A.gx2), lambda = C psi with <C> (partials to ge) and the reverse
// sweep's first pass (gm, A.gx, dE/dbeta partials to gb), in one sweep.
template <typename WT>
inline int dual_turn_dispatch(fq_ctx* ctx, int gm, int gmf, const PassArgs& A, double* gb,
                              double* ge) {
    FQ_CHECK((gm == GM_TAN || gm == GM_COT) && (gmf == GM_TAN || gmf == GM_COT), FQ_ERR_INVALID,
             "turnaround pass needs reduced gates (%d, %d)", gm, gmf);
    auto sc = [&](auto gtag, auto ftag) -> int {
        constexpr int G = decltype(gtag)::value, F = decltype(ftag)::value;
        switch (schedule_for(A.tmask)) {
            case SC_L021: return dual_launch<WT, false, SC_L021, G, F, true>(ctx, A, gb, ge, nullptr);
            case SC_L01: return dual_launch<WT, false, SC_L01, G, F, true>(ctx, A, gb, ge, nullptr);
            default: return dual_launch<WT, false, SC_L0, G, F, true>(ctx, A, gb, ge, nullptr);
        }
    };
    using T = std::integral_constant<int, GM_TAN>;
    using C = std::integral_constant<int, GM_COT>;
    if (gm == GM_TAN) return gmf == GM_TAN ? sc(T(), T()) : sc(T(), C());
    return gmf == GM_TAN ? sc(C(), T()) : sc(C(), C());
}

}  // namespace fq
