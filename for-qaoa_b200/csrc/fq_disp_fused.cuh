// fq_disp_fused.cuh -- launch of the fused two-layer pass (k_pass with
// GM2): RX of one layer, the next layer's cost phase and its RX, in one sweep.
#pragma once

#include "fq_launch.cuh"

namespace fq {

template <typename WT, int GM1, int GM2>
inline int fused_launch(fq_ctx* ctx, const PassArgs& A) {
    switch (schedule_for(A.tmask)) {
        case SC_L021: return launch_ldg<WT, PH_MUL, GM1, EX_NONE, true, SC_L021, GM2>(ctx, A);
        case SC_L01: return launch_ldg<WT, PH_MUL, GM1, EX_NONE, true, SC_L01, GM2>(ctx, A);
        default: return launch_ldg<WT, PH_MUL, GM1, EX_NONE, true, SC_L0, GM2>(ctx, A);
    }
}

template <typename WT>
inline int fused_dispatch(fq_ctx* ctx, int gm1, int gm2, const PassArgs& A) {
    FQ_CHECK((gm1 == GM_TAN || gm1 == GM_COT) && (gm2 == GM_TAN || gm2 == GM_COT),
             FQ_ERR_INVALID, "fused pass needs reduced gates (%d, %d)", gm1, gm2);
    if (gm1 == GM_TAN)
        return gm2 == GM_TAN ? fused_launch<WT, GM_TAN, GM_TAN>(ctx, A)
                             : fused_launch<WT, GM_TAN, GM_COT>(ctx, A);
    return gm2 == GM_TAN ? fused_launch<WT, GM_COT, GM_TAN>(ctx, A)
                         : fused_launch<WT, GM_COT, GM_COT>(ctx, A);
}

}  // namespace fq
