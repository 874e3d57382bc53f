// fq_disp_phase.cu -- passes with a cost phase: the first pass of a layer
// (phase + RX on the pass's tile qubits, any tile geometry) and the
// reference-path cost layer alone (fq_cost_phase).
#include "fq_launch.cuh"

namespace fq {

template <typename WT, int PH, int GM, int SC>
static int phase_launch_sc(fq_ctx* ctx, const PassArgs& A) {
    return launch_ldg<WT, PH, GM, EX_NONE, true, SC>(ctx, A);
}

template <typename WT, int PH, int GM>
static int phase_launch(fq_ctx* ctx, const PassArgs& A) {
    if constexpr (GM == GM_NONE) {
        return phase_launch_sc<WT, PH, GM, SC_L0>(ctx, A);
    } else {
        switch (schedule_for(A.tmask)) {
            case SC_L021: return phase_launch_sc<WT, PH, GM, SC_L021>(ctx, A);
            case SC_L01: return phase_launch_sc<WT, PH, GM, SC_L01>(ctx, A);
            default: return phase_launch_sc<WT, PH, GM, SC_L0>(ctx, A);
        }
    }
}

template <typename WT>
static int phase_pass(fq_ctx* ctx, int ph, int gm, const PassArgs& A) {
    if (ph == PH_INIT) {
        if (gm == GM_TAN) return phase_launch<WT, PH_INIT, GM_TAN>(ctx, A);
        if (gm == GM_COT) return phase_launch<WT, PH_INIT, GM_COT>(ctx, A);
        return phase_launch<WT, PH_INIT, GM_NONE>(ctx, A);
    }
    if (gm == GM_TAN) return phase_launch<WT, PH_MUL, GM_TAN>(ctx, A);
    if (gm == GM_COT) return phase_launch<WT, PH_MUL, GM_COT>(ctx, A);
    return phase_launch<WT, PH_MUL, GM_NONE>(ctx, A);
}

int dispatch_phase_pass(fq_ctx* ctx, bool integer, int ph, int gm, const PassArgs& A) {
    FQ_CHECK(ph == PH_INIT || ph == PH_MUL, FQ_ERR_INVALID, "bad phase mode %d", ph);
    FQ_CHECK(gm == GM_NONE || gm == GM_TAN || gm == GM_COT, FQ_ERR_INVALID, "bad gate mode %d",
             gm);
    return integer ? phase_pass<int>(ctx, ph, gm, A) : phase_pass<double>(ctx, ph, gm, A);
}

}  // namespace fq
