// fq_disp_phase.cu -- passes with a cost phase: the layer pass of the fused
// engine (phase + RX on tile bits 0..11, schedule L0 -> L2 -> L1) and the
// reference-path cost layer alone (fq_cost_phase).
#include "fq_launch.cuh"

namespace fq {

template <typename WT, int PH, int GM>
static int phase_launch(fq_ctx* ctx, const PassArgs& A) {
    constexpr int SC = GM == GM_NONE ? SC_L0 : SC_L021;
    FQ_CHECK(GM == GM_NONE || schedule_for(A.tmask) == SC_L021, FQ_ERR_INVALID,
             "phase pass with gates needs two or more targets among tile bits 0..3");
    if (PH == PH_MUL && tma_for(PH)) {
        alignas(64) CUtensorMap map;
        TmaGeom G;
        if (make_pass_tmap(A, &map, &G)) return launch_tma<WT, PH, GM, EX_NONE, SC>(ctx, A, map, G);
    }
    return launch_ldg<WT, PH, GM, EX_NONE, true, SC>(ctx, A);
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
