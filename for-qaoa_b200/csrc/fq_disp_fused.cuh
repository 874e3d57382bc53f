// fq_disp_fused.cuh -- launch of the fused two-layer pass (k_pass with
// GM2): RX of one layer, the next layer's cost phase and its RX, in one sweep.
#pragma once

#include "fq_launch.cuh"
#include "fq_pass_tmaf.cuh"

namespace fq {

// Which fused passes run as TMA pipelines (k_pass_tmaf) instead of k_pass
// (FQ_TMAF): 0 none (default), 1 the strided ones, 2 all.  Measured on B200
// at N=30 p=5: 58.5 layers/s with none, 57.9 with 1, 54.4 with 2 -- the
// fused passes are bound by their arithmetic and barriers, not by the load
// latency the ring hides, and one CTA per SM hides less of that than k_pass
// at two.
inline int tmaf_mode() {
    static int m = -1;
    if (m < 0) {
        const char* e = getenv("FQ_TMAF");
        m = e ? std::max(0, std::min(2, atoi(e))) : 0;
    }
    return m;
}

template <typename WT, int GM1, int GM2, int SC>
inline int launch_tmaf(fq_ctx* ctx, const PassArgs& A, const CUtensorMap& map, TmaGeom G) {
    auto fn = k_pass_tmaf<WT, GM1, GM2, SC>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tmaf_smem_bytes<WT>()));
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->num_sms);
    const int tok = prof_begin(ctx);
    fn<<<(unsigned)grid, kPassThreads, tmaf_smem_bytes<WT>(), ctx->stream>>>(A, map, G);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, pass_kind<PH_MUL, GM1, EX_NONE, true>(),
             pass_bytes<PH_MUL, EX_NONE, true>(A.N));
    ctx->launches++;
    return FQ_OK;
}

template <typename WT, int GM1, int GM2>
inline int fused_launch(fq_ctx* ctx, const PassArgs& A) {
    const int m = tmaf_mode();
    if (m == 2 || (m == 1 && A.l < kTileBits)) {
        alignas(64) CUtensorMap map;
        TmaGeom G;
        if (make_pass_tmap(A, &map, &G)) {
            switch (schedule_for(A.tmask)) {
                case SC_L021: return launch_tmaf<WT, GM1, GM2, SC_L021>(ctx, A, map, G);
                case SC_L01: return launch_tmaf<WT, GM1, GM2, SC_L01>(ctx, A, map, G);
                default: return launch_tmaf<WT, GM1, GM2, SC_L0>(ctx, A, map, G);
            }
        }
    }
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
