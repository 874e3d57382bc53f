// fq_launch.cuh -- host-side launch of the tile passes (k_pass, k_pass_tma):
// schedule selection, TMA tensor maps, profiling brackets.
// The kernel variants are instantiated in a few translation units
// (fq_disp_*.cu) so they compile in parallel; fq_engine.cu calls the
// dispatch_* entry points declared at the end.
#pragma once

#include <cudaTypedefs.h>
#include <stdlib.h>

#include <algorithm>

#include "fq_ctx.h"
#include "fq_pass.cuh"
#include "fq_pass_tma.cuh"

namespace fq {

// Kind of a pass for profiling, and the HBM bytes it must move.
template <int PH, int GM, int EX, bool ST>
inline int pass_kind() {
    if ((EX == EX_ENERGY || EX == EX_COSTATE) && !ST) return FQ_KIND_EXPECT;
    if (EX == EX_DIAG) return FQ_KIND_EXPECT;
    if (GM == GM_FULL) return FQ_KIND_RX;
    if (GM == GM_NONE) return FQ_KIND_COST;
    if (PH == PH_INIT) return FQ_KIND_INIT_PASS;
    return PH != PH_NONE ? FQ_KIND_PHASE_PASS : FQ_KIND_MIXER_PASS;
}

template <int PH, int EX, bool ST>
inline double pass_bytes(int N) {
    const double n = (double)(1ull << N);
    const bool load = (PH != PH_INIT) && (ST || EX == EX_ENERGY || EX == EX_COSTATE);
    return n * ((load ? 16.0 : 0.0) + (ST ? 16.0 : 0.0) + (EX == EX_DIAG ? 8.0 : 0.0) +
                (EX == EX_COSTATE ? 16.0 : 0.0));
}

// Strided tiles with 128-byte rows run as paired CTAs (k_pass with PAIR:
// the two tiles that differ in physical bit 3 at once, so DRAM sees 256-byte
// rows).  Measured on B200 at N=30, p=5 (A/B in one call): 59.8-60.1
// layers/s with every such pass paired, 59.5-59.7 with the strided RX pass
// on the TMA pipeline instead.
// Strided tiles with rows of 2, 4 or 8 amplitudes run paired (k_pass PAIR):
// rows of 16 and more are DRAM-friendly alone.  Rows of 2 and 4 (N = 23,
// 22, 32) paired: 0.527 against 0.542 ms per N=23 circuit (p=5), 233
// against 242 ms per N=32 circuit (p=3), A/B in one call.
inline bool pair_ok(const PassArgs& A) { return A.l >= 1 && A.l <= 3 && A.a > A.l && A.ntiles >= 2; }

template <typename WT, int PH, int GM, int EX, bool ST, int SC, int GM2 = GM_NONE,
          bool PAIR = false>
inline int launch_ldg_as(fq_ctx* ctx, const PassArgs& A) {
    auto fn = k_pass<WT, PH, GM, EX, ST, SC, GM2, PAIR>;
    const size_t smem = pass_smem_bytes<WT>(A.N, PAIR);
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const i64 units = PAIR ? A.ntiles / 2 : A.ntiles;
    const i64 grid = std::min<i64>(units, (i64)(PAIR ? 1 : ctx->ctas_per_sm) * ctx->num_sms);
    const int tok = prof_begin(ctx);
    fn<<<(unsigned)grid, PAIR ? 2 * kPassThreads : kPassThreads, smem, ctx->stream>>>(A);
    FQ_CUDA(cudaGetLastError());
    ctx->last_grid = (int)grid;
    prof_end(ctx, tok, pass_kind<PH, GM, EX, ST>(), pass_bytes<PH, EX, ST>(A.N));
    ctx->launches++;
    return FQ_OK;
}

template <typename WT, int PH, int GM, int EX, bool ST, int SC, int GM2 = GM_NONE>
inline int launch_ldg(fq_ctx* ctx, const PassArgs& A) {
    if (pair_ok(A)) return launch_ldg_as<WT, PH, GM, EX, ST, SC, GM2, true>(ctx, A);
    return launch_ldg_as<WT, PH, GM, EX, ST, SC, GM2, false>(ctx, A);
}

inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
        else
            cudaGetLastError();
    }
    return fn;
}

// The TMA pipeline k_pass_tma runs the read-write RX passes (no cost phase)
// over strided tiles with rows of 16 or more amplitudes.  Contiguous tiles
// and tiles with 128-byte rows (paired) run on k_pass, whose per-thread
// loads from two CTAs per SM measured faster there on B200 at N=30 (the
// contiguous RX pass: 6.0 ms against 6.9 ms on the TMA pipeline); passes
// with a phase always do.
inline bool tma_for(int ph, const PassArgs& A) {
    return ph == PH_NONE && A.l >= 4 && A.l < kTileBits;
}

// The state as a tensor of float64 whose innermost dimension is one 128-byte
// row of 8 amplitudes; the box is one tile (4096 amplitudes) in tile order.
// Returns false for tiles with rows narrower than 8 amplitudes.
inline bool make_pass_tmap(const PassArgs& A, CUtensorMap* map, TmaGeom* G) {
    auto enc = tmap_encoder();
    if (!enc || !A.sv || ((uintptr_t)A.sv & 127) != 0) return false;
    // The tensor spans the amplitudes in A.sv: 2^12 per tile (A.N can be
    // larger for a shard of a bigger state, see PassArgs::goff).
    const int N = kTileBits + __builtin_ctzll((unsigned long long)A.ntiles);
    const int l = A.l, a = A.a, k = kTileBits - l;
    cuuint64_t dims[5];
    cuuint64_t strides[4];
    cuuint32_t box[5];
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    int rank;
    if (l == kTileBits) {
        rank = 3;
        G->kind = TG_CONTIG;
        dims[0] = 16; dims[1] = 256; dims[2] = 1ull << (N - 11);
        strides[0] = 128; strides[1] = 128ull * 256;
        box[0] = 16; box[1] = 256; box[2] = 2;
    } else if (l >= 4 && l <= 11) {
        rank = 5;
        G->kind = TG_ROWS;
        dims[0] = 16; dims[1] = 1ull << (l - 3); dims[2] = 1ull << (a - l);
        dims[3] = 1ull << k; dims[4] = 1ull << (N - a - k);
        strides[0] = 128; strides[1] = 16ull << l; strides[2] = 16ull << a;
        strides[3] = 16ull << (a + k);
        box[0] = 16; box[1] = 1u << (l - 3); box[2] = 1; box[3] = 1u << k; box[4] = 1;
    } else if (l == 3) {
        rank = 5;
        G->kind = TG_ROWS8;
        dims[0] = 16; dims[1] = 1ull << (a - 3); dims[2] = 32; dims[3] = 16;
        dims[4] = 1ull << (N - a - 9);
        strides[0] = 128; strides[1] = 16ull << a; strides[2] = 16ull << (a + 5);
        strides[3] = 16ull << (a + 9);
        box[0] = 16; box[1] = 1; box[2] = 32; box[3] = 16; box[4] = 1;
    } else {
        return false;
    }
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, (void*)A.sv, dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <typename WT, int PH, int GM, int EX, int SC>
inline int launch_tma(fq_ctx* ctx, const PassArgs& A, const CUtensorMap& map, TmaGeom G) {
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->num_sms);
    const int tok = prof_begin(ctx);
    auto fn = k_pass_tma<WT, PH, GM, EX, SC>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tma_pass_smem_bytes<WT>(kMaxQubits)));
    fn<<<(unsigned)grid, kPassThreads, tma_pass_smem_bytes<WT>(A.N), ctx->stream>>>(A, map, G);
    FQ_CUDA(cudaGetLastError());
    ctx->last_grid = (int)grid;
    prof_end(ctx, tok, pass_kind<PH, GM, EX, true>(), pass_bytes<PH, EX, true>(A.N));
    ctx->launches++;
    return FQ_OK;
}

// Launch one pass with the round schedule its target mask needs.  Passes
// without RX (cost phase, <C>, cut diagonal) use the L0 schedule.  RX passes
// that read and write the state run as TMA pipelines where tma_for() and
// the tile geometry allow; every other pass uses k_pass.
template <typename WT, int PH, int GM, int EX, bool ST>
inline int launch_pass(fq_ctx* ctx, const PassArgs& A) {
    if constexpr (ST && PH != PH_INIT && EX != EX_DIAG && EX != EX_COSTATE) {
        if (tma_for(PH, A)) {
            alignas(64) CUtensorMap map;
            TmaGeom G;
            if (make_pass_tmap(A, &map, &G)) {
                if constexpr (GM == GM_NONE) {
                    return launch_tma<WT, PH, GM, EX, SC_L0>(ctx, A, map, G);
                } else {
                    switch (schedule_for(A.tmask)) {
                        case SC_L021: return launch_tma<WT, PH, GM, EX, SC_L021>(ctx, A, map, G);
                        case SC_L01: return launch_tma<WT, PH, GM, EX, SC_L01>(ctx, A, map, G);
                        default: return launch_tma<WT, PH, GM, EX, SC_L0>(ctx, A, map, G);
                    }
                }
            }
        }
    }
    if constexpr (GM == GM_NONE) {
        return launch_ldg<WT, PH, GM, EX, ST, SC_L0>(ctx, A);
    } else {
        switch (schedule_for(A.tmask)) {
            case SC_L021: return launch_ldg<WT, PH, GM, EX, ST, SC_L021>(ctx, A);
            case SC_L01: return launch_ldg<WT, PH, GM, EX, ST, SC_L01>(ctx, A);
            default: return launch_ldg<WT, PH, GM, EX, ST, SC_L0>(ctx, A);
        }
    }
}

// Grid (and <C> partial count) of the tile pass launched last.
inline int pass_grid(fq_ctx* ctx, const PassArgs&, int, bool) { return ctx->last_grid; }

// ---- dispatch entry points (one translation unit each) -------------------

// Layer pass with a cost phase (ph = PH_INIT or PH_MUL) and RX on A.tmask
// (gm = GM_TAN or GM_COT), or the cost phase alone (gm = GM_NONE).
int dispatch_phase_pass(fq_ctx* ctx, bool integer, int ph, int gm, const PassArgs& A);
// RX on A.tmask without a phase (reduced gates), optionally with <C>.
int dispatch_rx_tan(fq_ctx* ctx, bool integer, bool energy, const PassArgs& A);
int dispatch_rx_cot(fq_ctx* ctx, bool integer, bool energy, const PassArgs& A);
// RX with the full formula of src/rx.cu:47-50 (reference-path kernels).
int dispatch_rx_full(fq_ctx* ctx, const PassArgs& A);
// Fused pass: RX (gm1, A.gx) on A.tmask, the next layer's phase, RX (gm2,
// A.gx2) on A.tmask (k_pass with GM2); one translation unit per weight type.
int dispatch_fused_int(fq_ctx* ctx, int gm1, int gm2, const PassArgs& A);
int dispatch_fused_fp(fq_ctx* ctx, int gm1, int gm2, const PassArgs& A);
inline int dispatch_fused(fq_ctx* ctx, bool integer, int gm1, int gm2, const PassArgs& A) {
    return integer ? dispatch_fused_int(ctx, gm1, gm2, A) : dispatch_fused_fp(ctx, gm1, gm2, A);
}
// Adjoint pass that completes a layer's mixer (k_pass_dual with PHI):
// RX(-beta) (gm, A.gx) on A.tmask, dE/dgamma and the inverse phase, then
// with gm2 != GM_NONE the earlier layer's RX(-beta) (gm2, A.gx2) on A.tmask.
// Partials: gb (beta), gg (gamma), gb2 (the earlier layer's beta).
// store = false (gm2 == GM_NONE only) leaves both vectors unwritten.
int dispatch_dual_phase_int(fq_ctx* ctx, int gm, int gm2, const PassArgs& A, double* gb,
                            double* gg, double* gb2, bool store = true);
int dispatch_dual_phase_fp(fq_ctx* ctx, int gm, int gm2, const PassArgs& A, double* gb,
                           double* gg, double* gb2, bool store = true);
// The gradient's turnaround (k_pass_dual with TURN): the forward's last pass
// (gmf, A.gx2), lambda = C psi with <C> (partials to ge), and the reverse
// sweep's first pass (gm, A.gx; dE/dbeta partials to gb), in one sweep.
int dispatch_dual_turn_int(fq_ctx* ctx, int gm, int gmf, const PassArgs& A, double* gb,
                           double* ge);
int dispatch_dual_turn_fp(fq_ctx* ctx, int gm, int gmf, const PassArgs& A, double* gb,
                          double* ge);
// Read-only sweeps: <C> partials or the cut diagonal (diag != 0).
int dispatch_readonly(fq_ctx* ctx, bool integer, bool diag, const PassArgs& A);
// <C> partials and the costate A.sv2 = C * A.sv.
int dispatch_costate(fq_ctx* ctx, bool integer, const PassArgs& A);

inline int dispatch_rx(fq_ctx* ctx, bool integer, int gm, bool energy, const PassArgs& A) {
    if (gm == GM_TAN) return dispatch_rx_tan(ctx, integer, energy, A);
    if (gm == GM_COT) return dispatch_rx_cot(ctx, integer, energy, A);
    return dispatch_rx_full(ctx, A);
}

}  // namespace fq
