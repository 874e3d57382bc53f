// fq_engine.cu -- fused QAOA engine and the reference-path cost / RX entry
// points, all built on the streaming tile pass (fq_pass.cuh).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <cudaTypedefs.h>

#include "fq_ctx.h"
#include "fq_pass.cuh"
#include "fq_pass_tma.cuh"

namespace fq {

// ---------------------------------------------------------------- kernels --

// Phase of every integer cut value c in [cmin, cmin + n): scale *
// (cos, sin)(S * gamma / 2), S = 2c - W, the same double argument the
// reference forms from its exact integer sum (src/rzz.cu:146).
__global__ void k_phase_table(double2* tab, int cmin, int n, long long W, double gamma,
                              double scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double S = (double)(2ll * (cmin + i) - W);
        double sn, cs;
        sincos(S * gamma / 2, &sn, &cs);
        tab[i] = make_double2(cs * scale, sn * scale);
    }
}

// Two-level phase table of the engine: tab[j] = exp(i*gamma*j) for j < 32,
// tab[32 + h] = scale * (cos, sin)(S * gamma / 2) with S = 2(cmin + 32h) - W.
__global__ void k_phase_table2(double2* tab, int cmin, int nhi, long long W, double gamma,
                               double scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double sn, cs;
    if (i < kPhaseLo) {
        sincos(gamma * (double)i, &sn, &cs);
        tab[i] = make_double2(cs, sn);
    } else if (i < kPhaseLo + nhi) {
        const double S = (double)(2ll * (cmin + 32ll * (i - kPhaseLo)) - W);
        sincos(S * gamma / 2, &sn, &cs);
        tab[i] = make_double2(cs * scale, sn * scale);
    }
}

// Deterministic sum of n partials into out[0]: fixed strided split and a
// fixed tree, so the same inputs always give the same bits.
__global__ void k_reduce_partials(const double* partial, int n, double* out) {
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

struct Perm {
    int p[kMaxQubits];
};

__global__ void k_permute(const double2* __restrict__ src, double2* __restrict__ dst, int N,
                          Perm P) {
    const u64 n = 1ull << N;
    for (u64 x = blockIdx.x * (u64)blockDim.x + threadIdx.x; x < n;
         x += (u64)gridDim.x * blockDim.x) {
        u64 y = 0;
        for (int b = 0; b < N; b++) y |= ((x >> b) & 1ull) << P.p[b];
        dst[y] = src[x];
    }
}

// Small states (N < 12, at most 2048 amplitudes): one CTA, the reference's
// per-amplitude pair-order sum (src/rzz.cu:127-156) on a symmetric FP64
// weight matrix.
__global__ void k_cost_small(double2* sv, int N, double angle, const double* w, int first,
                             double amp) {
    for (int b = threadIdx.x; b < (1 << N); b += blockDim.x) {
        double sum = 0;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++) {
                const double wij = w[i * N + j];
                if (wij != 0) sum += (((b >> i) ^ (b >> j)) & 1) ? wij : -wij;
            }
        double sn, cs;
        sincos(sum * angle / 2, &sn, &cs);
        if (first) {
            sv[b] = make_double2(cs * amp, sn * amp);
        } else {
            const double2 in = sv[b];
            sv[b] = make_double2(in.x * cs - in.y * sn, in.x * sn + in.y * cs);
        }
    }
}

struct Targets {
    int t[kMaxQubits];
};

// src/rx.cu:32-53 applied target by target over a small state (one CTA).
__global__ void k_rx_small(double2* sv, int N, Targets T, int nt, double c, double s) {
    for (int g = 0; g < nt; g++) {
        const int t = T.t[g];
        for (int k = threadIdx.x; k < (1 << (N - 1)); k += blockDim.x) {
            const int up = ((k >> t) << (t + 1)) | (k & ((1 << t) - 1));
            const int lo = up + (1 << t);
            const double2 q0 = sv[up], q1 = sv[lo];
            sv[up] = make_double2(q0.x * c + q1.y * s, q0.y * c - q1.x * s);
            sv[lo] = make_double2(q0.y * s + q1.x * c, -q0.x * s + q1.y * c);
        }
        __syncthreads();
    }
}

// <C> or the cut diagonal of a small state (one CTA).
__global__ void k_cut_small(const double2* sv, int N, const double* w, double* energy,
                            double* diag) {
    __shared__ double sh[256];
    double acc = 0;
    for (int b = threadIdx.x; b < (1 << N); b += blockDim.x) {
        double cz = 0;
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (((b >> i) ^ (b >> j)) & 1) cz += w[i * N + j];
        if (diag) diag[b] = cz;
        if (energy) {
            const double2 v = sv[b];
            acc = fma(fma(v.x, v.x, v.y * v.y), cz, acc);
        }
    }
    if (energy) {
        sh[threadIdx.x] = acc;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) energy[0] = sh[0];
    }
}

// ------------------------------------------------------------ pass launch --

// Kind of a pass for profiling, and the HBM bytes it must move.
template <int PH, int GM, int EX, bool ST>
static int pass_kind() {
    if (EX == EX_ENERGY && !ST) return FQ_KIND_EXPECT;
    if (EX == EX_DIAG) return FQ_KIND_EXPECT;
    if (GM == GM_FULL) return FQ_KIND_RX;
    if (GM == GM_NONE) return FQ_KIND_COST;
    return PH != PH_NONE ? FQ_KIND_LAYER_PASS : FQ_KIND_STRIDED_PASS;
}

template <int PH, int EX, bool ST>
static double pass_bytes(int N) {
    const double n = (double)(1ull << N);
    const bool load = (PH != PH_INIT) && (ST || EX == EX_ENERGY);
    return n * ((load ? 16.0 : 0.0) + (ST ? 16.0 : 0.0) + (EX == EX_DIAG ? 8.0 : 0.0));
}

template <typename WT, int PH, int GM, int EX, bool ST, int SC>
static int launch_pass(fq_ctx* ctx, const PassArgs& A) {
    auto fn = k_pass<WT, PH, GM, EX, ST, SC>;
    const size_t smem = pass_smem_bytes<WT>(A.N);
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pass_smem_bytes<WT>(kMaxQubits)));
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->ctas_per_sm * ctx->num_sms);
    const int tok = prof_begin(ctx);
    fn<<<(unsigned)grid, kPassThreads, smem, ctx->stream>>>(A);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, pass_kind<PH, GM, EX, ST>(), pass_bytes<PH, EX, ST>(A.N));
    ctx->launches++;
    return FQ_OK;
}

// ------------------------------------------------------------ TMA pass --

static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
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

// Which passes run as TMA pipelines (FQ_TMA overrides; measured on B200 at
// N=30, see the profiles):
//   0  none (every pass uses per-thread loads, k_pass)
//   1  passes without a cost phase use the one-group TMA pass (default:
//      strided passes are fastest there, the phase pass with k_pass)
//   2  every read-write pass uses the two-group TMA pass
//   3  every read-write pass uses the one-group TMA pass
static int tma_mode() {
    static int m = -1;
    if (m < 0) {
        const char* e = getenv("FQ_TMA");
        m = e ? std::max(0, std::min(3, atoi(e))) : 1;
    }
    return m;
}
static bool tma_for(int ph) {
    const int m = tma_mode();
    return m >= 2 || (m == 1 && ph == PH_NONE);
}
static int tma_groups() { return tma_mode() == 2 ? 2 : 1; }

// The state as a tensor of float64 whose innermost dimension is one 128-byte
// row of 8 amplitudes; the box is one tile (4096 amplitudes) in tile order.
// Returns false for tiles with rows narrower than 8 amplitudes.
static bool make_pass_tmap(const PassArgs& A, CUtensorMap* map, TmaGeom* G) {
    auto enc = tmap_encoder();
    if (!enc || !A.sv || ((uintptr_t)A.sv & 127) != 0) return false;
    const int N = A.N, l = A.l, a = A.a, k = kTileBits - l;
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
static int launch_tma(fq_ctx* ctx, const PassArgs& A, const CUtensorMap& map, TmaGeom G) {
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->num_sms);
    const int tok = prof_begin(ctx);
    if (tma_groups() == 2) {
        auto fn = k_pass_tma2<WT, PH, GM, EX, SC>;
        FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tma2_pass_smem_bytes<WT>(kMaxQubits)));
        fn<<<(unsigned)grid, 2 * kPassThreads, tma2_pass_smem_bytes<WT>(A.N), ctx->stream>>>(
            A, map, G);
    } else {
        auto fn = k_pass_tma<WT, PH, GM, EX, SC>;
        FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tma_pass_smem_bytes<WT>(kMaxQubits)));
        fn<<<(unsigned)grid, kPassThreads, tma_pass_smem_bytes<WT>(A.N), ctx->stream>>>(A, map,
                                                                                        G);
    }
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, pass_kind<PH, GM, EX, true>(), pass_bytes<PH, EX, true>(A.N));
    ctx->launches++;
    return FQ_OK;
}

// Passes without RX (cost phase, <C>, cut diagonal) use the L0 schedule.
// Passes that read and write the state run as TMA pipelines where the tile
// geometry allows; write-only (layer-0) and read-only passes use k_pass.
template <typename WT, int PH, int GM, int EX, bool ST>
static int launch_pass(fq_ctx* ctx, const PassArgs& A) {
    if (GM == GM_NONE && !(ST && PH == PH_MUL)) return launch_pass<WT, PH, GM, EX, ST, SC_L0>(ctx, A);
    const int sc = GM == GM_NONE ? SC_L0 : schedule_for(A.tmask);
    if (ST && PH != PH_INIT && EX != EX_DIAG && tma_for(PH)) {
        alignas(64) CUtensorMap map;
        TmaGeom G;
        if (make_pass_tmap(A, &map, &G)) {
            constexpr int EXT = EX == EX_ENERGY ? EX_ENERGY : EX_NONE;
            switch (sc) {
                case SC_L021: return launch_tma<WT, PH, GM, EXT, SC_L021>(ctx, A, map, G);
                case SC_L01: return launch_tma<WT, PH, GM, EXT, SC_L01>(ctx, A, map, G);
                default: return launch_tma<WT, PH, GM, EXT, SC_L0>(ctx, A, map, G);
            }
        }
    }
    switch (sc) {
        case SC_L021: return launch_pass<WT, PH, GM, EX, ST, SC_L021>(ctx, A);
        case SC_L01: return launch_pass<WT, PH, GM, EX, ST, SC_L01>(ctx, A);
        default: return launch_pass<WT, PH, GM, EX, ST, SC_L0>(ctx, A);
    }
}

static int pass_grid(fq_ctx* ctx, const PassArgs& A) {
    return (int)std::min<i64>(A.ntiles, (i64)ctx->ctas_per_sm * ctx->num_sms);
}

// Whether launch_pass will run A as a TMA pipeline (one CTA per SM).
static bool runs_as_tma(const PassArgs& A, int ph) {
    if (!tma_for(ph) || ph == PH_INIT) return false;
    if (!tmap_encoder() || !A.sv || ((uintptr_t)A.sv & 127) != 0) return false;
    return A.l >= 3;
}

template <typename WT, int PH, int EX>
static int launch_gm(fq_ctx* ctx, int gm, const PassArgs& A) {
    if (gm == GM_TAN) return launch_pass<WT, PH, GM_TAN, EX, true>(ctx, A);
    return launch_pass<WT, PH, GM_COT, EX, true>(ctx, A);
}

template <typename WT>
static int launch_engine_pass(fq_ctx* ctx, int ph, int gm, int ex, const PassArgs& A) {
    if (ph == PH_INIT)
        return ex ? launch_gm<WT, PH_INIT, EX_ENERGY>(ctx, gm, A)
                  : launch_gm<WT, PH_INIT, EX_NONE>(ctx, gm, A);
    if (ph == PH_MUL)
        return ex ? launch_gm<WT, PH_MUL, EX_ENERGY>(ctx, gm, A)
                  : launch_gm<WT, PH_MUL, EX_NONE>(ctx, gm, A);
    return ex ? launch_gm<WT, PH_NONE, EX_ENERGY>(ctx, gm, A)
              : launch_gm<WT, PH_NONE, EX_NONE>(ctx, gm, A);
}

// ------------------------------------------------------------- planning --

struct PassPlan {
    int l, a;
    unsigned tmask;
};

static int passes_for(int N, int lrows) {
    return 1 + (N - kTileBits + (kTileBits - lrows) - 1) / (kTileBits - lrows);
}

// Row bits of the strided passes: the widest rows (best DRAM locality) that
// still give the fewest passes.  FQ_LROWS overrides (1..8) for tuning.
static int choose_lrows(int N) {
    const char* e = getenv("FQ_LROWS");
    if (e) {
        const int v = atoi(e);
        if (v >= 1 && v <= 8) return v;
    }
    int best = 4;
    for (int lr = 4; lr >= 1; lr--)
        if (passes_for(N, lr) < passes_for(N, best)) best = lr;
    return best;
}

// One layer's passes: the contiguous tile 0..11 (cost phase + 12 RX), then
// strided tiles bringing the next 12 - lrows qubits on chip each.  The last
// strided pass widens its rows when fewer qubits remain.
static std::vector<PassPlan> plan_layer(int N) {
    std::vector<PassPlan> v;
    v.push_back({kTileBits, kTileBits, (1u << kTileBits) - 1});
    const int lrows = choose_lrows(N);
    for (int q = kTileBits; q < N;) {
        const int k = std::min(kTileBits - lrows, N - q);
        const int l = kTileBits - k;
        v.push_back({l, q, ((1u << k) - 1) << l});
        q += k;
    }
    return v;
}

// Reduced RX: RX(beta) = f * G with G = [[1,-it],[-it,1]] (t = s/c, f = c)
// or [[u,-i],[-i,u]] (u = c/s, f = s), whichever keeps |t|,|u| <= 1.  The
// factor f of every gate in a layer is folded into that layer's phase.
static void gate_params(double beta, int& gm, double& g, double& f) {
    const double s = sin(beta / 2), c = cos(beta / 2);
    if (fabs(c) >= fabs(s)) {
        gm = GM_TAN;
        g = s / c;
        f = c;
    } else {
        gm = GM_COT;
        g = c / s;
        f = s;
    }
}

// Tiles a pass prefetches ahead into L2 (FQ_PREFETCH overrides, 0 = off).
static int prefetch_distance() {
    static int d = -1;
    if (d < 0) {
        const char* e = getenv("FQ_PREFETCH");
        d = e ? std::max(0, std::min(4, atoi(e))) : 1;
    }
    return d;
}

static PassArgs base_args(fq_ctx* ctx, void* sv, int N, const GraphPrep& g) {
    PassArgs A;
    memset(&A, 0, sizeof(A));
    A.sv = (double2*)sv;
    A.w = ctx->d_w;
    A.ptab = ctx->d_ptab;
    A.partial = ctx->d_partial;
    A.diag = nullptr;
    A.ntiles = 1ll << (N - kTileBits);
    A.N = N;
    A.l = kTileBits;
    A.a = kTileBits;
    A.tmask = 0;
    A.cmin = (int)g.cmin;
    A.ntab = g.integer ? (int)(g.cmax - g.cmin + 1) : 1;
    A.nhi = 0;
    A.W = g.integer ? (double)g.W_int : g.W;
    A.scale = 1.0;
    A.pf_dist = prefetch_distance();
    A.err = ctx->d_err;
    return A;
}

// High-part entries of the engine's two-level phase table (0: the range is
// too wide for shared memory and the one-level global table is used).
static int engine_nhi(const GraphPrep& g) {
    const long long range = g.cmax - g.cmin + 1;
    const long long nhi = (range + kPhaseLo - 1) / kPhaseLo;
    return nhi <= kPhaseHiMax ? (int)nhi : 0;
}

static int launch_table2(fq_ctx* ctx, const GraphPrep& g, double gamma, double scale) {
    const int nhi = engine_nhi(g);
    if (nhi == 0) return FQ_ERR_INVALID;
    const int n = kPhaseLo + nhi;
    const int tok = prof_begin(ctx);
    k_phase_table2<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ptab, (int)g.cmin, nhi,
                                                              g.W_int, gamma, scale);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
    ctx->launches++;
    return FQ_OK;
}

static int launch_table(fq_ctx* ctx, const GraphPrep& g, double gamma, double scale) {
    const int n = (int)(g.cmax - g.cmin + 1);
    k_phase_table<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ptab, (int)g.cmin, n, g.W_int,
                                                             gamma, scale);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}

static int read_result(fq_ctx* ctx, double* host) {
    FQ_CUDA(cudaMemcpyAsync(ctx->h_result, ctx->d_result, sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    FQ_TRY(check_device_error(ctx));
    *host = ctx->h_result[0];
    return FQ_OK;
}

static int reduce_to_result(fq_ctx* ctx, int n) {
    k_reduce_partials<<<1, 256, 0, ctx->stream>>>(ctx->d_partial, n, ctx->d_result);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}

static int check_state(void* sv, int N) {
    FQ_CHECK(sv != nullptr, FQ_ERR_INVALID, "null state pointer");
    FQ_CHECK(((uintptr_t)sv & 15) == 0, FQ_ERR_INVALID, "state pointer not 16-byte aligned");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range [1,%d]", N, kMaxQubits);
    return FQ_OK;
}

// Prepare the graph; small states always use the FP64 weights.
static int setup_graph(fq_ctx* ctx, const double* graph, int N, GraphPrep& g) {
    FQ_TRY(prep_graph(graph, N, g));
    if (N < kTileBits) g.integer = false;
    FQ_TRY(upload_graph(ctx, g, graph));
    return FQ_OK;
}

}  // namespace fq

using namespace fq;

extern "C" {

int fq_qaoa_forward(fq_ctx* ctx, void* sv, int N, int P, const double* graph,
                    const double* gammas, const double* betas, double* energy) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state(sv, N));
    FQ_CHECK(N >= 2, FQ_ERR_INVALID, "N=%d: need at least 2 qubits", N);
    FQ_CHECK(P >= 1 && gammas && betas, FQ_ERR_INVALID, "need P >= 1 and angle arrays");
    for (int p = 0; p < P; p++)
        FQ_CHECK(isfinite(gammas[p]) && isfinite(betas[p]), FQ_ERR_INVALID,
                 "non-finite angle at layer %d", p);
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    const double amp0 = fq_init_amp(N);
    if (N < kTileBits) {
        Targets T;
        for (int q = 0; q < N; q++) T.t[q] = q;
        for (int p = 0; p < P; p++) {
            k_cost_small<<<1, 1024, 0, ctx->stream>>>((double2*)sv, N, gammas[p],
                                                      (const double*)ctx->d_w, p == 0, amp0);
            k_rx_small<<<1, 1024, 0, ctx->stream>>>((double2*)sv, N, T, N, cos(betas[p] / 2),
                                                    sin(betas[p] / 2));
            ctx->launches += 2;
        }
        FQ_CUDA(cudaGetLastError());
        if (energy) {
            k_cut_small<<<1, 256, 0, ctx->stream>>>((const double2*)sv, N,
                                                    (const double*)ctx->d_w, ctx->d_result,
                                                    nullptr);
            FQ_CUDA(cudaGetLastError());
            ctx->launches++;
            FQ_TRY(read_result(ctx, energy));
        }
        return FQ_OK;
    }
    const std::vector<PassPlan> plan = plan_layer(N);
    int last_grid = 0;
    for (int p = 0; p < P; p++) {
        int gm;
        double gx, f;
        gate_params(betas[p], gm, gx, f);
        const double scale = pow(f, N) * (p == 0 ? amp0 : 1.0);
        const int nhi = g.integer ? engine_nhi(g) : 0;
        if (g.integer) {
            if (nhi > 0)
                FQ_TRY(launch_table2(ctx, g, gammas[p], scale));
            else
                FQ_TRY(launch_table(ctx, g, gammas[p], scale));
        }
        for (size_t i = 0; i < plan.size(); i++) {
            PassArgs A = base_args(ctx, sv, N, g);
            A.l = plan[i].l;
            A.a = plan[i].a;
            A.tmask = plan[i].tmask;
            A.gx = gx;
            A.nhi = nhi;
            A.gamma = gammas[p];
            A.scale = g.integer ? 1.0 : scale;
            const int ph = i == 0 ? (p == 0 ? PH_INIT : PH_MUL) : PH_NONE;
            const int ex = (energy && p == P - 1 && i + 1 == plan.size()) ? 1 : 0;
            if (g.integer)
                FQ_TRY(launch_engine_pass<int>(ctx, ph, gm, ex, A));
            else
                FQ_TRY(launch_engine_pass<double>(ctx, ph, gm, ex, A));
            last_grid = runs_as_tma(A, ph) ? (int)std::min<i64>(A.ntiles, ctx->num_sms)
                                           : pass_grid(ctx, A);
        }
    }
    if (energy) {
        FQ_TRY(reduce_to_result(ctx, last_grid));
        FQ_TRY(read_result(ctx, energy));
    }
    return FQ_OK;
}

int fq_expectation(fq_ctx* ctx, const void* sv, int N, const double* graph, double* energy) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state((void*)sv, N));
    FQ_CHECK(energy != nullptr, FQ_ERR_INVALID, "null energy pointer");
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    if (N < kTileBits) {
        k_cut_small<<<1, 256, 0, ctx->stream>>>((const double2*)sv, N, (const double*)ctx->d_w,
                                                ctx->d_result, nullptr);
        FQ_CUDA(cudaGetLastError());
        ctx->launches++;
        return read_result(ctx, energy);
    }
    PassArgs A = base_args(ctx, (void*)sv, N, g);
    if (g.integer)
        FQ_TRY((launch_pass<int, PH_NONE, GM_NONE, EX_ENERGY, false>(ctx, A)));
    else
        FQ_TRY((launch_pass<double, PH_NONE, GM_NONE, EX_ENERGY, false>(ctx, A)));
    FQ_TRY(reduce_to_result(ctx, pass_grid(ctx, A)));
    return read_result(ctx, energy);
}

int fq_cut_diagonal(fq_ctx* ctx, void* out, int N, const double* graph) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(out != nullptr && ((uintptr_t)out & 7) == 0, FQ_ERR_INVALID, "bad output pointer");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range", N);
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    if (N < kTileBits) {
        k_cut_small<<<1, 256, 0, ctx->stream>>>(nullptr, N, (const double*)ctx->d_w, nullptr,
                                                (double*)out);
        FQ_CUDA(cudaGetLastError());
        ctx->launches++;
        return FQ_OK;
    }
    PassArgs A = base_args(ctx, nullptr, N, g);
    A.diag = (double*)out;
    if (g.integer)
        return launch_pass<int, PH_NONE, GM_NONE, EX_DIAG, false>(ctx, A);
    return launch_pass<double, PH_NONE, GM_NONE, EX_DIAG, false>(ctx, A);
}

// src/rzz.cu:173-206.  Layer 0 writes phase * init_amp (launch control,
// src/rzz.cu:148-150); later layers multiply (src/rzz.cu:152-154).
int fq_cost_phase(fq_ctx* ctx, void* sv, int N, double angle, const double* graph,
                  int is_first_layer, double init_amp) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state(sv, N));
    FQ_CHECK(isfinite(angle) && isfinite(init_amp), FQ_ERR_INVALID, "non-finite angle");
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    if (N < kTileBits) {
        k_cost_small<<<1, 1024, 0, ctx->stream>>>((double2*)sv, N, angle, (const double*)ctx->d_w,
                                                  is_first_layer ? 1 : 0, init_amp);
        FQ_CUDA(cudaGetLastError());
        ctx->launches++;
        return FQ_OK;
    }
    PassArgs A = base_args(ctx, sv, N, g);
    A.gamma = angle;
    A.scale = is_first_layer ? init_amp : 1.0;
    if (g.integer) {
        FQ_TRY(launch_table(ctx, g, angle, 1.0));
        if (is_first_layer) return launch_pass<int, PH_INIT, GM_NONE, EX_NONE, true>(ctx, A);
        return launch_pass<int, PH_MUL, GM_NONE, EX_NONE, true>(ctx, A);
    }
    if (is_first_layer) return launch_pass<double, PH_INIT, GM_NONE, EX_NONE, true>(ctx, A);
    return launch_pass<double, PH_MUL, GM_NONE, EX_NONE, true>(ctx, A);
}

}  // extern "C"

namespace fq {

// RX(angle) (full form, src/rx.cu:47-50) on every qubit of `mask`: qubits
// below 12 share the contiguous tile, higher ones are covered by strided
// tiles of up to 9 qubits.
static int rx_mask(fq_ctx* ctx, void* sv, int N, unsigned long long mask, double angle) {
    const double s = sin(angle / 2), c = cos(angle / 2);  // src/rx.cu:121
    if (!mask) return FQ_OK;
    if (N < kTileBits) {
        Targets T;
        int nt = 0;
        for (int q = 0; q < N; q++)
            if ((mask >> q) & 1ull) T.t[nt++] = q;
        k_rx_small<<<1, 1024, 0, ctx->stream>>>((double2*)sv, N, T, nt, c, s);
        FQ_CUDA(cudaGetLastError());
        ctx->launches++;
        return FQ_OK;
    }
    GraphPrep g;  // RX passes read no cost data
    g.N = N;
    if (mask & 0xFFFull) {
        PassArgs A = base_args(ctx, sv, N, g);
        A.tmask = (unsigned)(mask & 0xFFFull);
        A.c = c;
        A.s = s;
        FQ_TRY((launch_pass<int, PH_NONE, GM_FULL, EX_NONE, true>(ctx, A)));
    }
    unsigned long long rest = mask & ~0xFFFull;
    const int k = std::min(kTileBits - 3, N - kTileBits);
    while (rest) {
        const int t0 = __builtin_ctzll(rest);
        const int a = std::min(t0, N - k);
        PassArgs A = base_args(ctx, sv, N, g);
        A.l = kTileBits - k;
        A.a = a;
        A.tmask = 0;
        for (int t = a; t < a + k; t++)
            if ((rest >> t) & 1ull) {
                A.tmask |= 1u << (A.l + t - a);
                rest &= ~(1ull << t);
            }
        A.c = c;
        A.s = s;
        FQ_TRY((launch_pass<int, PH_NONE, GM_FULL, EX_NONE, true>(ctx, A)));
    }
    return FQ_OK;
}

}  // namespace fq

using namespace fq;

extern "C" {

// src/rx.cu:118-174: RX(angle) on every listed target of the chunk.
int fq_rx_chunk(fq_ctx* ctx, void* sv, int N, int chunk_qubits, const int* targets, int gate_size,
                double angle) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state(sv, N));
    FQ_CHECK(isfinite(angle), FQ_ERR_INVALID, "non-finite angle");
    FQ_CHECK(chunk_qubits >= 1 && chunk_qubits <= 13 && chunk_qubits <= N, FQ_ERR_INVALID,
             "chunk_qubits=%d must be in [1, min(13, N)]", chunk_qubits);
    FQ_CHECK(gate_size >= 0 && gate_size <= chunk_qubits && (gate_size == 0 || targets),
             FQ_ERR_INVALID, "gate_size=%d must be in [0, chunk_qubits]", gate_size);
    unsigned long long seen = 0;
    for (int i = 0; i < gate_size; i++) {
        const int t = targets[i];
        FQ_CHECK(t >= 0 && t < chunk_qubits, FQ_ERR_INVALID,
                 "target %d outside the %d-qubit chunk", t, chunk_qubits);
        FQ_CHECK(!((seen >> t) & 1ull), FQ_ERR_INVALID, "target %d repeated", t);
        seen |= 1ull << t;
    }
    return rx_mask(ctx, sv, N, seen, angle);
}

int fq_rx_targets(fq_ctx* ctx, void* sv, int N, const int* targets, int n, double angle) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state(sv, N));
    FQ_CHECK(isfinite(angle), FQ_ERR_INVALID, "non-finite angle");
    FQ_CHECK(n >= 0 && n <= N && (n == 0 || targets), FQ_ERR_INVALID, "bad target list");
    unsigned long long seen = 0;
    for (int i = 0; i < n; i++) {
        const int t = targets[i];
        FQ_CHECK(t >= 0 && t < N, FQ_ERR_INVALID, "target %d out of range", t);
        FQ_CHECK(!((seen >> t) & 1ull), FQ_ERR_INVALID, "target %d repeated", t);
        seen |= 1ull << t;
    }
    return rx_mask(ctx, sv, N, seen, angle);
}

int fq_permute_qubits(fq_ctx* ctx, const void* src, void* dst, int N, const int* perm) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state((void*)src, N));
    FQ_TRY(check_state(dst, N));
    FQ_CHECK(src != dst, FQ_ERR_INVALID, "permutation must be out of place");
    FQ_CHECK(perm != nullptr, FQ_ERR_INVALID, "null permutation");
    Perm P;
    unsigned long long seen = 0;
    for (int b = 0; b < N; b++) {
        FQ_CHECK(perm[b] >= 0 && perm[b] < N && !((seen >> perm[b]) & 1ull), FQ_ERR_INVALID,
                 "perm is not a permutation of 0..N-1");
        seen |= 1ull << perm[b];
        P.p[b] = perm[b];
    }
    const u64 n = 1ull << N;
    const unsigned grid = (unsigned)std::min<u64>((n + 255) / 256, (u64)ctx->num_sms * 16);
    k_permute<<<grid, 256, 0, ctx->stream>>>((const double2*)src, (double2*)dst, N, P);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}

}  // extern "C"
