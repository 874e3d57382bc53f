// fq_engine.cu -- fused QAOA engine and the reference-path cost / RX entry
// points, all built on the streaming tile pass (fq_pass.cuh).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fq_ctx.h"
#include "fq_engine.h"
#include "fq_launch.cuh"

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

// Two-level table of powers of z = exp(i*gamma) used by the engine's
// passes: tab[j] = z^j for j < 32, tab[32 + h] = z^(dlo + 32h).
__global__ void k_phase_table2(double2* tab, int dlo, int nhi, double gamma) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double sn, cs;
    if (i < kPhaseLo) {
        sincos(gamma * (double)i, &sn, &cs);
        tab[i] = make_double2(cs, sn);
    } else if (i < kPhaseLo + nhi) {
        sincos(gamma * (double)(dlo + 32ll * (i - kPhaseLo)), &sn, &cs);
        tab[i] = make_double2(cs, sn);
    }
}

// Tables of k_phase_table2 for up to kMaxTableLayers layers in one launch:
// layer p's table at tab + p * kTableStride.
struct LayerGammas {
    double g[kMaxTableLayers];
};

__global__ void k_phase_tables2(double2* tab, int dlo, int nhi, LayerGammas lg, int P) {
    const int p = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    double sn, cs;
    double2* t = tab + (size_t)p * kTableStride;
    if (i < kPhaseLo) {
        sincos(lg.g[p] * (double)i, &sn, &cs);
        t[i] = make_double2(cs, sn);
    } else if (i < kPhaseLo + nhi) {
        sincos(lg.g[p] * (double)(dlo + 32ll * (i - kPhaseLo)), &sn, &cs);
        t[i] = make_double2(cs, sn);
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

// Per-block max|a-b|^2, max|b|^2, sum|a-b|^2, sum|b|^2 over a grid-stride
// split (fixed per launch geometry, so the same inputs give the same bits).
__global__ void k_state_diff(const double2* a, const double2* b, u64 n, double* part) {
    __shared__ double sh[4][256];
    double m = 0, mb = 0, s = 0, sb = 0;
    for (u64 i = blockIdx.x * 256ull + threadIdx.x; i < n; i += (u64)gridDim.x * 256ull) {
        const double2 x = a[i], y = b[i];
        const double dx = x.x - y.x, dy = x.y - y.y;
        const double d2 = dx * dx + dy * dy, b2 = y.x * y.x + y.y * y.y;
        m = fmax(m, d2);
        mb = fmax(mb, b2);
        s += d2;
        sb += b2;
    }
    sh[0][threadIdx.x] = m;
    sh[1][threadIdx.x] = mb;
    sh[2][threadIdx.x] = s;
    sh[3][threadIdx.x] = sb;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + o]);
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + o]);
            sh[2][threadIdx.x] += sh[2][threadIdx.x + o];
            sh[3][threadIdx.x] += sh[3][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) part[4 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

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

// ------------------------------------------------------------- planning --


static int passes_for(int N, int lrows) {
    return 1 + (N - kTileBits + (kTileBits - lrows) - 1) / (kTileBits - lrows);
}

// Row bits of the strided passes: the widest rows (best DRAM locality) that
// still give the fewest passes.
static int choose_lrows(int N) {
    int best = 4;
    for (int lr = 4; lr >= 1; lr--)
        if (passes_for(N, lr) < passes_for(N, best)) best = lr;
    return best;
}

// One layer's passes: the contiguous tile 0..11 and strided tiles bringing
// the next 12 - lrows qubits on chip each (the last strided pass widens its
// rows when fewer qubits remain).  The first pass of a layer carries its
// cost phase (layer 0: the launch-control init), and the fused schedule
// runs the first and last passes of consecutive layers as one sweep, so
// with three or more passes the contiguous pass (four exchanges when fused,
// two alone) goes second and never fuses: on B200 at N=30, p=5, 59.5-59.7
// layers/s against 57.2-57.6 with it first (A/B in one call).  The strided
// passes over the highest qubits lead and the one over the lowest closes
// each layer: an odd circuit then ends on the faster of the two strided
// geometries (61.2-61.8 against 60.3-61.0 layers/s, A/B in one call).
std::vector<PassPlan> plan_layer(int N) {
    std::vector<PassPlan> v;
    v.push_back({kTileBits, kTileBits, (1u << kTileBits) - 1});
    const int lrows = choose_lrows(N);
    for (int q = kTileBits; q < N;) {
        const int k = std::min(kTileBits - lrows, N - q);
        const int l = kTileBits - k;
        v.push_back({l, q, ((1u << k) - 1) << l});
        q += k;
    }
    if (v.size() >= 3) {  // [last strided, contiguous, ..., first strided]
        std::swap(v[0], v[v.size() - 1]);
        std::swap(v[1], v[v.size() - 1]);
    }
    return v;
}

// Reduced RX: RX(beta) = f * G with G = [[1,-it],[-it,1]] (t = s/c, f = c)
// or [[u,-i],[-i,u]] (u = c/s, f = s), whichever keeps |t|,|u| <= 1.  The
// factor f of every gate in a layer is folded into that layer's phase.
void gate_params(double beta, int& gm, double& g, double& f) {
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

PassArgs base_args(fq_ctx* ctx, void* sv, int N, const GraphPrep& g) {
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

// Range [dlo, dhi] of the powers of z the passes look up: every cut value
// and every single-qubit flip change g (|g| <= gmax).
static void table_range(const GraphPrep& g, long long& dlo, long long& dhi) {
    dlo = std::min(g.cmin, -g.gmax);
    dhi = std::max(g.cmax, g.gmax);
}

// High-part entries of the engine's two-level table (0: the range is too
// wide for shared memory and the one-level global phase table is used).
int engine_nhi(const GraphPrep& g) {
    long long dlo, dhi;
    table_range(g, dlo, dhi);
    const long long nhi = (dhi - dlo + 1 + kPhaseLo - 1) / kPhaseLo;
    return nhi <= kPhaseHiMax ? (int)nhi : 0;
}

int launch_tables2(fq_ctx* ctx, const GraphPrep& g, const double* gammas, int P) {
    const int nhi = engine_nhi(g);
    if (nhi == 0 || P > kMaxTableLayers) return FQ_ERR_INVALID;
    long long dlo, dhi;
    table_range(g, dlo, dhi);
    LayerGammas lg;
    for (int p = 0; p < kMaxTableLayers; p++) lg.g[p] = p < P ? gammas[p] : 0.0;
    const int n = kPhaseLo + nhi;
    const int tok = prof_begin(ctx);
    k_phase_tables2<<<dim3((n + 255) / 256, P), 256, 0, ctx->stream>>>(ctx->d_ptab, (int)dlo, nhi,
                                                                       lg, P);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
    ctx->launches++;
    return FQ_OK;
}

int launch_table2(fq_ctx* ctx, const GraphPrep& g, double gamma) {
    const int nhi = engine_nhi(g);
    if (nhi == 0) return FQ_ERR_INVALID;
    long long dlo, dhi;
    table_range(g, dlo, dhi);
    const int n = kPhaseLo + nhi;
    const int tok = prof_begin(ctx);
    k_phase_table2<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ptab, (int)dlo, nhi, gamma);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
    ctx->launches++;
    return FQ_OK;
}

bool phase_tree_ok(const GraphPrep& g, double gamma) { return fabs(gamma) * g.wabs <= 512.0; }

void set_table_args(PassArgs& A, const GraphPrep& g, double gamma, double scale) {
    A.nhi = engine_nhi(g);
    if (A.nhi > 0) {
        long long dlo, dhi;
        table_range(g, dlo, dhi);
        A.dlo = (int)dlo;
        A.ntab = (int)(dhi - dlo + 1);
        const double th = -gamma * (double)g.W_int / 2;
        A.ph0x = scale * cos(th);
        A.ph0y = scale * sin(th);
    }
}

int launch_table(fq_ctx* ctx, const GraphPrep& g, double gamma, double scale) {
    const int n = (int)(g.cmax - g.cmin + 1);
    k_phase_table<<<(n + 255) / 256, 256, 0, ctx->stream>>>(ctx->d_ptab, (int)g.cmin, n, g.W_int,
                                                             gamma, scale);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}

int read_result(fq_ctx* ctx, double* host) {
    FQ_CUDA(cudaMemcpyAsync(ctx->h_result, ctx->d_result, sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    FQ_TRY(check_device_error(ctx));
    *host = ctx->h_result[0];
    return FQ_OK;
}

int reduce_partials(fq_ctx* ctx, const double* partial, int n, double* out_dev) {
    const int tok = prof_begin(ctx);
    k_reduce_partials<<<1, 256, 0, ctx->stream>>>(partial, n, out_dev);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
    ctx->launches++;
    return FQ_OK;
}

int reduce_to_result(fq_ctx* ctx, int n) {
    k_reduce_partials<<<1, 256, 0, ctx->stream>>>(ctx->d_partial, n, ctx->d_result);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    return FQ_OK;
}

int check_state(void* sv, int N) {
    FQ_CHECK(sv != nullptr, FQ_ERR_INVALID, "null state pointer");
    FQ_CHECK(((uintptr_t)sv & 15) == 0, FQ_ERR_INVALID, "state pointer not 16-byte aligned");
    FQ_CHECK(N >= 1 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range [1,%d]", N, kMaxQubits);
    return FQ_OK;
}

// Prepare the graph; small states always use the FP64 weights.
int setup_graph(fq_ctx* ctx, const double* graph, int N, GraphPrep& g) {
    FQ_TRY(prep_graph(graph, N, g));
    if (N < kTileBits) g.integer = false;
    FQ_TRY(upload_graph(ctx, g, graph));
    return FQ_OK;
}

// Cut constants of every tile of each plan geometry (k_tile_cuts, one
// launch) in ctx->d_tcut, grown on demand and kept while the weights and N
// stay the same: tabs[i] serves plan[i].  Below
// N = 21 (512 tiles) and without the buffer (a failed allocation) tabs
// stays null and the passes compute the constants per tile, as they do for
// shards and the read-only <C> pass.
// The table is 64 B per tile (128 B with FP64 weights), 1/1024 of the
// state per geometry; it replaces per-tile work on two warps of each tile
// and the barrier after it.  On B200 at N=30, p=5, with the layer-0 pass
// alternating its exchanges: layer-0 pass 5.26-5.32 against 5.66-5.78 ms,
// fused passes 9.27-9.34 against 9.62-9.66, the circuit 79.1-79.6 against
// 80.4-80.8 ms (A/B in one call).
static int tile_cut_tables(fq_ctx* ctx, const GraphPrep& g, int N,
                           const std::vector<PassPlan>& plan, std::vector<const void*>& tabs) {
    tabs.assign(plan.size(), nullptr);
    if (N < 21 || plan.size() > 4) return FQ_OK;
    const size_t wt = g.integer ? sizeof(int) : sizeof(double);
    const i64 ntiles = 1ll << (N - kTileBits);
    const size_t per = (size_t)ntiles * kTcutStride * wt;
    const size_t need = per * plan.size();
    // Built for these weights (no upload since) and this N: reuse them, as
    // an optimiser's calls on one graph do.
    if (ctx->d_tcut && need <= ctx->tcut_bytes && ctx->tcut_version == ctx->g_version &&
        ctx->tcut_n == N) {
        for (size_t i = 0; i < plan.size(); i++) tabs[i] = (char*)ctx->d_tcut + i * per;
        return FQ_OK;
    }
    ctx->tcut_version = -1;
    if (need > ctx->tcut_bytes) {
        if (ctx->d_tcut) {
            FQ_CUDA(cudaStreamSynchronize(ctx->stream));
            FQ_CUDA(cudaFree(ctx->d_tcut));
            ctx->d_tcut = nullptr;
            ctx->tcut_bytes = 0;
        }
        if (cudaMalloc(&ctx->d_tcut, need) != cudaSuccess) {
            cudaGetLastError();  // clear the allocation failure
            ctx->d_tcut = nullptr;
            return FQ_OK;
        }
        ctx->tcut_bytes = need;
    }
    const int grid = (int)std::min<i64>((ntiles + 3) / 4, (i64)ctx->num_sms * 8);
    // The attribute is the same for every N: contexts on other threads (the
    // server's lanes) set it concurrently, and a launch needing more than
    // another thread's smaller setting would fail.
    const size_t smem = g.integer ? tcut_smem_bytes<int>(N) : tcut_smem_bytes<double>(N);
    if (g.integer)
        FQ_CUDA(cudaFuncSetAttribute(k_tile_cuts<int>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tcut_smem_bytes<int>(kMaxQubits)));
    else
        FQ_CUDA(cudaFuncSetAttribute(k_tile_cuts<double>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)tcut_smem_bytes<double>(kMaxQubits)));
    TcutGeoms G;
    memset(&G, 0, sizeof(G));
    for (size_t i = 0; i < plan.size(); i++) {
        G.l[i] = plan[i].l;
        G.a[i] = plan[i].a;
    }
    const dim3 grid2(grid, (unsigned)plan.size());
    if (g.integer)
        k_tile_cuts<int><<<grid2, kPassThreads, smem, ctx->stream>>>((const int*)ctx->d_w, N, G,
                                                                     ntiles, (int*)ctx->d_tcut);
    else
        k_tile_cuts<double><<<grid2, kPassThreads, smem, ctx->stream>>>(
            (const double*)ctx->d_w, N, G, ntiles, (double*)ctx->d_tcut);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    ctx->tcut_version = ctx->g_version;
    ctx->tcut_n = N;
    for (size_t i = 0; i < plan.size(); i++) tabs[i] = (char*)ctx->d_tcut + i * per;
    return FQ_OK;
}

bool fuse_enabled() {
    static int m = -1;
    if (m < 0) {
        const char* e = getenv("FQ_FUSE");
        m = e ? (atoi(e) != 0) : 1;
    }
    return m != 0;
}

// The fused forward circuit for N >= 12 (see fq_qaoa_forward); with energy
// != NULL the last sweep also sums <C> and *energy receives it.

// The fused schedule: layer p visits its passes in plan order when p is even
// and in reverse order when p is odd, so the last pass of layer p and the
// first of layer p+1 have the same tile geometry and run as one fused pass
// (RX of layer p, phase of layer p+1, RX of layer p+1).  The phase still
// precedes every RX of its layer and follows every RX of the layer before:
// RX gates on different qubits commute.  Sweeps: npass + (P-1)(npass-1)
// instead of P * npass (11 instead of 15 at N=30, p=5).
static int engine_forward_fused(fq_ctx* ctx, void* sv, int N, int P, const GraphPrep& g,
                                const double* gammas, const double* betas, double* energy,
                                const std::vector<PassPlan>& plan,
                                const std::vector<const void*>& tcut, int& last_grid,
                                bool skip_last) {
    const double amp0 = fq_init_amp(N);
    const int npass = (int)plan.size();
    std::vector<int> gm(P);
    std::vector<double> gx(P), scale(P);
    for (int p = 0; p < P; p++) {
        double f;
        gate_params(betas[p], gm[p], gx[p], f);
        scale[p] = pow(f, N) * (p == 0 ? amp0 : 1.0);
    }
    if (g.integer) FQ_TRY(launch_tables2(ctx, g, gammas, P));
    // Phase arguments of layer q on a pass.
    auto phase_args = [&](PassArgs& A, int q) {
        if (g.integer) {
            set_table_args(A, g, gammas[q], scale[q]);
            A.ptab = ctx->d_ptab + (size_t)q * kTableStride;
        }
        A.tree = phase_tree_ok(g, gammas[q]) ? 1 : 0;
        A.gamma = gammas[q];
        A.scale = g.integer ? 1.0 : scale[q];
    };
    for (int p = 0; p < P; p++) {
        for (int j = (p == 0 ? 0 : 1); j < npass; j++) {
            if (skip_last && p == P - 1 && j == npass - 1) break;
            const int idx = (p % 2 == 0) ? j : npass - 1 - j;
            PassArgs A = base_args(ctx, sv, N, g);
            A.l = plan[idx].l;
            A.a = plan[idx].a;
            A.tmask = plan[idx].tmask;
            A.tcut = tcut[idx];
            A.gx = gx[p];
            const bool last_of_layer = j == npass - 1;
            int ph = PH_NONE;
            if (p == 0 && j == 0) {  // launch-control init + layer-0 phase + RX
                phase_args(A, 0);
                ph = PH_INIT;
                FQ_TRY(dispatch_phase_pass(ctx, g.integer, PH_INIT, gm[0], A));
            } else if (last_of_layer && p + 1 < P) {
                phase_args(A, p + 1);
                A.gx2 = gx[p + 1];
                ph = PH_MUL;
                FQ_TRY(dispatch_fused(ctx, g.integer, gm[p], gm[p + 1], A));
            } else {
                const bool ex = energy && p == P - 1 && last_of_layer;
                FQ_TRY(dispatch_rx(ctx, g.integer, gm[p], ex, A));
            }
            last_grid = pass_grid(ctx, A, ph, true);
        }
    }
    return FQ_OK;
}

bool engine_fused(const GraphPrep& g, int N, int P) {
    return fuse_enabled() && plan_layer(N).size() >= 2 && P >= 2 &&
           (!g.integer || (engine_nhi(g) > 0 && P <= kMaxTableLayers));
}

int engine_last_pass(const GraphPrep& g, int N, int P) {
    const int npass = (int)plan_layer(N).size();
    return (engine_fused(g, N, P) && (P - 1) % 2 == 1) ? 0 : npass - 1;
}

int engine_forward(fq_ctx* ctx, void* sv, int N, int P, const GraphPrep& g, const double* gammas,
                   const double* betas, double* energy, bool skip_last) {
    const double amp0 = fq_init_amp(N);
    const std::vector<PassPlan> plan = plan_layer(N);
    int last_grid = 0;
    const bool fused = engine_fused(g, N, P);
    FQ_CHECK(!(skip_last && (energy || plan.size() < 2)), FQ_ERR_INVALID,
             "the forward circuit can stop before its last pass only without <C> and with two "
             "or more passes per layer");
    std::vector<const void*> tcut;
    FQ_TRY(tile_cut_tables(ctx, g, N, plan, tcut));
    if (fused)
        FQ_TRY(engine_forward_fused(ctx, sv, N, P, g, gammas, betas, energy, plan, tcut,
                                    last_grid, skip_last));
    for (int p = 0; p < (fused ? 0 : P); p++) {
        int gm;
        double gx, f;
        gate_params(betas[p], gm, gx, f);
        const double scale = pow(f, N) * (p == 0 ? amp0 : 1.0);
        const int nhi = g.integer ? engine_nhi(g) : 0;
        // Two-level tables: all layers' in one launch (layer p's at slot p,
        // kept for the reverse sweep of a gradient); else one global table
        // per layer.
        const bool all_tables = nhi > 0 && P <= kMaxTableLayers;
        if (g.integer) {
            if (all_tables) {
                if (p == 0) FQ_TRY(launch_tables2(ctx, g, gammas, P));
            } else if (nhi > 0) {
                FQ_TRY(launch_table2(ctx, g, gammas[p]));
            } else {
                FQ_TRY(launch_table(ctx, g, gammas[p], scale));
            }
        }
        for (size_t i = 0; i < plan.size(); i++) {
            if (skip_last && p == P - 1 && i + 1 == plan.size()) break;
            PassArgs A = base_args(ctx, sv, N, g);
            A.l = plan[i].l;
            A.a = plan[i].a;
            A.tmask = plan[i].tmask;
            A.tcut = tcut[i];
            A.gx = gx;
            if (nhi > 0) set_table_args(A, g, gammas[p], scale);
            if (all_tables) A.ptab = ctx->d_ptab + (size_t)p * kTableStride;
            A.tree = phase_tree_ok(g, gammas[p]) ? 1 : 0;
            A.gamma = gammas[p];
            A.scale = g.integer ? 1.0 : scale;
            const int ph = i == 0 ? (p == 0 ? PH_INIT : PH_MUL) : PH_NONE;
            const int ex = (energy && p == P - 1 && i + 1 == plan.size() && i > 0) ? 1 : 0;
            if (ph != PH_NONE)
                FQ_TRY(dispatch_phase_pass(ctx, g.integer, ph, gm, A));
            else
                FQ_TRY(dispatch_rx(ctx, g.integer, gm, ex != 0, A));
            last_grid = pass_grid(ctx, A, ph, true);
        }
    }
    if (energy) {
        if (plan.size() == 1) {  // the only pass carries the phase: <C> in its own sweep
            PassArgs A = base_args(ctx, sv, N, g);
            FQ_TRY(dispatch_readonly(ctx, g.integer, false, A));
            last_grid = pass_grid(ctx, A, PH_NONE, false);
        }
        FQ_TRY(reduce_to_result(ctx, last_grid));
        FQ_TRY(read_result(ctx, energy));
    }
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
    return engine_forward(ctx, sv, N, P, g, gammas, betas, energy);
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
    FQ_TRY(dispatch_readonly(ctx, g.integer, false, A));
    FQ_TRY(reduce_to_result(ctx, pass_grid(ctx, A, PH_NONE, false)));
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
    return dispatch_readonly(ctx, g.integer, true, A);
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
    }
    return dispatch_phase_pass(ctx, g.integer, is_first_layer ? PH_INIT : PH_MUL, GM_NONE, A);
}

}  // extern "C"

namespace fq {

// RX(angle) (full form, src/rx.cu:47-50) on every qubit of `mask`: qubits
// below 12 share the contiguous tile, higher ones are covered by strided
// tiles of up to 9 qubits.
int rx_mask(fq_ctx* ctx, void* sv, int N, unsigned long long mask, double angle) {
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
        FQ_TRY(dispatch_rx_full(ctx, A));
    }
    // Targets above bit 11: strided tiles whose high bits are a window of
    // k qubits, in 9-qubit windows; a window spans only as many qubits as
    // its targets do (at least one), so few targets, such as the one or two
    // a sharded state swaps in per layer, leave the rows wide (2^(12-k)
    // contiguous amplitudes) and the pass streams at the copy rate.
    unsigned long long rest = mask & ~0xFFFull;
    const int kmax = std::min(kTileBits - 3, N - kTileBits);
    while (rest) {
        const int t0 = __builtin_ctzll(rest);
        int hi = t0;
        for (int t = t0; t < t0 + kmax && t < N; t++)
            if ((rest >> t) & 1ull) hi = t;
        const int k = hi - t0 + 1;
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
        FQ_TRY(dispatch_rx_full(ctx, A));
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

int fq_state_diff(fq_ctx* ctx, const void* a, const void* b, int N, double* out) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_state((void*)a, N));
    FQ_TRY(check_state((void*)b, N));
    FQ_CHECK(out != nullptr, FQ_ERR_INVALID, "null output");
    const u64 n = 1ull << N;
    const int grid = (int)std::min<u64>((n + 255) / 256, (u64)ctx->partial_cap / 4);
    k_state_diff<<<grid, 256, 0, ctx->stream>>>((const double2*)a, (const double2*)b, n,
                                                ctx->d_partial);
    FQ_CUDA(cudaGetLastError());
    ctx->launches++;
    std::vector<double> part(4 * (size_t)grid);
    FQ_CUDA(cudaMemcpyAsync(part.data(), ctx->d_partial, sizeof(double) * part.size(),
                            cudaMemcpyDeviceToHost, ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    double m = 0, mb = 0, s = 0, sb = 0;
    for (int i = 0; i < grid; i++) {
        m = std::max(m, part[4 * i]);
        mb = std::max(mb, part[4 * i + 1]);
        s += part[4 * i + 2];
        sb += part[4 * i + 3];
    }
    out[0] = sqrt(m);
    out[1] = sqrt(mb);
    out[2] = sqrt(s);
    out[3] = sqrt(sb);
    return FQ_OK;
}

}  // extern "C"
