// fq_grad.cu -- <C> and its adjoint gradient with respect to every gamma_k
// and beta_k in one forward and one reverse sweep (fq_qaoa_energy_grad), and
// batches of small instances in one launch (fq_small_batch).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "fq_ctx.h"
#include "fq_engine.h"
#include "fq_launch.cuh"
#include "fq_disp_dual.cuh"
#include "fq_small.cuh"

namespace fq {

// RX(-beta) on A.tmask alone (the weights are not read: one instance).
static int dispatch_dual_rx(fq_ctx* ctx, int gm, const PassArgs& A, double* gb) {
    FQ_CHECK(gm == GM_TAN || gm == GM_COT, FQ_ERR_INVALID, "adjoint pass gate mode %d", gm);
    return gm == GM_TAN ? dual_sc<int, false, GM_TAN, GM_NONE>(ctx, A, gb, nullptr, nullptr)
                        : dual_sc<int, false, GM_COT, GM_NONE>(ctx, A, gb, nullptr, nullptr);
}

// Destinations of the reverse sweep's partial sums: sum j (the grid
// partials at part + j * grid) goes to out[dst[j]], or nowhere if -1.
constexpr int kMaxGradSums = 768;
struct GradSums {
    int dst[kMaxGradSums];
};

// One block per sum, in a fixed order (deterministic results).
__global__ void k_reduce_grad(const double* part, int grid, const GradSums S, double* out) {
    __shared__ double sh[256];
    const int j = blockIdx.x;
    const int d = S.dst[j];
    if (d < 0) return;  // uniform across the block
    const double* pb = part + (size_t)j * grid;
    double s = 0;
    for (int t = threadIdx.x; t < grid; t += 256) s += pb[t];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[d] = sh[0];
}

// n jobs of one size class: CB = 0 (N <= 12, one CTA each, nl = the
// largest N) or CB = N - 12 (a cluster of 2^CB CTAs each, nl = 12).
template <int CB>
static int launch_small_class(const SmallJob* jobs, int n, int nl, cudaStream_t stream) {
    auto fn = k_small_jobs<CB>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)small_smem_bytes(kSmallMaxQubits)));
    if (CB == 0) {
        fn<<<n, kSmallThreads, small_smem_bytes(nl), stream>>>(jobs, n);
        FQ_CUDA(cudaGetLastError());
        return FQ_OK;
    }
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)n << CB);
    cfg.blockDim = dim3(kSmallThreads);
    cfg.dynamicSmemBytes = small_smem_bytes(kSmallMaxQubits);
    cfg.stream = stream;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeClusterDimension;
    at.val.clusterDim.x = 1u << CB;
    at.val.clusterDim.y = 1;
    at.val.clusterDim.z = 1;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    FQ_CUDA(cudaLaunchKernelEx(&cfg, fn, jobs, n));
    return FQ_OK;
}

int launch_small_jobs(const SmallJob* jobs, const int* counts, int nmax0, cudaStream_t stream) {
    int off = 0;
    for (int c = 0; c <= kSmallJobMaxQubits - kSmallMaxQubits; c++) {
        if (counts[c] == 0) continue;
        switch (c) {
            case 0: FQ_TRY(launch_small_class<0>(jobs, counts[0], nmax0, stream)); break;
            case 1: FQ_TRY(launch_small_class<1>(jobs + off, counts[1], 12, stream)); break;
            case 2: FQ_TRY(launch_small_class<2>(jobs + off, counts[2], 12, stream)); break;
            default: FQ_TRY(launch_small_class<3>(jobs + off, counts[3], 12, stream)); break;
        }
        off += counts[c];
    }
    return FQ_OK;
}

// Upload a batch of small jobs (descriptors + their data) through the
// pinned staging buffer into ctx->d_scratch and launch one CTA per job.
// data: per job, N*N weights, P gammas, P betas (doubles, host); outputs go
// to d_result starting at word out_base.
struct SmallHostJob {
    int N, P, flags;
    const double* w;  // N*N symmetric (host)
    const double* gammas;
    const double* betas;
    double2* state;   // device or null
};

static int run_small_jobs(fq_ctx* ctx, const SmallHostJob* jobs, int njobs, int out_base,
                          std::vector<int>& out_off) {
    size_t need = sizeof(SmallJob) * njobs;
    int nmax = 1, outw = 0;
    for (int i = 0; i < njobs; i++) {
        need += sizeof(double) * (jobs[i].N * jobs[i].N + 2 * jobs[i].P);
        if (small_class(jobs[i].N) == 0) nmax = std::max(nmax, jobs[i].N);  // class 0's largest
        outw += 1 + 2 * jobs[i].P;
    }
    FQ_CHECK(need <= ctx->h_stage_bytes && need <= kScratchBytes, FQ_ERR_INVALID,
             "small batch too large for the staging buffer (%zu bytes)", need);
    FQ_CHECK(out_base + outw <= kResultWords, FQ_ERR_INVALID, "too many small-job outputs");
    FQ_TRY(stage_acquire(ctx));
    unsigned char* h = ctx->h_stage;
    SmallJob* hj = reinterpret_cast<SmallJob*>(h);
    double* hd = reinterpret_cast<double*>(h + sizeof(SmallJob) * njobs);
    const double* dd = reinterpret_cast<const double*>(ctx->d_scratch + sizeof(SmallJob) * njobs);
    size_t off = 0;
    int o = out_base;
    out_off.assign(njobs, 0);
    for (int i = 0; i < njobs; i++) {
        const SmallHostJob& J = jobs[i];
        SmallJob d;
        d.N = J.N;
        d.P = J.P;
        d.flags = J.flags;
        d.pad = 0;
        memcpy(hd + off, J.w, sizeof(double) * J.N * J.N);
        d.w = dd + off;
        off += J.N * J.N;
        memcpy(hd + off, J.gammas, sizeof(double) * J.P);
        d.gammas = dd + off;
        off += J.P;
        memcpy(hd + off, J.betas, sizeof(double) * J.P);
        d.betas = dd + off;
        off += J.P;
        d.out = ctx->d_result + o;
        out_off[i] = o;
        o += 1 + 2 * J.P;
        d.state = J.state;
        hj[i] = d;
    }
    FQ_CUDA(cudaMemcpyAsync(ctx->d_scratch, h, need, cudaMemcpyHostToDevice, ctx->stream));
    FQ_CUDA(cudaEventRecord(ctx->stage_evt, ctx->stream));
    const int tok = prof_begin(ctx);
    int counts[kSmallClasses] = {};
    for (int i = 0; i < njobs; i++) counts[small_class(jobs[i].N)]++;
    for (int i = 1; i < njobs; i++)
        FQ_CHECK(small_class(jobs[i].N) >= small_class(jobs[i - 1].N), FQ_ERR_INVALID,
                 "small jobs must come ordered by size class");
    FQ_TRY(launch_small_jobs(reinterpret_cast<const SmallJob*>(ctx->d_scratch), counts, nmax,
                             ctx->stream));
    prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
    ctx->launches++;
    return FQ_OK;
}

static int read_results(fq_ctx* ctx, int words) {
    FQ_CUDA(cudaMemcpyAsync(ctx->h_result, ctx->d_result, sizeof(double) * words,
                            cudaMemcpyDeviceToHost, ctx->stream));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

static int check_angles(int P, const double* gammas, const double* betas) {
    FQ_CHECK(P >= 1 && gammas && betas, FQ_ERR_INVALID, "need P >= 1 and angle arrays");
    for (int p = 0; p < P; p++)
        FQ_CHECK(isfinite(gammas[p]) && isfinite(betas[p]), FQ_ERR_INVALID,
                 "non-finite angle at layer %d", p);
    return FQ_OK;
}

// Enqueue the gradient of an N >= 13 circuit on ctx's stream; the results
// land in ctx->h_result once the stream reaches this point (grad_collect).
int grad_enqueue(fq_ctx* ctx, void* sv, void* costate, int N, int P, const double* graph,
                 const double* gammas, const double* betas) {
    FQ_TRY(check_angles(P, gammas, betas));
    FQ_TRY(check_state(sv, N));
    FQ_TRY(check_state(costate, N));
    FQ_CHECK(sv != costate, FQ_ERR_INVALID, "state and costate must be different buffers");
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    const std::vector<PassPlan> plan = plan_layer(N);
    const int npass = (int)plan.size();
    FQ_CHECK(1 + P + P * npass < kResultWords, FQ_ERR_INVALID, "P=%d too large", P);

    // Reverse sweep.  Layer k visits its passes in the reverse of the
    // forward order (descending plan order for even k, ascending for odd
    // k); its last pass completes the layer's mixer, so it also takes
    // dE/dgamma_k and the inverse phase, and shares its tile geometry with
    // the first pass of layer k-1, which it runs too unless FQ_FUSE=0
    // (sweeps: npass + (P-1)(npass-1) instead of P * npass).  RX(-beta)
    // runs in reduced form f * G (gate_params): the kernels track the scale
    // the vectors gain (1/f per rotation) and the phase pass multiplies f^N
    // back in.  Each pass writes its partials (beta, gamma, the earlier
    // layer's beta: grid each) to its own segment of d_partial, summed by
    // one launch at the end (right after the pass if they do not fit).
    // The two-level phase tables of the forward sweep are reused.
    struct RevPass {
        int k, i;    // layer, plan pass
        bool phi;    // completes layer k's mixer
        bool fused;  // also runs layer k-1's first pass
    };
    const bool fuse = fuse_enabled();
    std::vector<RevPass> rev;
    for (int k = P - 1; k >= 0; k--)
        for (int j = 0; j < npass; j++) {
            if (fuse && j == 0 && k < P - 1) continue;  // ran fused with layer k+1's last pass
            const int i = (k % 2 == 0) ? npass - 1 - j : j;
            const bool last = j == npass - 1;
            rev.push_back({k, i, last, last && fuse && k > 0});
        }
    const int nrev = (int)rev.size();
    // Turnaround: the forward circuit's last pass, lambda = C psi with <C>
    // and the reverse sweep's first pass share one tile geometry, so they
    // run as one sweep (k_pass_dual with TURN) whenever the first reverse
    // pass is an RX pass over the last forward pass's tile.  Otherwise the
    // forward circuit runs to its end and a <C> sweep writes lambda.
    const bool turn = !rev[0].phi && rev[0].i == engine_last_pass(g, N, P);
    FQ_TRY(engine_forward(ctx, sv, N, P, g, gammas, betas, nullptr, turn));
    if (!turn) {
        PassArgs A = base_args(ctx, sv, N, g);
        A.sv2 = (double2*)costate;
        FQ_TRY(dispatch_costate(ctx, g.integer, A));
        FQ_TRY(reduce_partials(ctx, ctx->d_partial, pass_grid(ctx, A, PH_NONE, false),
                               ctx->d_result));
    }
    const int grid = (int)std::min<i64>(1ll << (N - kTileBits), (i64)ctx->num_sms);
    const bool batched = (i64)nrev * 3 * grid <= ctx->partial_cap && 3 * nrev <= kMaxGradSums;
    const bool all_tables = g.integer && engine_nhi(g) > 0 && P <= kMaxTableLayers;
    const int nhi = g.integer ? engine_nhi(g) : 0;
    std::vector<int> gm(P);
    std::vector<double> gx(P), f(P);
    for (int k = 0; k < P; k++) gate_params(-betas[k], gm[k], gx[k], f[k]);
    std::vector<int> rotated(P, 0);  // qubits of layer k rotated so far
    GradSums sums;
    for (int j = 0; j < kMaxGradSums; j++) sums.dst[j] = -1;
    for (int q = 0; q < nrev; q++) {
        const RevPass& R = rev[q];
        const int k = R.k, i = R.i;
        PassArgs A = base_args(ctx, sv, N, g);
        A.sv2 = (double2*)costate;
        A.l = plan[i].l;
        A.a = plan[i].a;
        A.tmask = plan[i].tmask;
        const int nt = __builtin_popcount(plan[i].tmask);
        A.gx = gx[k];
        A.f2 = f[k] * f[k];
        A.sc0 = pow(f[k] * f[k], rotated[k]);
        rotated[k] += nt;
        double* gb = ctx->d_partial + (batched ? (size_t)q * 3 * grid : 0);
        double* gg = gb + grid;
        double* gb2 = gb + 2 * grid;
        const int dst_b = 1 + P + k * npass + i, dst_g = 1 + k;
        const int dst_b2 = 1 + P + (k - 1) * npass + i;
        if (turn && q == 0) {
            int gmf;
            double f_unused;
            gate_params(betas[k], gmf, A.gx2, f_unused);
            FQ_TRY(g.integer ? dispatch_dual_turn_int(ctx, gm[k], gmf, A, gb, gg)
                             : dispatch_dual_turn_fp(ctx, gm[k], gmf, A, gb, gg));
        } else if (!R.phi) {
            FQ_TRY(dispatch_dual_rx(ctx, gm[k], A, gb));
        } else {
            if (g.integer && !all_tables) {
                if (nhi > 0)
                    FQ_TRY(launch_table2(ctx, g, gammas[k]));
                else
                    FQ_TRY(launch_table(ctx, g, gammas[k], 1.0));
            }
            A.gamma = gammas[k];
            if (nhi > 0) set_table_args(A, g, gammas[k], 1.0);
            if (all_tables) A.ptab = ctx->d_ptab + (size_t)k * kTableStride;
            A.tree = phase_tree_ok(g, gammas[k]) ? 1 : 0;
            // Inverse phase (times f^N) only where layers remain.
            A.scale = k > 0 ? pow(f[k], N) : 0.0;
            int gm2 = GM_NONE;
            if (R.fused) {
                gm2 = gm[k - 1];
                A.gx2 = gx[k - 1];
                A.f2b = f[k - 1] * f[k - 1];
                rotated[k - 1] += nt;
            }
            // Layer 0's completing pass ends the sweep: psi and lambda are
            // workspaces whose final contents nothing reads, so it only
            // reads them (32 instead of 64 B per amplitude).
            const bool store = q + 1 < nrev;
            FQ_TRY(g.integer ? dispatch_dual_phase_int(ctx, gm[k], gm2, A, gb, gg, gb2, store)
                             : dispatch_dual_phase_fp(ctx, gm[k], gm2, A, gb, gg, gb2, store));
        }
        const bool energy_here = turn && q == 0;  // <C> partials of the turnaround
        if (batched) {
            sums.dst[3 * q] = dst_b;
            if (R.phi) sums.dst[3 * q + 1] = dst_g;
            if (energy_here) sums.dst[3 * q + 1] = 0;
            if (R.fused) sums.dst[3 * q + 2] = dst_b2;
        } else {
            FQ_TRY(reduce_partials(ctx, gb, grid, ctx->d_result + dst_b));
            if (energy_here) FQ_TRY(reduce_partials(ctx, gg, grid, ctx->d_result));
            if (R.phi) FQ_TRY(reduce_partials(ctx, gg, grid, ctx->d_result + dst_g));
            if (R.fused) FQ_TRY(reduce_partials(ctx, gb2, grid, ctx->d_result + dst_b2));
        }
    }
    if (batched) {
        const int tok = prof_begin(ctx);
        k_reduce_grad<<<3 * nrev, 256, 0, ctx->stream>>>(ctx->d_partial, grid, sums,
                                                         ctx->d_result);
        FQ_CUDA(cudaGetLastError());
        prof_end(ctx, tok, FQ_KIND_OTHER, 0.0);
        ctx->launches++;
    }
    FQ_CUDA(cudaMemcpyAsync(ctx->h_result, ctx->d_result, sizeof(double) * (1 + P + P * npass),
                            cudaMemcpyDeviceToHost, ctx->stream));
    // The kernels' error flag travels with the results (last result word).
    FQ_CUDA(cudaMemcpyAsync(ctx->h_result + kResultWords - 1, ctx->d_err, sizeof(int),
                            cudaMemcpyDeviceToHost, ctx->stream));
    return FQ_OK;
}

int grad_collect(fq_ctx* ctx, int N, int P, double* energy, double* grad_gamma,
                 double* grad_beta) {
    const int npass = (int)plan_layer(N).size();
    const double* r = ctx->h_result;
    int flag = 0;
    memcpy(&flag, r + kResultWords - 1, sizeof(int));
    if (flag) {
        FQ_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        set_error("a device-side bounded wait gave up (flag %d); results are incomplete", flag);
        return FQ_ERR_TIMEOUT;
    }
    *energy = r[0];
    for (int k = 0; k < P; k++) {
        grad_gamma[k] = -r[1 + k];
        double s = 0;
        for (int i = 0; i < npass; i++) s += r[1 + P + k * npass + i];
        grad_beta[k] = s;
    }
    return FQ_OK;
}

}  // namespace fq

using namespace fq;

extern "C" {

int fq_qaoa_energy_grad(fq_ctx* ctx, void* sv, void* costate, int N, int P, const double* graph,
                        const double* gammas, const double* betas, double* energy,
                        double* grad_gamma, double* grad_beta) {
    FQ_TRY(validate_ctx(ctx));
    FQ_CHECK(N >= 2 && N <= kMaxQubits, FQ_ERR_INVALID, "N=%d out of range [2,%d]", N,
             kMaxQubits);
    FQ_TRY(check_angles(P, gammas, betas));
    FQ_CHECK(energy && grad_gamma && grad_beta, FQ_ERR_INVALID, "null output");
    if (N <= kSmallJobMaxQubits) {
        FQ_CHECK(1 + 2 * P <= kResultWords, FQ_ERR_INVALID, "P=%d too large", P);
        GraphPrep g;
        FQ_TRY(prep_graph(graph, N, g));
        SmallHostJob J{N, P, SJ_ENERGY | SJ_GRAD, g.wd.data(), gammas, betas, nullptr};
        std::vector<int> off;
        FQ_TRY(run_small_jobs(ctx, &J, 1, 0, off));
        FQ_TRY(read_results(ctx, 1 + 2 * P));
        *energy = ctx->h_result[0];
        for (int k = 0; k < P; k++) {
            grad_gamma[k] = ctx->h_result[1 + k];
            grad_beta[k] = ctx->h_result[1 + P + k];
        }
        return FQ_OK;
    }
    FQ_TRY(grad_enqueue(ctx, sv, costate, N, P, graph, gammas, betas));
    FQ_CUDA(cudaStreamSynchronize(ctx->stream));
    return grad_collect(ctx, N, P, energy, grad_gamma, grad_beta);
}

}  // extern "C"
