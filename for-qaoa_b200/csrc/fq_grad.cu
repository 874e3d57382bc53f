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
#include "fq_pass_dual.cuh"
#include "fq_small.cuh"

namespace fq {

template <typename WT, bool PHI, int SC, int GM>
static int launch_dual(fq_ctx* ctx, const PassArgs& A, double* gb, double* gg) {
    auto fn = k_pass_dual<WT, PHI, SC, true, GM>;
    FQ_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dual_smem_bytes<WT>(kMaxQubits)));
    const i64 grid = std::min<i64>(A.ntiles, (i64)ctx->num_sms);
    const int tok = prof_begin(ctx);
    fn<<<(unsigned)grid, kPassThreads, dual_smem_bytes<WT>(A.N), ctx->stream>>>(A, gb, gg);
    FQ_CUDA(cudaGetLastError());
    prof_end(ctx, tok, FQ_KIND_ADJOINT, 64.0 * (double)(1ull << A.N));
    ctx->launches++;
    return FQ_OK;
}

template <int GM>
static int dispatch_dual_gm(fq_ctx* ctx, bool integer, bool phi, const PassArgs& A, double* gb,
                            double* gg) {
    if (phi) {
        FQ_CHECK(schedule_for(A.tmask) == SC_L021, FQ_ERR_INVALID, "adjoint phase pass mask");
        return integer ? launch_dual<int, true, SC_L021, GM>(ctx, A, gb, gg)
                       : launch_dual<double, true, SC_L021, GM>(ctx, A, gb, gg);
    }
    switch (schedule_for(A.tmask)) {
        case SC_L021: return launch_dual<int, false, SC_L021, GM>(ctx, A, gb, gg);
        case SC_L01: return launch_dual<int, false, SC_L01, GM>(ctx, A, gb, gg);
        default: return launch_dual<int, false, SC_L0, GM>(ctx, A, gb, gg);
    }
}

static int dispatch_dual(fq_ctx* ctx, bool integer, bool phi, int gm, const PassArgs& A,
                         double* gb, double* gg) {
    return gm == GM_TAN ? dispatch_dual_gm<GM_TAN>(ctx, integer, phi, A, gb, gg)
                        : dispatch_dual_gm<GM_COT>(ctx, integer, phi, A, gb, gg);
}

// One block per reverse pass q (in execution order: layers P-1..0, passes
// 1..npass-1 then 0): the fixed-order sum of its grid dE/dbeta partials
// (at part + q * stride) into out[1 + P + k * npass + i] and, for the
// contiguous pass (i = 0), of its dE/dgamma partials (at + grid) into
// out[1 + k].
__global__ void k_reduce_grad(const double* part, int stride, int grid, int P, int npass,
                              double* out) {
    __shared__ double sh[2][256];
    const int q = blockIdx.x;
    const int k = P - 1 - q / npass, i = (q % npass + 1) % npass;
    const double* pb = part + (size_t)q * stride;
    double sb = 0, sg = 0;
    for (int t = threadIdx.x; t < grid; t += 256) {
        sb += pb[t];
        if (i == 0) sg += pb[grid + t];
    }
    sh[0][threadIdx.x] = sb;
    sh[1][threadIdx.x] = sg;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + o];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[1 + P + k * npass + i] = sh[0][0];
        if (i == 0) out[1 + k] = sh[1][0];
    }
}

int launch_small_jobs(const SmallJob* jobs, int njobs, int nmax, cudaStream_t stream) {
    FQ_CUDA(cudaFuncSetAttribute(k_small_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)small_smem_bytes(kSmallMaxQubits)));
    k_small_jobs<<<njobs, kSmallThreads, small_smem_bytes(nmax), stream>>>(jobs, njobs);
    FQ_CUDA(cudaGetLastError());
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
        nmax = std::max(nmax, jobs[i].N);
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
    FQ_TRY(launch_small_jobs(reinterpret_cast<const SmallJob*>(ctx->d_scratch), njobs, nmax,
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

    // Forward circuit, then lambda = C psi with <C>.
    FQ_TRY(engine_forward(ctx, sv, N, P, g, gammas, betas, nullptr));
    {
        PassArgs A = base_args(ctx, sv, N, g);
        A.sv2 = (double2*)costate;
        FQ_TRY(dispatch_costate(ctx, g.integer, A));
        FQ_TRY(reduce_partials(ctx, ctx->d_partial, pass_grid(ctx, A, PH_NONE, false),
                               ctx->d_result));
    }
    // Reverse sweep: per layer the strided passes, then the contiguous pass
    // with dE/dgamma and the inverse phase.  RX(-beta) runs in reduced form
    // f * G (gate_params): the kernels track the scale the vectors gain
    // (1/f per rotation) and the contiguous pass multiplies f^N back in.
    // Partials of every reverse pass go to their own segment of d_partial
    // and are summed by one launch at the end (per-pass sums if they do not
    // fit).  The two-level phase tables of the forward sweep are reused.
    const int grid = (int)std::min<i64>(1ll << (N - kTileBits), (i64)ctx->num_sms);
    const int seg = 2 * ctx->num_sms;
    const bool batched = (i64)P * npass * seg <= ctx->partial_cap;
    const bool all_tables = g.integer && engine_nhi(g) > 0 && P <= kMaxTableLayers;
    int q = 0;
    for (int k = P - 1; k >= 0; k--) {
        int gm;
        double gx, f;
        gate_params(-betas[k], gm, gx, f);
        int rotated = 0;  // qubits rotated so far in this layer's reverse sweep
        const int nhi = g.integer ? engine_nhi(g) : 0;
        if (g.integer && !all_tables) {
            if (nhi > 0)
                FQ_TRY(launch_table2(ctx, g, gammas[k]));
            else
                FQ_TRY(launch_table(ctx, g, gammas[k], 1.0));
        }
        for (int o = 1; o <= npass; o++, q++) {
            const int i = o % npass;  // 1, 2, ..., npass-1, then 0
            PassArgs A = base_args(ctx, sv, N, g);
            A.sv2 = (double2*)costate;
            A.l = plan[i].l;
            A.a = plan[i].a;
            A.tmask = plan[i].tmask;
            A.gx = gx;
            A.f2 = f * f;
            A.sc0 = pow(f * f, rotated);
            rotated += __builtin_popcount(plan[i].tmask);
            A.gamma = gammas[k];
            if (nhi > 0) set_table_args(A, g, gammas[k], 1.0);
            if (all_tables) A.ptab = ctx->d_ptab + (size_t)k * kTableStride;
            A.tree = phase_tree_ok(g, gammas[k]) ? 1 : 0;
            // Inverse phase (times f^N) only where layers remain.
            A.scale = k > 0 ? pow(f, N) : 0.0;
            double* gb = ctx->d_partial + (batched ? (size_t)q * seg : 0);
            double* gg = gb + grid;
            FQ_TRY(dispatch_dual(ctx, g.integer, i == 0, gm, A, gb, gg));
            if (!batched) {
                FQ_TRY(reduce_partials(ctx, gb, grid, ctx->d_result + 1 + P + k * npass + i));
                if (i == 0) FQ_TRY(reduce_partials(ctx, gg, grid, ctx->d_result + 1 + k));
            }
        }
    }
    if (batched) {
        const int tok = prof_begin(ctx);
        k_reduce_grad<<<P * npass, 256, 0, ctx->stream>>>(ctx->d_partial, seg, grid, P, npass,
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
    if (N <= kSmallMaxQubits) {
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
