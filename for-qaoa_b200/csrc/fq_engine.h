// fq_engine.h -- host-side pieces of the fused engine shared by the forward
// circuit (fq_engine.cu) and the gradient (fq_grad.cu).
#pragma once

#include <vector>

#include "fq_ctx.h"
#include "fq_pass.cuh"
#include "fq_small.h"

namespace fq {

// One pass of a layer: tile bits 0..l-1 = physical 0..l-1, tile bits
// l..11 = physical a..a+11-l, RX on the tile bits of tmask.
struct PassPlan {
    int l, a;
    unsigned tmask;
};

// Passes of one layer for N >= 12: the contiguous tile over qubits 0..11
// and strided tiles over the remaining qubits (the first strided one leads
// when there are three or more passes); the first pass carries the phase.
std::vector<PassPlan> plan_layer(int N);
// Reduced RX for angle beta: gate mode, t or u, and the factor f.
void gate_params(double beta, int& gm, double& g, double& f);
PassArgs base_args(fq_ctx* ctx, void* sv, int N, const GraphPrep& g);
// High-part entries of the two-level phase table (0: use the global table).
int engine_nhi(const GraphPrep& g);
// Two-level table of powers of exp(i*gamma) in ctx->d_ptab (nhi > 0), and
// the pass arguments that read it (nhi, dlo, ntab, ph0 = scale*exp(-i*gamma*W/2)).
int launch_table2(fq_ctx* ctx, const GraphPrep& g, double gamma);
// The same for layers 0..P-1 (P <= kMaxTableLayers) in one launch, layer p's
// table at ctx->d_ptab + p * kTableStride.
int launch_tables2(fq_ctx* ctx, const GraphPrep& g, const double* gammas, int P);
void set_table_args(PassArgs& A, const GraphPrep& g, double gamma, double scale);
// FP64 weights: whether product-tree phases keep the phase arguments within
// the reference's own rounding (|gamma| * sum|w| small).  Above the bound
// each amplitude takes sincos of the reference's argument (2C - W)*gamma/2,
// which is exact for integer-valued weights.
bool phase_tree_ok(const GraphPrep& g, double gamma);
int launch_table(fq_ctx* ctx, const GraphPrep& g, double gamma, double scale);
// Whether the fused two-layer schedules run (the forward circuit's and the
// gradient's reverse sweep); FQ_FUSE=0 turns them off (one sweep per pass of
// every layer).
bool fuse_enabled();
// Fixed-order sum of n partials into one device word.
int reduce_partials(fq_ctx* ctx, const double* partial, int n, double* out_dev);
int reduce_to_result(fq_ctx* ctx, int n);
// Copies ctx->d_result[0] to *host (synchronises).
int read_result(fq_ctx* ctx, double* host);
int check_state(void* sv, int N);
// RX(angle) (full form) on every qubit whose bit is set in mask (fq_rx_targets).
int rx_mask(fq_ctx* ctx, void* sv, int N, unsigned long long mask, double angle);
int setup_graph(fq_ctx* ctx, const double* graph, int N, GraphPrep& g);
// The forward circuit (fq_qaoa_forward); skip_last stops before the last
// pass of the last layer (the gradient's turnaround pass runs it).
int engine_forward(fq_ctx* ctx, void* sv, int N, int P, const GraphPrep& g, const double* gammas,
                   const double* betas, double* energy, bool skip_last = false);
// Whether engine_forward uses the fused two-layer schedule, and the plan
// index of the last pass it runs.
bool engine_fused(const GraphPrep& g, int N, int P);
int engine_last_pass(const GraphPrep& g, int N, int P);

// The N >= 13 gradient split for asynchronous use: grad_enqueue puts every
// kernel and the final device-to-host copy of the results on ctx's stream;
// once the stream has passed that point, grad_collect assembles them.
int grad_enqueue(fq_ctx* ctx, void* sv, void* costate, int N, int P, const double* graph,
                 const double* gammas, const double* betas);
int grad_collect(fq_ctx* ctx, int N, int P, double* energy, double* grad_gamma,
                 double* grad_beta);

// k_small_jobs (fq_small.cuh) over jobs ordered by size class
// (small_class): counts[c] jobs of class c, one launch per class present;
// nmax0 = the largest N of class 0.
int launch_small_jobs(const SmallJob* jobs, const int* counts, int nmax0, cudaStream_t stream);

}  // namespace fq
