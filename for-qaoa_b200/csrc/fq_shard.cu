// fq_shard.cu -- one layer of the circuit on one shard of a state split
// over 2^D devices (fq_shard_layer, fq_shard_expectation).
//
// A state of N qubits is split by its top D index bits: the shard of rank r
// holds the 2^(N-D) amplitudes whose physical qubits N-D..N-1 read r.  The
// tile passes run on the shard as on a whole state of N-D qubits, except
// that cut values take the rank's bits as fixed bits (PassArgs::goff), so
// the cost phase and <C> see the whole graph.  RX on the D top qubits needs
// the other shards: the caller exchanges them (an all-to-all that swaps
// qubit blocks [N-2D, N-D) and [N-D, N)) and rotates the swapped-in qubits
// with fq_rx_targets; the driver is for-qaoa_b200/sharded.py.  This
// replaces the D > 0 paths of the reference's cost, mixer and swap
// launchers (src/rzz.cu:173-206, src/rx.cu:118-174, src/swap.cu:104-165,
// 223-345).
#include <math.h>

#include <vector>

#include "fq_engine.h"
#include "fq_launch.cuh"

using namespace fq;

namespace {

int check_shard(void* sv, int N, int D, int rank) {
    FQ_CHECK(D >= 1 && D <= 8, FQ_ERR_INVALID, "D=%d out of range [1,8]", D);
    FQ_CHECK(N - D >= kTileBits + 1 && N <= kMaxQubits, FQ_ERR_INVALID,
             "N=%d, D=%d: a shard needs at least %d qubits", N, D, kTileBits + 1);
    FQ_CHECK(rank >= 0 && rank < (1 << D), FQ_ERR_INVALID, "rank %d out of range for D=%d", rank,
             D);
    return check_state(sv, N - D);
}

// Pass arguments for this rank's shard: the weights and fixed bits of the
// whole N-qubit graph, the tiles of the shard.
PassArgs shard_args(fq_ctx* ctx, void* sv, int N, int D, int rank, const GraphPrep& g) {
    PassArgs A = base_args(ctx, sv, N, g);
    A.ntiles = 1ll << (N - D - kTileBits);
    A.goff = (i64)rank << (N - D);
    return A;
}

// One layer on a shard; pre != nullptr: first RX(*pre) on local qubits
// n-D..n-1, inside the first pass when its tile holds them in tile bits
// 8..11 (the layout-L0 register bits), else as a pass of its own.
int shard_layer(fq_ctx* ctx, void* shard, int N, int D, int rank, const double* graph,
                double gamma, double beta, int first_layer, const double* pre) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_shard(shard, N, D, rank));
    FQ_CHECK(isfinite(gamma) && isfinite(beta), FQ_ERR_INVALID, "non-finite angle");
    FQ_CHECK(!pre || isfinite(*pre), FQ_ERR_INVALID, "non-finite angle");
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    const int n = N - D;
    const std::vector<PassPlan> plan = plan_layer(n);
    unsigned pre_mask = 0;
    if (pre) {
        const PassPlan& f = plan[0];
        const int k = kTileBits - f.l;  // the first pass's strided targets: qubits a..a+k-1
        if (D <= 4 && f.l < kTileBits && f.a + k == n && k >= D)
            pre_mask = ((1u << D) - 1) << (4 - D);  // tile bits 12-D..11 = qubits n-D..n-1
        else
            FQ_TRY(rx_mask(ctx, shard, n, ((1ull << D) - 1) << (n - D), *pre));
    }
    int gm;
    double gx, f;
    gate_params(beta, gm, gx, f);
    // The reduced gates of the n local qubits are folded into the phase; the
    // D top qubits are rotated later in full form (fq_rx_targets, or the
    // next layer's first pass).
    const double scale = pow(f, n) * (first_layer ? fq_init_amp(N) : 1.0);
    const int nhi = g.integer ? engine_nhi(g) : 0;
    if (g.integer) {
        if (nhi > 0)
            FQ_TRY(launch_table2(ctx, g, gamma));
        else
            FQ_TRY(launch_table(ctx, g, gamma, scale));
    }
    for (size_t i = 0; i < plan.size(); i++) {
        PassArgs A = shard_args(ctx, shard, N, D, rank, g);
        A.l = plan[i].l;
        A.a = plan[i].a;
        A.tmask = plan[i].tmask;
        A.gx = gx;
        if (nhi > 0) set_table_args(A, g, gamma, scale);
        A.tree = phase_tree_ok(g, gamma) ? 1 : 0;
        A.gamma = gamma;
        A.scale = g.integer ? 1.0 : scale;
        if (i == 0 && pre_mask) {  // the formula and operand order of rx_mask's passes
            A.pre_mask = pre_mask;
            A.pc = cos(*pre / 2);
            A.ps = sin(*pre / 2);
        }
        if (i == 0)
            FQ_TRY(dispatch_phase_pass(ctx, g.integer, first_layer ? PH_INIT : PH_MUL, gm, A));
        else
            FQ_TRY(dispatch_rx(ctx, g.integer, gm, false, A));
    }
    return FQ_OK;
}

}  // namespace

extern "C" {

int fq_shard_layer(fq_ctx* ctx, void* shard, int N, int D, int rank, const double* graph,
                   double gamma, double beta, int first_layer) {
    return shard_layer(ctx, shard, N, D, rank, graph, gamma, beta, first_layer, nullptr);
}

int fq_shard_layer_after_swap(fq_ctx* ctx, void* shard, int N, int D, int rank,
                              const double* graph, double gamma, double beta, double beta_prev) {
    return shard_layer(ctx, shard, N, D, rank, graph, gamma, beta, 0, &beta_prev);
}

int fq_shard_expectation(fq_ctx* ctx, const void* shard, int N, int D, int rank,
                         const double* graph, double* partial) {
    FQ_TRY(validate_ctx(ctx));
    FQ_TRY(check_shard((void*)shard, N, D, rank));
    FQ_CHECK(partial != nullptr, FQ_ERR_INVALID, "null output pointer");
    GraphPrep g;
    FQ_TRY(setup_graph(ctx, graph, N, g));
    PassArgs A = shard_args(ctx, (void*)shard, N, D, rank, g);
    FQ_TRY(dispatch_readonly(ctx, g.integer, false, A));
    FQ_TRY(reduce_to_result(ctx, pass_grid(ctx, A, PH_NONE, false)));
    return read_result(ctx, partial);
}

}  // extern "C"
