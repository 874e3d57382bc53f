// fq_ctx.h -- the context object behind fq_ctx* and host-side helpers.
#pragma once

#include <vector>

#include "fq_common.cuh"

struct fq_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 0;
    int ctas_per_sm = 2;  // resident pass CTAs per SM (64 KB tile each)
    int last_grid = 0;    // CTAs (and <C> partials) of the last tile pass launched
    // Device scratch, allocated once at creation.
    void* d_w = nullptr;          // N*N weights (int32 or float64)
    double2* d_ptab = nullptr;    // integer phase table
    double* d_partial = nullptr;  // per-CTA reduction partials
    double* d_result = nullptr;   // small device results (kResultWords)
    unsigned char* d_scratch = nullptr;  // small-instance job data (kScratchBytes)
    int* d_err = nullptr;         // kernels' error flag (nonzero: a bounded wait gave up)
    void* d_tcut = nullptr;       // per-tile cut constants of the engine's passes (grown on demand)
    size_t tcut_bytes = 0;
    long long tcut_version = -1;  // g_version the tables were built for (-1: none)
    int tcut_n = -1;              // and N
    int partial_cap = 0;
    // Pinned host staging (uploads of weights and small tables).
    unsigned char* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    double* h_result = nullptr;
    cudaEvent_t stage_evt = nullptr;
    // Graph cache: the last weights uploaded to d_w.
    std::vector<double> g_key;
    int g_n = -1;
    long long g_version = 0;  // counts uploads: d_w changed
    long long launches = 0;
    // Optional per-kernel timing (fq_ctx_set_profiling): an event pair per
    // launch, resolved when the profile is read.
    struct ProfRec {
        cudaEvent_t a, b;
        int kind;
        double bytes;
    };
    bool profiling = false;
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    double prof_ms[FQ_KIND_COUNT] = {};
    double prof_bytes[FQ_KIND_COUNT] = {};
    long long prof_count[FQ_KIND_COUNT] = {};
};

namespace fq {

constexpr int kResultWords = 4096;
constexpr size_t kScratchBytes = 1 << 20;

// Host view of a graph, prepared for the kernels.
struct GraphPrep {
    int N = 0;
    bool integer = false;      // every weight an integer, cut range fits a table
    std::vector<int> wi;       // N*N symmetric
    std::vector<double> wd;    // N*N symmetric
    long long W_int = 0;       // sum of weights (integer path)
    double W = 0;              // sum of weights
    long long cmin = 0, cmax = 0;  // range of cut values (integer path)
    long long gmax = 0;            // max over qubits of sum_v |w_uv| (integer path)
    double wabs = 0;               // sum of |w| over all edges
};

int prep_graph(const double* upper, int N, GraphPrep& g);
// Uploads the graph's weights to ctx->d_w (skipped when unchanged).
int upload_graph(fq_ctx* ctx, const GraphPrep& g, const double* upper);
// Waits until the pinned staging buffer can be rewritten.
int stage_acquire(fq_ctx* ctx);
int validate_ctx(fq_ctx* ctx);
// After a stream sync: FQ_ERR_TIMEOUT (and clears the flag) if a kernel
// recorded a bounded wait that gave up.
int check_device_error(fq_ctx* ctx);

// Profiling brackets around one kernel launch: prof_begin records the start
// event (returns a token, -1 when profiling is off), prof_end the stop event
// with the launch's kind and algorithmic HBM bytes.
int prof_begin(fq_ctx* ctx);
void prof_end(fq_ctx* ctx, int token, int kind, double bytes);

}  // namespace fq
