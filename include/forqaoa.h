/*
 * forqaoa.h -- C ABI of the FOR-QAOA B200 library (libforqaoa.so).
 *
 * A QAOA Max-Cut state-vector simulator for one NVIDIA B200 (sm_100a),
 * written from scratch with the semantics of FOR-QAOA's single-device path
 * (D = 0).  Every entry point takes plain pointers and sizes and returns an
 * int status (FQ_OK = 0); nothing here exits the process.  On failure,
 * fq_last_error() gives a message for the calling thread.
 *
 * Conventions (FOR-QAOA's own, see each function):
 *  - a state is 2^N complex128 amplitudes, AoS {re, im}, in device memory;
 *    bit q of the amplitude index is qubit q;
 *  - a graph is an N x N row-major FP64 matrix on the HOST whose strict
 *    upper triangle holds the edge weights, 0 = no edge (include/graph.h:
 *    init2DGraph / addEdgeTo2DGraph, src/graph.cpp:46-64);
 *  - cost layer: psi(z) *= exp(+i*gamma*S(z)/2), S(z) = sum over edges of
 *    (+w if the edge is cut else -w)  (src/rzz.cu:121-156);
 *  - mixer layer: RX(beta) = exp(-i*beta*X/2) on each qubit (src/rx.cu:32-53);
 *  - <C> is the expected cut weight sum_z |psi(z)|^2 C(z), C = (S + W)/2.
 * All work is asynchronous on the context's stream unless a function says
 * it returns a host value.
 */
#ifndef FORQAOA_H
#define FORQAOA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FQ_OK 0
#define FQ_ERR_INVALID 1     /* bad argument (size, pointer, graph, angle) */
#define FQ_ERR_UNSUPPORTED 2 /* valid in the reference but not on this path (D > 0) */
#define FQ_ERR_CUDA 3        /* a CUDA runtime call failed */
#define FQ_ERR_OOM 4         /* device or host memory exhausted / over budget */
#define FQ_ERR_TIMEOUT 5     /* a bounded device-side wait gave up */
#define FQ_ERR_BUSY 6        /* resource in use (serving admission) */

typedef struct fq_ctx fq_ctx;

/* ---- status / version ------------------------------------------------ */
const char* fq_status_string(int status);
const char* fq_last_error(void);
int fq_version(void);

/* ---- context ------------------------------------------------------------
 * One context per (device, stream).  It owns the small device scratch used
 * by the kernels (weights, phase tables, reduction partials) and pinned
 * staging memory, allocated once at creation.  stream == NULL creates a
 * private non-blocking stream (the reference's compute_stream,
 * src/state.cpp:139). */
int fq_ctx_create(int device, void* stream, fq_ctx** out);
int fq_ctx_destroy(fq_ctx* ctx);
int fq_ctx_synchronize(fq_ctx* ctx);
/* Self-test of the failure path (no counterpart in the reference, whose
 * waits are unbounded): enqueues one kernel that waits, with the bounded
 * wait of the TMA pipelines (2^16 polls instead of 2^18: 0.26 s instead of
 * about 1 s on B200), on a barrier
 * nothing completes.  The wait gives up, the next synchronising call (e.g.
 * fq_ctx_synchronize) returns FQ_ERR_TIMEOUT and clears the flag, and the
 * context stays usable. */
int fq_ctx_selftest_wait(fq_ctx* ctx);
void* fq_ctx_stream(fq_ctx* ctx);
/* Number of library kernels this context has launched so far. */
int fq_ctx_kernel_launches(fq_ctx* ctx, long long* count);
/* Resident CTAs per SM and SM count the streaming kernels are sized for. */
int fq_ctx_device_info(fq_ctx* ctx, int* num_sms, int* ctas_per_sm);

/* Per-kernel timing.  While enabled, every library kernel launch is
 * bracketed by CUDA events on the context's stream; fq_ctx_profile
 * synchronises the stream and returns, for one kernel kind, the summed
 * device time (ms), the launch count and the summed algorithmic HBM bytes
 * (bytes the kernel must move: 16 per amplitude read, 16 per amplitude
 * written).  Kinds: */
#define FQ_KIND_PHASE_PASS 0    /* engine tile pass with a cost phase and RX: a fused
                                   two-layer pass, or a later layer's first pass */
#define FQ_KIND_MIXER_PASS 1    /* engine tile pass with RX only */
#define FQ_KIND_COST 2          /* fq_cost_phase */
#define FQ_KIND_RX 3            /* fq_rx_chunk / fq_rx_targets */
#define FQ_KIND_SWAP 4          /* fq_swap_blocks */
#define FQ_KIND_EXPECT 5        /* <C> / cut diagonal sweeps */
#define FQ_KIND_OTHER 6         /* tables, reductions, permutations, small instances */
#define FQ_KIND_ADJOINT 7       /* reverse-sweep passes over state and costate */
#define FQ_KIND_INIT_PASS 8     /* engine's layer-0 pass: launch-control init, write-only */
#define FQ_KIND_COUNT 9
int fq_ctx_set_profiling(fq_ctx* ctx, int enable);
int fq_ctx_profile(fq_ctx* ctx, int kind, double* total_ms, long long* launches,
                   double* bytes);
int fq_ctx_profile_reset(fq_ctx* ctx);

/* ---- state memory (include/state.h, src/state.cpp) ---------------------- */
/* cudaMalloc of 16 * 2^N bytes; replaces createState's allocation
 * (src/state.cpp:89-159, D = 0). */
int fq_state_alloc(fq_ctx* ctx, int N, void** sv);
int fq_state_free(fq_ctx* ctx, void* sv);
/* |0...0>: replaces stateInitDeviceState (src/state.cpp:198-219). */
int fq_state_init_basis0(fq_ctx* ctx, void* sv, int N);
/* Synchronous copies: replace stateCpyDeviceToHost / stateCpyHostToDevice
 * (src/state.cpp:320-336). */
int fq_state_to_host(fq_ctx* ctx, const void* sv, int N, void* host);
int fq_state_from_host(fq_ctx* ctx, void* sv, int N, const void* host);

/* ---- reference-path kernels (one per reference launcher) ---------------- */
/* pow(1/sqrt(2), N): replaces initH (src/rzz.cu:26-28). */
double fq_init_amp(int N);
/* Cost layer with launch-control init: replaces rotationCompressionWeighted
 * (src/rzz.cu:173-206, kernel :121-156).  is_first_layer != 0 writes
 * psi = phase * init_amp without reading psi; otherwise psi *= phase. */
int fq_cost_phase(fq_ctx* ctx, void* sv, int N, double angle,
                  const double* graph_upper, int is_first_layer, double init_amp);
/* RX(angle) on each of targets[0..gate_size): replaces multiRotateX
 * (src/rx.cu:118-174).  chunk_qubits is the reference's CHUNK_QUBIT (the
 * chunk the targets live in, 1..13); every target must be < chunk_qubits. */
int fq_rx_chunk(fq_ctx* ctx, void* sv, int N, int chunk_qubits, const int* targets,
                int gate_size, double angle);
/* RX(angle) on each listed qubit, any target < N: replaces rotateX, which
 * the reference declares (include/rx.h:25) but does not define. */
int fq_rx_targets(fq_ctx* ctx, void* sv, int N, const int* targets, int n, double angle);
/* Exchange qubit blocks [swap_out, swap_out+k) <-> [swap_in, swap_in+k) of
 * every index: replaces swap_gate_conti's D = 0 path (src/swap.cu:104-202,
 * kernel :76-102).  Requires swap_out + k <= swap_in and swap_in + k <= N. */
int fq_swap_blocks(fq_ctx* ctx, void* sv, int N, int swap_out, int swap_in,
                   int num_swap);
/* Host-side graph relabel matching fq_swap_blocks: replaces
 * mapping_after_swap_conti (src/swap.cu:27-50).  Returns a status. */
int fq_relabel_graph(double* graph_upper, int N, int swap_out, int swap_in,
                     int num_swap);

/* ---- sharded state (D > 0) ------------------------------------------------
 * A state of N qubits split over 2^D devices by its top D index bits: the
 * shard of rank r holds the 2^(N-D) amplitudes whose physical qubits
 * N-D..N-1 read r (1 <= D <= 8, N-D >= 13, rank < 2^D).  graph_upper is
 * the N x N graph in the shards' current physical order.  A layer is
 * fq_shard_layer on every shard, then an all-to-all of equal chunks (chunk
 * d of every shard to rank d; it swaps qubit blocks [N-2D, N-D) and
 * [N-D, N)), then fq_rx_targets on qubits N-2D..N-D-1 of every shard and
 * fq_relabel_graph(graph, N, N-2D, N-D, D); for-qaoa_b200/sharded.py
 * drives it over torch.distributed.
 * Replaces the D > 0 paths of rotationCompressionWeighted, multiRotateX and
 * swap_gate_conti (src/rzz.cu:173-206, src/rx.cu:118-174,
 * src/swap.cu:104-165,223-345). */
/* Cost phase of angle gamma (first_layer != 0: launch-control init with
 * fq_init_amp(N), the shard is written without being read) followed by
 * RX(beta) on the shard's local qubits 0..N-D-1. */
int fq_shard_layer(fq_ctx* ctx, void* shard, int N, int D, int rank,
                   const double* graph_upper, double gamma, double beta, int first_layer);
/* RX(beta_prev) on local qubits N-2D..N-D-1 (the qubits the previous
 * layer's all-to-all swapped in), then fq_shard_layer with first_layer = 0:
 * the same result as fq_rx_targets followed by fq_shard_layer.  For D <= 4
 * and N-D >= 24 (the layer's first pass then tiles the top local qubits)
 * the rotation runs inside that pass, one HBM sweep fewer per layer; a
 * P-layer circuit then calls fq_shard_layer once, this function P-1 times,
 * and fq_rx_targets once after the last all-to-all. */
int fq_shard_layer_after_swap(fq_ctx* ctx, void* shard, int N, int D, int rank,
                              const double* graph_upper, double gamma, double beta,
                              double beta_prev);
/* <C> summed over this shard's amplitudes (the shards' partials add up to
 * <C>); synchronises the stream. */
int fq_shard_expectation(fq_ctx* ctx, const void* shard, int N, int D, int rank,
                         const double* graph_upper, double* partial);

/* ---- fused engine --------------------------------------------------------
 * The whole P-layer circuit from |+>^N in as few HBM sweeps as possible:
 * cost phase, launch-control init and the first 12 RX gates share one
 * sweep, the remaining qubits are rotated in strided tiles, no block swaps.
 * The state is left in LOGICAL qubit order.  If energy != NULL, <C> is
 * computed in the last sweep and written to *energy (host), which
 * synchronises the stream. */
int fq_qaoa_forward(fq_ctx* ctx, void* sv, int N, int P, const double* graph_upper,
                    const double* gammas, const double* betas, double* energy);
/* <C> and its gradient with respect to every gamma_k and beta_k of the
 * P-layer circuit from |+>^N, by adjoint differentiation: one forward sweep,
 * lambda = C psi, and one reverse sweep that moves psi and lambda back
 * through the exact inverse of each layer (no stored intermediate states):
 *   dE/dbeta_k = Im <lambda|sum_q X_q|psi>,  dE/dgamma_k = -Im <lambda|S|psi>.
 * sv and costate are device workspaces of 2^N amplitudes each (contents
 * unspecified on return; unused, may be NULL, for N <= FQ_SMALL_MAX_QUBITS,
 * where the whole instance runs in shared memory: one CTA's up to 12
 * qubits, a cluster of 2^(N-12) CTAs above).  Writes *energy, grad_gamma[P],
 * grad_beta[P] (host) and synchronises. */
#define FQ_SMALL_MAX_QUBITS 15
int fq_qaoa_energy_grad(fq_ctx* ctx, void* sv, void* costate, int N, int P,
                        const double* graph_upper, const double* gammas, const double* betas,
                        double* energy, double* grad_gamma, double* grad_beta);
/* <C> of a state (read-only sweep).  Writes *energy (host); synchronises. */
int fq_expectation(fq_ctx* ctx, const void* sv, int N, const double* graph_upper,
                   double* energy);
/* Cut values C(z) for every z as float64 (exact for integer weights). */
int fq_cut_diagonal(fq_ctx* ctx, void* out, int N, const double* graph_upper);
/* dst[y] = src[x], y having bit perm[b] equal to bit b of x (out of place). */
int fq_permute_qubits(fq_ctx* ctx, const void* src, void* dst, int N, const int* perm);
/* Compares two device states: out[0] = max|a-b|, out[1] = max|b|,
 * out[2] = ||a-b||_2, out[3] = ||b||_2 (host, synchronises).  For checks of
 * full-size states without copying them to the host.  No counterpart in the
 * reference. */
int fq_state_diff(fq_ctx* ctx, const void* a, const void* b, int N, double* out);
/* <C> of a device state without allocating any device memory, for callers
 * that cannot call cudaMalloc (their device memory belongs to another
 * allocator, or they cannot afford cudaMalloc's implicit synchronisation).
 * No counterpart in the reference.  Needs no fq_ctx: sv is the caller's
 * state, graph_upper the host graph, stream the caller's stream (NULL = the
 * legacy default stream); writes *energy (host) and synchronises the stream.
 * All scratch (weights, partial sums, result) lives in one fixed 32 KiB
 * device array that every GPU loading the library keeps until exit; N must
 * be in [2, 33].  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress) and should come before any stream capture.
 * Calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int fq_expectation_noalloc(const void* sv, int N, const double* graph_upper, double* energy,
                           void* stream);
/* Physical -> logical qubit map the reference schedule leaves after P layers
 * with chunk size C (src/Weighted.cpp:97-138): label_map[b] = logical qubit
 * at physical position b.  Host only. */
int fq_reference_label_map(int N, int C, int P, int* label_map);

/* ---- serving -------------------------------------------------------------
 * A server admits energy+gradient requests (fq_qaoa_energy_grad's
 * computation) and runs them with continuous batching on one device:
 * requests with N <= FQ_SMALL_MAX_QUBITS are packed one per CTA (N <= 12)
 * or one per cluster of CTAs into batched launches, larger ones overlap on
 * `lanes` independent streams.  Requests of one session (an optimiser loop
 * on one graph) run in submission order and, for larger N, keep their state and costate buffers (2 x 16 x 2^N bytes)
 * resident between steps; resident buffers stay within hbm_budget_bytes,
 * idle sessions being released least recently used first.  No counterpart
 * in the reference, whose CLI runs one circuit per process
 * (src/Weighted.cpp:58-160). */
#define FQ_SERVE_MAX_LAYERS 16

typedef struct fq_server fq_server;

typedef struct fq_request {
    uint64_t session;           /* caller's session id */
    int N, P;                   /* 2 <= N <= 33, 1 <= P <= FQ_SERVE_MAX_LAYERS */
    const double* graph_upper;  /* N*N row-major, upper triangle read; copied */
    const double* gammas;       /* P; copied */
    const double* betas;        /* P; copied */
} fq_request;

typedef struct fq_result {
    uint64_t ticket, session;
    int N, P, status, pad;
    double energy;
    double grad_gamma[FQ_SERVE_MAX_LAYERS];
    double grad_beta[FQ_SERVE_MAX_LAYERS];
    double t_submit, t_start, t_done; /* steady clock, seconds */
} fq_result;

typedef struct fq_server_counters {
    long long pending;           /* submitted, not yet polled as done */
    long long kernel_launches;   /* kernels launched so far */
    long long batched_requests;  /* requests run in one-CTA batches */
    long long lane_requests;     /* requests run on lanes */
    long long resident_sessions; /* sessions holding device buffers */
    double resident_bytes;       /* their bytes */
} fq_server_counters;

/* Starts a server with its scheduler thread on `device`. */
int fq_server_create(int device, double hbm_budget_bytes, int lanes, fq_server** out);
/* Finishes every submitted request, then frees everything. */
int fq_server_destroy(fq_server* server);
/* Queues a request (validated and copied); *ticket identifies its result.
 * FQ_ERR_OOM if one session of this N exceeds the budget. */
int fq_server_submit(fq_server* server, const fq_request* request, uint64_t* ticket);
/* Moves up to max_results finished results to out (completion order),
 * waiting up to wait_ms for the first; *n_out = number moved.  A non-OK
 * return reports the first failure the scheduler met (per-request status is
 * in each result). */
int fq_server_poll(fq_server* server, fq_result* out, int max_results, int* n_out,
                   int wait_ms);
/* Releases a session's resident buffers (after its running and queued steps,
 * if any). */
int fq_server_close_session(fq_server* server, uint64_t session);
int fq_server_stats(fq_server* server, fq_server_counters* counters);

#ifdef __cplusplus
}
#endif
#endif
