// refapi.cpp -- FOR-QAOA's single-device C++ API (include/state.h, graph.h,
// rzz.h, rx.h, swap.h, utils.h of the reference) on top of the C ABI.
// Same names, arguments and meaning; errors throw fq::Error instead of
// calling exit() (include/helper_cuda.h:582-595 in the reference).
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "refapi/graph.h"
#include "refapi/rx.h"
#include "refapi/rzz.h"
#include "refapi/state.h"
#include "refapi/swap.h"
#include "refapi/utils.h"

// src/utils.cpp:19-27
struct timeval start;
struct timeval end_;
unsigned long diff;
float rx_gate_time_ms;
float csqs_time_ms;
float transmission_time_ms;

// src/rzz.cu:24
Fp initialAmp;

namespace {

void check(int status, const char* what) {
    if (status != FQ_OK)
        throw fq::Error(status, std::string(what) + ": " + fq_status_string(status) + " (" +
                                    fq_last_error() + ")");
}

fq_ctx* ctx_of(const State& q) {
    if (!q.gpus || !q.gpus[0].ctx) throw fq::Error(FQ_ERR_INVALID, "state not created");
    return q.gpus[0].ctx;
}

}  // namespace

// src/state.cpp:89-159 (D = 0): one device, its non-blocking stream, the
// 16*2^N state, the host mirror (calloc, |0..0> in it) and |0..0> on the
// device.
State createState(int N, int D, int B, int C) {
    if (D != 0)
        throw fq::Error(FQ_ERR_UNSUPPORTED,
                        "createState: D=" + std::to_string(D) +
                            " needs the multi-device path, which this library does not provide");
    if (N < 1 || N > 33) throw fq::Error(FQ_ERR_INVALID, "createState: N out of range [1,33]");
    if (C < 1) throw fq::Error(FQ_ERR_INVALID, "createState: C must be >= 1");
    State q;
    memset(&q, 0, sizeof(q));
    q.numQubits = N;
    q.numDevice = 1;
    q.numQubitsPerDevice = N;
    q.numAmpsPerDevice = 1ull << N;
    q.stateSizePerDevice = q.numAmpsPerDevice * sizeof(Complex);
    q.numQubitsPerBuffer = B;
    q.numAmpsPerBuf = (B >= 0 && B < 63) ? (1ull << B) : 0;
    q.bufSize = q.numAmpsPerBuf * sizeof(Complex);
    q.chunkQubits = C;
    q.gpus = (GPUState*)calloc(1, sizeof(GPUState));
    if (!q.gpus) throw fq::Error(FQ_ERR_OOM, "createState: host allocation failed");
    fq_ctx* ctx = nullptr;
    int st = fq_ctx_create(0, nullptr, &ctx);
    if (st != FQ_OK) {
        free(q.gpus);
        check(st, "createState");
    }
    q.gpus[0].ctx = ctx;
    q.gpus[0].compute_stream = (cudaStream_t)fq_ctx_stream(ctx);
    void* sv = nullptr;
    st = fq_state_alloc(ctx, N, &sv);
    if (st != FQ_OK) {
        fq_ctx_destroy(ctx);
        free(q.gpus);
        check(st, "createState");
    }
    q.gpus[0].dState = (Complex*)sv;
    q.hState = (Complex*)calloc(q.numAmpsPerDevice, sizeof(Complex));
    if (!q.hState) {
        fq_state_free(ctx, sv);
        fq_ctx_destroy(ctx);
        free(q.gpus);
        throw fq::Error(FQ_ERR_OOM, "createState: host state allocation failed");
    }
    q.hState[0].real = 1;
    ncclWarnup(q);
    stateInitDeviceState(q);
    prepare(q, C);
    return q;
}

void destroyState(const State& q) {
    if (!q.gpus) return;
    fq_ctx* ctx = q.gpus[0].ctx;
    if (ctx) {
        fq_state_free(ctx, q.gpus[0].dState);
        fq_ctx_destroy(ctx);
    }
    free(q.gpus);
    free(q.hState);
}

void stateCpyDeviceToHost(const State& q) {
    check(fq_state_to_host(ctx_of(q), q.gpus[0].dState, q.numQubits, q.hState),
          "stateCpyDeviceToHost");
}

void stateCpyHostToDevice(const State& q) {
    check(fq_state_from_host(ctx_of(q), q.gpus[0].dState, q.numQubits, q.hState),
          "stateCpyHostToDevice");
}

void stateInitDeviceState(const State& q) {
    check(fq_state_init_basis0(ctx_of(q), q.gpus[0].dState, q.numQubits), "stateInitDeviceState");
    check(fq_ctx_synchronize(ctx_of(q)), "stateInitDeviceState");
}

// src/state.cpp:222-318: with one device there is nothing to exchange.
void ncclWarnup(State&) {}

// src/state.cpp:162-196 allocates per-call device scratch; the context owns
// all scratch here, so only the chunk size is recorded.
void prepare(State& q, int C) {
    if (C < 1) throw fq::Error(FQ_ERR_INVALID, "prepare: C must be >= 1");
    q.chunkQubits = C;
}

// src/graph.cpp:23-44
ull* init1DGraph(const State& q) {
    ull* g = (ull*)calloc(q.numQubits > 0 ? q.numQubits : 1, sizeof(ull));
    if (!g) throw fq::Error(FQ_ERR_OOM, "init1DGraph");
    return g;
}

void free1DGraph(ull* graph) { free(graph); }

void addEdgeTo1DGraph(const State& q, ull* graph, int qubit1, int qubit2) {
    if (qubit1 < 0 || qubit2 < 0 || qubit1 >= q.numQubits || qubit2 >= q.numQubits ||
        qubit1 == qubit2)
        throw fq::Error(FQ_ERR_INVALID, "addEdgeTo1DGraph: bad vertices");
    if (qubit1 > qubit2) std::swap(qubit1, qubit2);
    graph[qubit1] |= 1ull << qubit2;
}

// src/graph.cpp:46-67
Fp* init2DGraph(const State& q) {
    Fp* g = (Fp*)calloc((size_t)q.numQubits * q.numQubits, sizeof(Fp));
    if (!g) throw fq::Error(FQ_ERR_OOM, "init2DGraph");
    return g;
}

void addEdgeTo2DGraph(const State& q, Fp* graph, int qubit1, int qubit2, Fp weight) {
    const int n = q.numQubits;
    if (qubit1 < 0 || qubit2 < 0 || qubit1 >= n || qubit2 >= n || qubit1 == qubit2)
        throw fq::Error(FQ_ERR_INVALID, "addEdgeTo2DGraph: bad vertices");
    if (qubit1 > qubit2) std::swap(qubit1, qubit2);
    graph[qubit1 * n + qubit2] = weight;
}

void free2DGraph(Fp* graph) { free(graph); }

// src/rzz.cu:26-28
void initH(const State& q) { initialAmp = fq_init_amp(q.numQubits); }

// src/rzz.cu:173-206
void rotationCompressionWeighted(State& q, const Fp angle, const Fp* graph,
                                 const bool isFirstLayer) {
    check(fq_cost_phase(ctx_of(q), q.gpus[0].dState, q.numQubits, angle, graph, isFirstLayer,
                        initialAmp),
          "rotationCompressionWeighted");
}

// Unit weights from the 1D neighbour masks, through the same exact integer
// cost path.
void rotationCompressionUnweighted(const State& q, Fp angle, ull* graph, bool isFirstLayer) {
    const int n = q.numQubits;
    std::vector<Fp> g((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if ((graph[i] >> j) & 1ull) g[i * n + j] = 1.0;
    check(fq_cost_phase(ctx_of(q), q.gpus[0].dState, n, angle, g.data(), isFirstLayer,
                        initialAmp),
          "rotationCompressionUnweighted");
}

// src/rx.cu:118-174: targets must lie in the chunk; chunks are up to 13
// qubits here (the reference is limited to its compile-time CHUNK_QUBIT).
void multiRotateX(State& q, vector<int>& targetQubits, const int gate_size, const Fp angle) {
    if (gate_size < 0 || gate_size > (int)targetQubits.size())
        throw fq::Error(FQ_ERR_INVALID, "multiRotateX: gate_size exceeds the target list");
    const int chunk = std::min(13, q.numQubits);
    check(fq_rx_chunk(ctx_of(q), q.gpus[0].dState, q.numQubits, chunk, targetQubits.data(),
                      gate_size, angle),
          "multiRotateX");
}

void rotateX(const State& q, const int targetQubit, const Fp angle) {
    check(fq_rx_targets(ctx_of(q), q.gpus[0].dState, q.numQubits, &targetQubit, 1, angle),
          "rotateX");
}

// src/swap.cu:104-202 (single-device branch :166-200)
void swap_gate_conti(const State& q, const int SwapOut, const int SwapIn, const int numSwap) {
    check(fq_swap_blocks(ctx_of(q), q.gpus[0].dState, q.numQubits, SwapOut, SwapIn, numSwap),
          "swap_gate_conti");
}

void swap_gate(const State& q, const int targ0, const int targ1) {
    const int a = std::min(targ0, targ1), b = std::max(targ0, targ1);
    if (a == b) return;
    check(fq_swap_blocks(ctx_of(q), q.gpus[0].dState, q.numQubits, a, b, 1), "swap_gate");
}

// src/swap.cu:27-50
void mapping_after_swap_conti(const State& q, Fp* graph, const int SwapOut, const int SwapIn,
                              const int numSwap) {
    check(fq_relabel_graph(graph, q.numQubits, SwapOut, SwapIn, numSwap),
          "mapping_after_swap_conti");
}

// The same relabel on 1D neighbour masks.
void mapping_after_swap_conti(const State& q, ull* graph, const int SwapOut, const int SwapIn,
                              const int numSwap) {
    const int n = q.numQubits;
    if (numSwap < 0 || SwapOut < 0 || SwapOut + numSwap > SwapIn || SwapIn + numSwap > n)
        throw fq::Error(FQ_ERR_INVALID, "mapping_after_swap_conti: bad block swap");
    std::vector<int> lab(n);
    for (int b = 0; b < n; b++) lab[b] = b;
    for (int m = 0; m < numSwap; m++) std::swap(lab[SwapOut + m], lab[SwapIn + m]);
    std::vector<ull> out(n, 0);
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if ((graph[i] >> j) & 1ull) {
                int a = lab[i], b = lab[j];
                if (a > b) std::swap(a, b);
                out[a] |= 1ull << b;
            }
    for (int i = 0; i < n; i++) graph[i] = out[i];
}
