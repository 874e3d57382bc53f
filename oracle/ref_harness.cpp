// ref_harness.cpp -- drives the UNMODIFIED FOR-QAOA single-device API
// (compiled from the reference's own sources by oracle/Makefile.ref) through
// the same schedule as its `main` (src/Weighted.cpp:81-138), but with the
// graph and per-layer angles read from a file, and dumps the final state.
//
// TEST INFRASTRUCTURE ONLY: used to produce golden vectors that pin the CPU
// oracle to the reference's actual output.  Nothing in the product links it.
//
// Input file (little endian):  int32 N, C, P; float64 graph[N*N] (upper
// triangle used); float64 gammas[P]; float64 betas[P].
// Output file: complex128 state[2^N] in the reference's physical order,
// then float64 graph_final[N*N] (the relabelled graph).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "graph.h"
#include "rx.h"
#include "rzz.h"
#include "state.h"
#include "swap.h"

static void die(const char* m) {
    fprintf(stderr, "ref_harness: %s\n", m);
    exit(2);
}

int main(int argc, char** argv) {
    if (argc != 3) die("usage: ref_harness <in.bin> <out.bin>");
    FILE* f = fopen(argv[1], "rb");
    if (!f) die("cannot open input");
    int hdr[3];
    if (fread(hdr, sizeof(int), 3, f) != 3) die("short header");
    const int N = hdr[0], C = hdr[1], P = hdr[2];
    // The reference's RX kernel holds 2^CHUNK_QUBIT amplitudes in a static
    // shared buffer and indexes it with the subcircuit targets (rx.cu:61,
    // 39-43); a chunk wider than CHUNK_QUBIT would index past it.  Its RX and
    // swap grids also use 32-bit products (rx.cu:62, swap.cu:78), so keep
    // N <= 31.
    if (N < 2 || N > 31 || C < 1 || C > CHUNK_QUBIT || N < CHUNK_QUBIT || P < 1)
        die("unsupported sizes for the reference build");
    std::vector<double> g(N * N), gam(P), bet(P);
    if (fread(g.data(), sizeof(double), N * N, f) != (size_t)(N * N)) die("short graph");
    if (fread(gam.data(), sizeof(double), P, f) != (size_t)P) die("short gammas");
    if (fread(bet.data(), sizeof(double), P, f) != (size_t)P) die("short betas");
    fclose(f);

    State qureg = createState(N, 0, C, C);  // B only sizes the unused D>0 buffer
    Fp* graph = init2DGraph(qureg);
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++)
            if (g[i * N + j] != 0) addEdgeTo2DGraph(qureg, graph, i, j, g[i * N + j]);
    initH(qureg);

    // Weighted.cpp:97-108
    std::vector<std::vector<int>> subcirs;
    for (int i = 0; i < N; i += C) {
        std::vector<int> q;
        for (int j = i; j < i + C && j < N; ++j) q.push_back(j);
        subcirs.push_back(q);
    }
    const int num_subcir = (int)subcirs.size();
    // Weighted.cpp:115-138 with per-layer angles
    for (int p = 0; p < P; p++) {
        rotationCompressionWeighted(qureg, gam[p], graph, p == 0);
        int swapIn_index = 0;
        for (int i = 0; i < num_subcir; i++) {
            multiRotateX(qureg, subcirs[0], subcirs[i].size(), bet[p]);
            if (i < num_subcir - 1) {
                swapIn_index += subcirs[i].size();
                swap_gate_conti(qureg, 0, swapIn_index, subcirs[i + 1].size());
                mapping_after_swap_conti(qureg, graph, 0, swapIn_index,
                                         subcirs[i + 1].size());
            }
        }
    }
    // The work ran on a non-blocking stream; the reference's copy uses the
    // legacy stream, so synchronise the device first.
    if (cudaDeviceSynchronize() != cudaSuccess) die("device error");
    stateCpyDeviceToHost(qureg);

    FILE* o = fopen(argv[2], "wb");
    if (!o) die("cannot open output");
    fwrite(qureg.hState, sizeof(Complex), 1ull << N, o);
    fwrite(graph, sizeof(double), N * N, o);
    fclose(o);
    free2DGraph(graph);
    destroyState(qureg);
    printf("ref_harness: N=%d C=%d P=%d CHUNK_QUBIT=%d ok\n", N, C, P, CHUNK_QUBIT);
    return 0;
}
