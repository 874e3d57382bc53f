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
// Output file (full mode): complex128 state[2^N] in the reference's physical
// order, then float64 graph_final[N*N] (the relabelled graph).
// Sample mode (`ref_harness in.bin out.bin sample idx.bin`, for states too
// large to write out; idx.bin = int64 physical indices): float64
// layer_loop_ms, norm, <C>; float64 abs2_sum_by_block[256]; complex128
// amplitude at each index; float64 graph_final[N*N].
// Either mode prints the layer loop's device time (CUDA events on the
// reference's compute stream around the loop, the host work of its
// launchers included).
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
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

// <C> = sum_z |psi_z|^2 C(z) of a state against an upper-triangular graph,
// C(z) = sum_{i<j} w_ij [z_i != z_j].  The index splits into lo (bits
// 0..l-1) and hi bits: C = C_lo(lo) + C_hi(hi) + sum_{i in lo} z_i a_i(hi)
// + b(hi), with a_i = sum_{j in hi} w_ij (1 - 2 z_j) and b = sum_{j in hi}
// z_j sum_{i in lo} w_ij, so every amplitude costs O(1) after an O(2^l)
// table per hi value.  Exact for integer weights; long double accumulation.
static void state_stats(const Complex* sv, int N, const std::vector<double>& g, double* norm,
                        double* energy, double* blocks) {
    const int l = N / 2, h = N - l;
    const long long nlo = 1ll << l, nhi = 1ll << h;
    auto w = [&](int i, int j) { return i < j ? g[i * N + j] : g[j * N + i]; };
    std::vector<double> clo(nlo);
    for (long long x = 0; x < nlo; x++) {
        double c = 0;
        for (int i = 0; i < l; i++)
            for (int j = i + 1; j < l; j++)
                if (((x >> i) ^ (x >> j)) & 1) c += w(i, j);
        clo[x] = c;
    }
    long double en = 0, nr = 0;
    std::vector<long double> bl(256, 0.0L);
    const long long per_block = N >= 8 ? (1ll << N) / 256 : 1;
#pragma omp parallel
    {
        std::vector<double> t(nlo);
        std::vector<long double> bl_t(256, 0.0L);
        long double en_t = 0, nr_t = 0;
#pragma omp for schedule(dynamic, 16)
        for (long long y = 0; y < nhi; y++) {
            double base = 0, a[64];
            for (int j = 0; j < h; j++) {
                const int zj = (y >> j) & 1;
                for (int j2 = j + 1; j2 < h; j2++)
                    if (zj ^ ((y >> j2) & 1)) base += w(l + j, l + j2);
                if (zj)
                    for (int i = 0; i < l; i++) base += w(i, l + j);
            }
            for (int i = 0; i < l; i++) {
                double s = 0;
                for (int j = 0; j < h; j++) s += ((y >> j) & 1) ? -w(i, l + j) : w(i, l + j);
                a[i] = s;
            }
            t[0] = 0;
            for (long long x = 1; x < nlo; x++) t[x] = t[x & (x - 1)] + a[__builtin_ctzll(x)];
            for (long long x = 0; x < nlo; x++) {
                const long long z = (y << l) | x;
                const Complex c = sv[z];
                const long double p = (long double)c.real * c.real + (long double)c.imag * c.imag;
                nr_t += p;
                en_t += p * (clo[x] + t[x] + base);
                bl_t[z / per_block] += p;
            }
        }
#pragma omp critical
        {
            en += en_t;
            nr += nr_t;
            for (int k = 0; k < 256; k++) bl[k] += bl_t[k];
        }
    }
    *norm = (double)nr;
    *energy = (double)en;
    for (int k = 0; k < 256; k++) blocks[k] = (double)bl[k];
}

int main(int argc, char** argv) {
    const bool sample = argc == 5 && strcmp(argv[3], "sample") == 0;
    if (argc != 3 && !sample)
        die("usage: ref_harness <in.bin> <out.bin> [sample <idx.bin>]");
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
    cudaStream_t st = qureg.gpus[0].compute_stream;
    cudaEvent_t ev0, ev1;
    if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess)
        die("event create");
    if (cudaDeviceSynchronize() != cudaSuccess) die("device error before the loop");
    cudaEventRecord(ev0, st);
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
    cudaEventRecord(ev1, st);
    // The work ran on a non-blocking stream; the reference's copy uses the
    // legacy stream, so synchronise the device first.
    if (cudaDeviceSynchronize() != cudaSuccess) die("device error");
    float loop_ms = 0;
    cudaEventElapsedTime(&loop_ms, ev0, ev1);
    stateCpyDeviceToHost(qureg);

    FILE* o = fopen(argv[2], "wb");
    if (!o) die("cannot open output");
    if (!sample) {
        fwrite(qureg.hState, sizeof(Complex), 1ull << N, o);
    } else {
        FILE* fi = fopen(argv[4], "rb");
        if (!fi) die("cannot open index file");
        std::vector<long long> idx;
        long long v;
        while (fread(&v, sizeof(v), 1, fi) == 1) {
            if (v < 0 || v >= (1ll << N)) die("index out of range");
            idx.push_back(v);
        }
        fclose(fi);
        std::vector<double> gf(graph, graph + N * N), blocks(256);
        double hdr2[3] = {loop_ms, 0, 0};
        state_stats(qureg.hState, N, gf, &hdr2[1], &hdr2[2], blocks.data());
        fwrite(hdr2, sizeof(double), 3, o);
        fwrite(blocks.data(), sizeof(double), 256, o);
        for (long long k : idx) fwrite(&qureg.hState[k], sizeof(Complex), 1, o);
    }
    fwrite(graph, sizeof(double), N * N, o);
    fclose(o);
    free2DGraph(graph);
    destroyState(qureg);
    printf("ref_harness: N=%d C=%d P=%d CHUNK_QUBIT=%d layer_loop_ms=%.3f ok\n", N, C, P,
           CHUNK_QUBIT, loop_ms);
    return 0;
}
