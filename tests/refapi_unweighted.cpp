// A program written only against the reference-style C++ API
// (include/refapi/*.h): the reference's layer loop (src/Weighted.cpp:97-138)
// on an UNWEIGHTED graph given as 64-bit neighbour masks, i.e. the
// rotationCompressionUnweighted / ull-overload mapping_after_swap_conti
// path.  Usage: refapi_unweighted P N C seed out.bin
// Writes the final state (raw complex128, the reference's physical order)
// and out.bin.edges (one "i j" line per edge, logical labels).
#include <stdio.h>
#include <stdlib.h>

#include <random>
#include <vector>

#include "refapi/graph.h"
#include "refapi/rx.h"
#include "refapi/rzz.h"
#include "refapi/state.h"
#include "refapi/swap.h"

int main(int argc, char** argv) {
    if (argc != 6) return 2;
    const int P = atoi(argv[1]), N = atoi(argv[2]), C = atoi(argv[3]);
    std::mt19937_64 rng(strtoull(argv[4], nullptr, 10));
    try {
        State q = createState(N, 0, N, C);
        ull* graph = init1DGraph(q);
        FILE* fe = fopen((std::string(argv[5]) + ".edges").c_str(), "w");
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (rng() % 2) {
                    addEdgeTo1DGraph(q, graph, i, j);
                    fprintf(fe, "%d %d\n", i, j);
                }
        fclose(fe);
        initH(q);
        std::vector<std::vector<int>> subcirs;
        for (int i = 0; i < N; i += C) {
            std::vector<int> s;
            for (int j = i; j < i + C && j < N; ++j) s.push_back(j);
            subcirs.push_back(s);
        }
        const double gamma = 0.7, beta = 0.45;
        for (int p = 0; p < P; p++) {
            rotationCompressionUnweighted(q, gamma, graph, p == 0);
            int swap_in = 0;
            for (size_t i = 0; i < subcirs.size(); i++) {
                multiRotateX(q, subcirs[0], (int)subcirs[i].size(), beta);
                if (i + 1 < subcirs.size()) {
                    swap_in += (int)subcirs[i].size();
                    swap_gate_conti(q, 0, swap_in, (int)subcirs[i + 1].size());
                    mapping_after_swap_conti(q, graph, 0, swap_in, (int)subcirs[i + 1].size());
                }
            }
        }
        stateCpyDeviceToHost(q);
        FILE* f = fopen(argv[5], "wb");
        fwrite(q.hState, sizeof(Complex), 1ull << N, f);
        fclose(f);
        free1DGraph(graph);
        destroyState(q);
    } catch (const fq::Error& e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
