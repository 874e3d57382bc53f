// weighted.cpp -- the `weighted <P> <N> <D> <C> <B>` driver of FOR-QAOA
// (src/Weighted.cpp:37-173), single device, on libforqaoa.
//
// With no options it runs the reference's own circuit: unit-weight complete
// graph, gamma = beta = pi/4 (src/Weighted.cpp:34-35,81-88), P layers, and
// prints the reference's "Total simulation time" / "Total RX time" lines.
// Options (after the five positional arguments):
//   --engine fused|reference  fused sweeps (default) or the reference's
//                             cost / RX-chunk / block-swap schedule
//   --weights unit|int|fp     unit (default), integers 1..10, U[0,1)
//   --graph complete|gnp|reg3 complete (default), G(N,1/2), 3-regular
//   --angles pi4|random       pi/4 (default), gamma~U[0,pi), beta~U[0,pi/2)
//   --seed S                  seed of the generators (default 1)
//   --expect                  print <C>
//   --dump FILE               write the final state (raw complex128) in the
//                             reference's physical qubit order, and beside it
//                             FILE.labels: the logical qubit at each physical
//                             bit position, and FILE.circuit: N P, gammas,
//                             betas, the N x N graph (validate_dump.py reads
//                             all three)
// Timing uses CUDA events around the layer loop, after a device sync, so it
// covers the GPU work (the reference's non-MPI timer stops before its sync,
// src/Weighted.cpp:140-150).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "forqaoa.h"
#include "refapi/graph.h"
#include "refapi/rx.h"
#include "refapi/rzz.h"
#include "refapi/state.h"
#include "refapi/swap.h"
#include "refapi/utils.h"

static void usage() {
    fprintf(stderr,
            "usage: weighted <P> <N> <D> <C> <B> [--engine fused|reference] [--weights "
            "unit|int|fp]\n"
            "                [--graph complete|gnp|reg3] [--angles pi4|random] [--seed S]\n"
            "                [--expect] [--dump FILE]\n");
}

static std::vector<double> make_graph(int N, const std::string& kind, const std::string& wk,
                                      std::mt19937_64& rng) {
    std::vector<double> g((size_t)N * N, 0.0);
    std::uniform_int_distribution<int> wi(1, 10);
    std::uniform_real_distribution<double> wf(0.0, 1.0);
    auto weight = [&]() { return wk == "int" ? (double)wi(rng) : wk == "fp" ? wf(rng) : 1.0; };
    if (kind == "reg3") {
        // Random 3-regular graph: seeded pairing with rejection.
        for (int tries = 0;; tries++) {
            std::vector<int> stubs;
            for (int v = 0; v < N; v++)
                for (int c = 0; c < 3; c++) stubs.push_back(v);
            std::shuffle(stubs.begin(), stubs.end(), rng);
            std::fill(g.begin(), g.end(), 0.0);
            bool ok = (N * 3) % 2 == 0;
            for (size_t e = 0; ok && e + 1 < stubs.size(); e += 2) {
                int a = std::min(stubs[e], stubs[e + 1]), b = std::max(stubs[e], stubs[e + 1]);
                if (a == b || g[a * N + b] != 0) ok = false;
                else g[a * N + b] = weight();
            }
            if (ok) break;
            if (tries > 100000) throw fq::Error(FQ_ERR_INVALID, "no 3-regular graph found");
        }
        return g;
    }
    std::bernoulli_distribution half(0.5);
    for (int i = 0; i < N; i++)
        for (int j = i + 1; j < N; j++)
            if (kind == "complete" || half(rng)) g[i * N + j] = weight();
    return g;
}

int main(int argc, char* argv[]) {
    int P = 1, N = 21, D = 0, C = 10, B = 19;  // src/Weighted.cpp:65-71
    int argi = 1;
    if (argc >= 2 && argv[1][0] != '-') {
        if (argc < 6) {
            usage();
            return 2;
        }
        P = atoi(argv[1]);
        N = atoi(argv[2]);
        D = atoi(argv[3]);
        C = atoi(argv[4]);
        B = atoi(argv[5]);
        argi = 6;
    }
    std::string engine = "fused", weights = "unit", graph_kind = "complete", angles = "pi4",
                dump;
    unsigned long long seed = 1;
    bool expect = false;
    for (; argi < argc; argi++) {
        std::string a = argv[argi];
        auto next = [&]() -> std::string {
            if (argi + 1 >= argc) {
                usage();
                exit(2);
            }
            return argv[++argi];
        };
        if (a == "--engine") engine = next();
        else if (a == "--weights") weights = next();
        else if (a == "--graph") graph_kind = next();
        else if (a == "--angles") angles = next();
        else if (a == "--seed") seed = strtoull(next().c_str(), nullptr, 10);
        else if (a == "--expect") expect = true;
        else if (a == "--dump") dump = next();
        else {
            usage();
            return 2;
        }
    }
    if (P < 1 || N < 2 || C < 1 || (engine != "fused" && engine != "reference")) {
        usage();
        return 2;
    }
    try {
        State qureg = createState(N, D, B, C);
        std::mt19937_64 rng(seed);
        std::vector<double> g0 = make_graph(N, graph_kind, weights, rng);
        Fp* graph = init2DGraph(qureg);
        for (int i = 0; i < N; i++)
            for (int j = i + 1; j < N; j++)
                if (g0[i * N + j] != 0) addEdgeTo2DGraph(qureg, graph, i, j, g0[i * N + j]);
        std::vector<double> gam(P, M_PI_4), bet(P, M_PI_4);  // src/Weighted.cpp:34-35
        if (angles == "random") {
            std::uniform_real_distribution<double> ug(0.0, M_PI), ub(0.0, M_PI / 2);
            for (int p = 0; p < P; p++) {
                gam[p] = ug(rng);
                bet[p] = ub(rng);
            }
        }
        initH(qureg);
        fq_ctx* ctx = qureg.gpus[0].ctx;
        cudaStream_t st = qureg.gpus[0].compute_stream;
        // src/Weighted.cpp:97-108
        std::vector<std::vector<int>> subcirs;
        for (int i = 0; i < N; i += C) {
            std::vector<int> q;
            for (int j = i; j < i + C && j < N; ++j) q.push_back(j);
            subcirs.push_back(q);
        }
        const int num_subcir = (int)subcirs.size();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaDeviceSynchronize();
        MEASURET_START;
        cudaEventRecord(e0, st);
        double energy = 0;
        if (engine == "reference") {
            // src/Weighted.cpp:115-138
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
        } else {
            int s = fq_qaoa_forward(ctx, qureg.gpus[0].dState, N, P, graph, gam.data(), bet.data(),
                                    nullptr);
            if (s != FQ_OK) throw fq::Error(s, fq_last_error());
        }
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        MEASURET_END;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        rx_gate_time_ms = ms;
        printf("Total simulation time : %10.6f\n", diff / 1000000.0);
        printf("Total RX time : %f ms\n", rx_gate_time_ms);
        printf("Device time : %f ms (%s engine, %.3f layers/s)\n", ms, engine.c_str(),
               P / (ms / 1000.0));
        // The fused engine leaves logical order; the reference schedule leaves
        // its physical order with the graph relabelled to match.
        std::vector<int> lab(N);
        if (engine == "reference")
            fq_reference_label_map(N, C, P, lab.data());
        else
            for (int b = 0; b < N; b++) lab[b] = b;
        if (expect) {
            int s = fq_expectation(ctx, qureg.gpus[0].dState, N, graph, &energy);
            if (s != FQ_OK) throw fq::Error(s, fq_last_error());
            printf("<C> : %.17g\n", energy);
        }
        if (!dump.empty()) {
            void* src = qureg.gpus[0].dState;
            void* tmp = nullptr;
            if (engine == "fused") {
                // logical -> the reference's physical order: perm = inverse label map
                std::vector<int> refl(N), inv(N);
                fq_reference_label_map(N, C, P, refl.data());
                for (int b = 0; b < N; b++) inv[refl[b]] = b;
                int s = fq_state_alloc(ctx, N, &tmp);
                if (s == FQ_OK) s = fq_permute_qubits(ctx, src, tmp, N, inv.data());
                if (s != FQ_OK) throw fq::Error(s, fq_last_error());
                src = tmp;
            }
            int s = fq_state_to_host(ctx, src, N, qureg.hState);
            if (s != FQ_OK) throw fq::Error(s, fq_last_error());
            if (tmp) fq_state_free(ctx, tmp);
            FILE* f = fopen(dump.c_str(), "wb");
            if (!f) throw fq::Error(FQ_ERR_INVALID, "cannot open " + dump);
            fwrite(qureg.hState, sizeof(Complex), 1ull << N, f);
            fclose(f);
            // Sidecar: the reference's physical -> logical label map after P
            // layers with chunk C (src/Weighted.cpp:97-138 never undoes it).
            std::vector<int> refl(N);
            fq_reference_label_map(N, C, P, refl.data());
            FILE* fl = fopen((dump + ".labels").c_str(), "w");
            if (!fl) throw fq::Error(FQ_ERR_INVALID, "cannot open " + dump + ".labels");
            for (int b = 0; b < N; b++) fprintf(fl, "%d%c", refl[b], b + 1 < N ? ' ' : '\n');
            fclose(fl);
            // Sidecar: the circuit (N P, gammas, betas, the N x N logical graph).
            FILE* fc = fopen((dump + ".circuit").c_str(), "w");
            if (!fc) throw fq::Error(FQ_ERR_INVALID, "cannot open " + dump + ".circuit");
            fprintf(fc, "%d %d\n", N, P);
            for (int p = 0; p < P; p++) fprintf(fc, "%.17g%c", gam[p], p + 1 < P ? ' ' : '\n');
            for (int p = 0; p < P; p++) fprintf(fc, "%.17g%c", bet[p], p + 1 < P ? ' ' : '\n');
            for (int i = 0; i < N; i++)
                for (int j = 0; j < N; j++)
                    fprintf(fc, "%.17g%c", j > i ? g0[i * N + j] : 0.0, j + 1 < N ? ' ' : '\n');
            fclose(fc);
        }
        fflush(stdout);
        free2DGraph(graph);
        destroyState(qureg);
    } catch (const fq::Error& e) {
        fprintf(stderr, "weighted: %s\n", e.what());
        return 1;
    }
    return 0;
}
