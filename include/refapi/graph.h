/*
 * graph.h -- FOR-QAOA's graph API (include/graph.h:22-28 of the reference).
 * 2D: N x N FP64 upper triangle (weights).  1D: one 64-bit neighbour mask
 * per vertex (unweighted), bit j of graph[i] for edge (i, j), i < j.
 * Graphs live in host memory (the reference uses managed memory; the
 * library only ever reads them on the host and uploads what it needs).
 */
#ifndef FQ_REFAPI_GRAPH_H_
#define FQ_REFAPI_GRAPH_H_

#include "state.h"

ull* init1DGraph(const State& qureg);
void free1DGraph(ull* graph);
void addEdgeTo1DGraph(const State& qureg, ull* graph, int qubit1, int qubit2);

Fp* init2DGraph(const State& qureg);
void addEdgeTo2DGraph(const State& qureg, Fp* graph, int qubit1, int qubit2, Fp weight);
void free2DGraph(Fp* graph);

#endif
