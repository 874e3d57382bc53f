/*
 * swap.h -- FOR-QAOA's qubit-block swap API (include/swap.h:20-28 of the
 * reference), single device.  swap_gate_conti exchanges bit blocks
 * [SwapOut, SwapOut+numSwap) and [SwapIn, SwapIn+numSwap) of the state
 * index; mapping_after_swap_conti relabels a graph the same way.
 */
#ifndef FQ_REFAPI_SWAP_H_
#define FQ_REFAPI_SWAP_H_

#include <cassert>
#include <iostream>
#include <vector>

#include "state.h"
using namespace std;

void mapping_after_swap_conti(const State& qureg, Fp* graph, const int SwapOut, const int SwapIn,
                              const int numSwap);
/* Declared without a definition in the reference (include/swap.h:25). */
void mapping_after_swap_conti(const State& qureg, ull* graph, const int SwapOut, const int SwapIn,
                              const int numSwap);
/* Declared without a definition in the reference (include/swap.h:27). */
void swap_gate(const State& qureg, const int targ0, const int targ1);
void swap_gate_conti(const State& qureg, const int SwapOut, const int SwapIn, const int numSwap);

#endif
