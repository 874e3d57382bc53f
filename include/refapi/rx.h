/*
 * rx.h -- FOR-QAOA's mixer API (include/rx.h:20-26 of the reference).
 * multiRotateX applies RX(angle) = exp(-i*angle*X/2) to targetQubits[0..
 * gate_size); the targets must lie in the state's chunk (< min(13, N)).
 */
#ifndef FQ_REFAPI_RX_H_
#define FQ_REFAPI_RX_H_

#include <cassert>
#include <iostream>
#include <vector>

#include "state.h"
using namespace std;

/* Declared without a definition in the reference (include/rx.h:25); here any
 * target < N. */
void rotateX(const State& qureg, const int targetQubit, const Fp angle);
void multiRotateX(State& qureg, vector<int>& targetQubits, const int gate_size, const Fp angle);

#endif
