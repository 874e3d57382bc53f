/*
 * rzz.h -- FOR-QAOA's cost-layer API (include/rzz.h:22-26 of the reference).
 * initH sets the launch-control amplitude pow(1/sqrt(2), N) used by the
 * first cost layer (src/rzz.cu:24-28).
 */
#ifndef FQ_REFAPI_RZZ_H_
#define FQ_REFAPI_RZZ_H_

#include "state.h"

extern Fp initialAmp;

void initH(const State& qureg);
/* Unit-weight cost layer on the 1D bitmask graph; the reference declares it
 * (include/rzz.h:25) with its kernel commented out (src/rzz.cu:30-82). */
void rotationCompressionUnweighted(const State& qureg, Fp angle, ull* graph, bool isFirstLayer);
void rotationCompressionWeighted(State& qureg, const Fp angle, const Fp* graph,
                                 const bool isFirstLayer);

#endif
