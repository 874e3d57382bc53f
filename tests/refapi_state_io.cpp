// A program written only against the reference-style C++ API
// (include/refapi/*.h) that exercises the state set-up and copy functions of
// src/state.cpp:89-219,320-336 beyond createState/stateCpyDeviceToHost:
//   stateCpyHostToDevice  -- a host state uploaded and then used by a kernel
//                            (multiRotateX on the first C qubits);
//   stateInitDeviceState  -- the device state reset to |0...0>;
//   prepare               -- the chunk size recorded, C < 1 refused.
// Usage: refapi_state_io N C angle out_prefix.  Writes out_prefix.in (the
// uploaded state) and out_prefix.out (after RX), raw complex128; prints one
// line per check and exits non-zero at the first failure.
#include <stdio.h>
#include <stdlib.h>

#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "refapi/rx.h"
#include "refapi/state.h"

static bool is_basis0(const State& q) {
    for (ull z = 0; z < q.numAmpsPerDevice; z++) {
        const double re = q.hState[z].real, im = q.hState[z].imag;
        if (im != 0.0 || re != (z == 0 ? 1.0 : 0.0)) return false;
    }
    return true;
}

static bool write_state(const State& q, const std::string& path) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t n = fwrite(q.hState, sizeof(Complex), q.numAmpsPerDevice, f);
    fclose(f);
    return n == q.numAmpsPerDevice;
}

int main(int argc, char** argv) {
    if (argc != 5) return 2;
    const int N = atoi(argv[1]), C = atoi(argv[2]);
    const double angle = atof(argv[3]);
    const std::string out = argv[4];
    try {
        State q = createState(N, 0, N, C);
        // createState leaves |0...0> on the device and in the host mirror.
        stateCpyDeviceToHost(q);
        if (!is_basis0(q)) return fprintf(stderr, "createState: not |0>\n"), 1;
        printf("createState |0> ok\n");

        // A seeded normalised state, uploaded from the host mirror.
        std::mt19937_64 rng(1234);
        std::normal_distribution<double> nd;
        double nrm = 0;
        for (ull z = 0; z < q.numAmpsPerDevice; z++) {
            q.hState[z].real = nd(rng);
            q.hState[z].imag = nd(rng);
            nrm += q.hState[z].real * q.hState[z].real + q.hState[z].imag * q.hState[z].imag;
        }
        nrm = 1.0 / std::sqrt(nrm);
        for (ull z = 0; z < q.numAmpsPerDevice; z++) {
            q.hState[z].real *= nrm;
            q.hState[z].imag *= nrm;
        }
        if (!write_state(q, out + ".in")) return fprintf(stderr, "write .in\n"), 1;
        stateCpyHostToDevice(q);
        // The mirror is cleared so that the next copy back is observed.
        for (ull z = 0; z < q.numAmpsPerDevice; z++) q.hState[z] = Complex{0.0, 0.0};
        std::vector<int> targets;
        for (int t = 0; t < C; t++) targets.push_back(t);
        multiRotateX(q, targets, C, angle);
        stateCpyDeviceToHost(q);
        if (!write_state(q, out + ".out")) return fprintf(stderr, "write .out\n"), 1;
        printf("stateCpyHostToDevice + multiRotateX ok\n");

        stateInitDeviceState(q);
        stateCpyDeviceToHost(q);
        if (!is_basis0(q)) return fprintf(stderr, "stateInitDeviceState: not |0>\n"), 1;
        printf("stateInitDeviceState ok\n");

        prepare(q, C > 1 ? C - 1 : 1);
        if (q.chunkQubits != (C > 1 ? C - 1 : 1)) return fprintf(stderr, "prepare: chunk\n"), 1;
        bool refused = false;
        try {
            prepare(q, 0);
        } catch (const fq::Error&) {
            refused = true;
        }
        if (!refused) return fprintf(stderr, "prepare(0) accepted\n"), 1;
        printf("prepare ok\n");
        destroyState(q);
    } catch (const fq::Error& e) {
        fprintf(stderr, "fq::Error %s\n", e.what());
        return 1;
    }
    return 0;
}
