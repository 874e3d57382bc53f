/*
 * state.h -- FOR-QAOA's State API (include/state.h of the reference),
 * single-device (D = 0), implemented by libforqaoa on a B200.
 *
 * Same type names, field names and function signatures as the reference
 * (include/state.h:23-77) so code written against it compiles unchanged with
 * -I include/refapi.  Differences, all deliberate:
 *  - D must be 0: the multi-device fields (dBuf, comm, texObj) stay empty
 *    and createState throws fq::Error(FQ_ERR_UNSUPPORTED) for D > 0;
 *  - errors throw fq::Error (status + message) instead of exit();
 *  - comm is a void* (no NCCL in the single-device library);
 *  - GPUState carries the library context (ctx) and State the chunk size.
 */
#ifndef FQ_REFAPI_STATE_H_
#define FQ_REFAPI_STATE_H_

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "../forqaoa.h"

#define RANK_PER_NODE 8

typedef double Fp;
typedef unsigned long long ull;
typedef long long ll;

typedef struct Complex {
    Fp real;
    Fp imag;
} Complex;

typedef struct {
    Complex* dState;
    Complex* dBuf;
    Complex* dTexMem;
    cudaTextureObject_t texObj;
    cudaStream_t compute_stream;
    void* comm;
    void* stateHandle;
    void* bufHandle;
    int id;
    Fp* d_graph_1D;
    int* d_subcirs;
    int* d_table;
    fq_ctx* ctx;
} GPUState;

typedef struct State {
    Complex* hState;
    int numDevice;
    int numQubits;
    int numQubitsPerDevice;
    int numBufsPerDevice;
    int numQubitsPerBuffer;
    ull numAmpsPerDevice;
    ull stateSizePerDevice;
    ull numAmpsPerBuf;
    ull bufSize;
    GPUState* gpus;
    int chunkQubits;
} State;

namespace fq {
/* Error thrown by the C++ API; status() is one of the FQ_* codes. */
class Error : public std::runtime_error {
  public:
    Error(int status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
    int status() const { return status_; }

  private:
    int status_;
};
}  // namespace fq

State createState(int N, int D, int B, int C);
void destroyState(const State& state);

void stateCpyDeviceToHost(const State& state);
void stateCpyHostToDevice(const State& state);

void stateInitDeviceState(const State& qureg);
void ncclWarnup(State& qureg);

void prepare(State& qureg, int C);

#endif
