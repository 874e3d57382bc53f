// fq_disp_fused_fp.cu -- fused two-layer passes, FP64 weights.
#include "fq_disp_fused.cuh"

namespace fq {

int dispatch_fused_fp(fq_ctx* ctx, int gm1, int gm2, const PassArgs& A) {
    return fused_dispatch<double>(ctx, gm1, gm2, A);
}

}  // namespace fq
