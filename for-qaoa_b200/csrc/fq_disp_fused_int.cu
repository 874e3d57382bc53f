// fq_disp_fused_int.cu -- fused two-layer passes, integer weights.
#include "fq_disp_fused.cuh"

namespace fq {

int dispatch_fused_int(fq_ctx* ctx, int gm1, int gm2, const PassArgs& A) {
    return fused_dispatch<int>(ctx, gm1, gm2, A);
}

}  // namespace fq
