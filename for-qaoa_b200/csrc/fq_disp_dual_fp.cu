// fq_disp_dual_fp.cu -- adjoint phase passes (plain and fused), FP64 weights.
#include "fq_disp_dual.cuh"

namespace fq {

int dispatch_dual_phase_fp(fq_ctx* ctx, int gm, int gm2, const PassArgs& A, double* gb,
                           double* gg, double* gb2, bool store) {
    return dual_phase_dispatch<double>(ctx, gm, gm2, A, gb, gg, gb2, store);
}

int dispatch_dual_turn_fp(fq_ctx* ctx, int gm, int gmf, const PassArgs& A, double* gb,
                           double* ge) {
    return dual_turn_dispatch<double>(ctx, gm, gmf, A, gb, ge);
}

}  // namespace fq
