// fq_disp_rx_tan.cu -- strided RX passes of the fused engine with the
// reduced gate [[1,-it],[-it,1]], t = tan(beta/2), optionally accumulating <C>.
#include "fq_launch.cuh"

namespace fq {

int dispatch_rx_tan(fq_ctx* ctx, bool integer, bool energy, const PassArgs& A) {
    if (!energy) return launch_pass<int, PH_NONE, GM_TAN, EX_NONE, true>(ctx, A);
    if (integer) return launch_pass<int, PH_NONE, GM_TAN, EX_ENERGY, true>(ctx, A);
    return launch_pass<double, PH_NONE, GM_TAN, EX_ENERGY, true>(ctx, A);
}

}  // namespace fq
