// ogx_mixed.cu -- mixed-precision form (FP32 P2P, split-precision tensor-core M2L).
#include "ogx_internal.cuh"

namespace ogx {
int fmm_mixed(Handle& h, double* d_acc, double* d_pot) {
    (void)h; (void)d_acc; (void)d_pot;
    set_last_error(OGX_ERR_UNSUPPORTED, "mixed-precision form not built yet");
    return OGX_ERR_UNSUPPORTED;
}
}  // namespace ogx
