// rz_mlp.cu -- learned launch-configuration predictor (filled in below this header).
#include "rz_internal.h"

namespace rz {

bool predict_cfg(rz_ctx*, uint32_t, uint32_t, uint32_t, const uint32_t*, cudaStream_t, rz_launch_cfg*) {
    return false;
}
void release_predictor(rz_ctx*) {}

}  // namespace rz
