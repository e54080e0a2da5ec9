// rz_extras.cpp -- configuration hooks used by rz_remove before the tuning table and the learned
// predictor are loaded into a context.
#include "rz_internal.h"

namespace rz {

bool predict_cfg(rz_ctx*, uint32_t, uint32_t, uint32_t, const uint32_t*, cudaStream_t, rz_launch_cfg*) {
    return false;
}
bool tuned_cfg(rz_ctx*, uint32_t, uint32_t, uint32_t, rz_launch_cfg*) { return false; }
void release_extras(rz_ctx*) {}

}  // namespace rz
