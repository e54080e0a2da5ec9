// rz_extras.cpp -- context teardown of the optional parts (tuning table, learned predictor, asynchronous host-index pipeline).
#include "rz_internal.h"

namespace rz {

void release_tune(rz_ctx* ctx);       // rz_autotune.cpp
void release_predictor(rz_ctx* ctx);  // rz_mlp.cu
void release_async(rz_ctx* ctx);      // rz_async.cpp

void release_extras(rz_ctx* ctx) {
    release_tune(ctx);
    release_predictor(ctx);
    release_async(ctx);
}

}  // namespace rz
