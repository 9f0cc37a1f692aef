// Batched screen runtime (filled in below the single-instance kernels).
#include "cee_internal.h"

namespace cee {

struct BatchState {};

void ReleaseBatch(cee_ctx* ctx) {
  delete ctx->batch;
  ctx->batch = nullptr;
}

uint64_t BatchResident(const cee_ctx*) { return 0; }

}  // namespace cee
