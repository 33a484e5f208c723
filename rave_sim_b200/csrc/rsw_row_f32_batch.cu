// Row-pass kernels of batched passes (float fields): per-instance transfer
// functions (PassArgs::bpr).
#include "rsw_row_dispatch.h"

namespace rsw {
cudaError_t launch_row_pass_f32_batch(const PassArgs &a, int e, cudaStream_t s) {
    return row_dispatch_f32<true>(a, e, s);
}
}  // namespace rsw
