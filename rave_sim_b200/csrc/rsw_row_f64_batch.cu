// Row-pass kernels of batched passes (double fields): per-instance transfer
// functions (PassArgs::bpr).
#include "rsw_row_dispatch.h"

namespace rsw {
cudaError_t launch_row_pass_f64_batch(const PassArgs &a, int e, cudaStream_t s) {
    return row_dispatch_f64<true>(a, e, s);
}
}  // namespace rsw
