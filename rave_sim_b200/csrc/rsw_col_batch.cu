// Column-pass kernels of batched passes (both precisions): per-instance
// transmission factors (PassArgs::btr).
#include "rsw_col_dispatch.h"

namespace rsw {
cudaError_t launch_col_pass_batch(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    return col_dispatch<false, true>(a, dbl, e, s);
}
}  // namespace rsw
