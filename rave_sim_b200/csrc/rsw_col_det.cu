// Column-pass kernels with fused detector binning: the last inverse column
// pass of a phase step (both precisions).
#include "rsw_col_dispatch.h"

namespace rsw {
cudaError_t launch_col_detect(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    return col_dispatch<true>(a, dbl, e, s);
}
}  // namespace rsw
