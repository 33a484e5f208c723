// Row-pass kernels (float fields). Instantiations of rsw_passes.cuh.
#include "rsw_row_dispatch.h"

namespace rsw {
cudaError_t launch_row_pass_f32(const PassArgs &a, int e, cudaStream_t s) { return row_dispatch_f32<false>(a, e, s); }
}  // namespace rsw
