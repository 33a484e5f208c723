// Column-pass kernels and row chirp tables (both precisions).
#include "rsw_col_dispatch.h"

namespace rsw {
cudaError_t launch_col_pass_batch(const PassArgs &a, bool dbl, int e, cudaStream_t s);
// per-instance transmission factors take the batched kernels (rsw_col_batch.cu)
cudaError_t launch_col_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    if (a.btr) return launch_col_pass_batch(a, dbl, e, s);
    return col_dispatch<false>(a, dbl, e, s);
}


#define RSW_CH_CASE(R, L) \
    case L: return e == 32 ? chirp_impl<R, L, 32>(out, hi, lo, s) : chirp_impl<R, L, 16>(out, hi, lo, s);
#define RSW_CH_CASE8(R, L) \
    case L: return e == 8 ? chirp_impl<R, L, 8>(out, hi, lo, s) \
                          : e == 32 ? chirp_impl<R, L, 32>(out, hi, lo, s) : chirp_impl<R, L, 16>(out, hi, lo, s);
#define RSW_CH_CASE16(R, L) \
    case L: return chirp_impl<R, L, 16>(out, hi, lo, s);

cudaError_t launch_chirp_table(void *out, int log_n2, double hi, double lo, bool dbl, int e, cudaStream_t s) {
    if (dbl) {
        switch (log_n2) {
            RSW_CH_CASE16(double, 4) RSW_CH_CASE16(double, 5) RSW_CH_CASE16(double, 6) RSW_CH_CASE16(double, 7)
            RSW_CH_CASE16(double, 8) RSW_CH_CASE(double, 9) RSW_CH_CASE(double, 10) RSW_CH_CASE8(double, 11)
            RSW_CH_CASE8(double, 12) RSW_CH_CASE8(double, 13)
        default: return cudaErrorInvalidValue;
        }
    }
    switch (log_n2) {
        RSW_CH_CASE16(float, 4) RSW_CH_CASE16(float, 5) RSW_CH_CASE16(float, 6) RSW_CH_CASE16(float, 7)
        RSW_CH_CASE16(float, 8) RSW_CH_CASE(float, 9) RSW_CH_CASE(float, 10) RSW_CH_CASE8(float, 11)
        RSW_CH_CASE8(float, 12) RSW_CH_CASE8(float, 13) RSW_CH_CASE(float, 14)
    default: return cudaErrorInvalidValue;
    }
}


}  // namespace rsw
