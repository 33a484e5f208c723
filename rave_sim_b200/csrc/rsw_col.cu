// Column-pass kernels and row chirp tables (both precisions).
#include "rsw_passes.cuh"

namespace rsw {
#define RSW_COL_CASE16(R, L) \
    case L: return col_impl<R, L, col_c(L), 16>(a, s);
// 8 or 16 samples per thread (C8 / C16 columns per CTA), 32 on request
#define RSW_COL_CASE_E(R, L, C8, C16) \
    case L: return e == 8 ? col_impl<R, L, C8, 8>(a, s) \
                          : e == 32 ? col_impl<R, L, 4, 32>(a, s) : col_impl<R, L, C16, 16>(a, s);
#define RSW_COL_CASE(R, L) \
    case L: return e == 32 ? col_impl<R, L, 4, 32>(a, s) : col_impl<R, L, col_c(L), 16>(a, s);

// Columns per CTA: col_c(L) (16-byte samples: 64- to 512-byte row
// segments); complex64 doubles them where the threads allow (col_c64).
cudaError_t launch_col_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    if (dbl) {
        switch (a.log_n1) {
            RSW_COL_CASE16(double, 4) RSW_COL_CASE16(double, 5) RSW_COL_CASE16(double, 6)
            RSW_COL_CASE16(double, 7)
            case 8: return e == 8 ? col_impl<double, 8, 16, 8>(a, s) : col_impl<double, 8, 16, 16>(a, s);
            RSW_COL_CASE_E(double, 9, 8, 8) RSW_COL_CASE_E(double, 10, 4, 4) RSW_COL_CASE_E(double, 11, 4, 4)
        default: return cudaErrorInvalidValue;
        }
    }
    switch (a.log_n1) {
        RSW_COL_CASE16(float, 4) RSW_COL_CASE16(float, 5) RSW_COL_CASE16(float, 6)
        RSW_COL_CASE16(float, 7)
        case 8: return e == 8 ? col_impl<float, 8, 32, 8>(a, s) : col_impl<float, 8, 16, 16>(a, s);
        RSW_COL_CASE_E(float, 9, 16, 8) RSW_COL_CASE_E(float, 10, 4, col_c64(10))
        RSW_COL_CASE_E(float, 11, 4, col_c64(11)) RSW_COL_CASE(float, 12)
    default: return cudaErrorInvalidValue;
    }
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
