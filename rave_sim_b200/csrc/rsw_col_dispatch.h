// Column-pass dispatch by column length, samples per thread and columns per
// CTA, shared by the plain column pass (rsw_col.cu) and its detection
// variant (rsw_col_det.cu).
#pragma once

#include "rsw_passes.cuh"

namespace rsw {
#define RSW_COL_CASE16(R, L) \
    case L: return col_impl<R, L, col_c(L), 16, DET, BT>(a, s);
// 8 or 16 samples per thread (C8 / C16 columns per CTA), 32 on request
#define RSW_COL_CASE_E(R, L, C8, C16)                                                       \
    case L: return e == 8 ? col_impl<R, L, C8, 8, DET, BT>(a, s)                           \
                          : e == 32 ? col_impl<R, L, 4, 32, DET, BT>(a, s) : col_impl<R, L, C16, 16, DET, BT>(a, s);
#define RSW_COL_CASE(R, L) \
    case L: return e == 32 ? col_impl<R, L, 4, 32, DET, BT>(a, s) : col_impl<R, L, col_c(L), 16, DET, BT>(a, s);

// Columns per CTA: col_c(L) (16-byte samples: 64- to 512-byte row
// segments); complex64 doubles them where the threads allow (col_c64).
// BT: the batched kernels (per-instance transmission factors, PassArgs::btr).
template <bool DET, bool BT = false> cudaError_t col_dispatch(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    if (dbl) {
        switch (a.log_n1) {
            RSW_COL_CASE16(double, 4) RSW_COL_CASE16(double, 5) RSW_COL_CASE16(double, 6)
            RSW_COL_CASE16(double, 7)
            case 8: return e == 8 ? col_impl<double, 8, 16, 8, DET, BT>(a, s) : col_impl<double, 8, 16, 16, DET, BT>(a, s);
            RSW_COL_CASE_E(double, 9, 8, 8) RSW_COL_CASE_E(double, 10, 4, 4) RSW_COL_CASE_E(double, 11, 4, 4)
            // 2^12 (tunings only): two columns per CTA, 32-byte row segments
            case 12: return e == 8 ? col_impl<double, 12, 2, 8, DET, BT>(a, s) : col_impl<double, 12, 2, 16, DET, BT>(a, s);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (a.log_n1) {
        RSW_COL_CASE16(float, 4) RSW_COL_CASE16(float, 5) RSW_COL_CASE16(float, 6)
        RSW_COL_CASE16(float, 7)
        case 8: return e == 8 ? col_impl<float, 8, 32, 8, DET, BT>(a, s) : col_impl<float, 8, 16, 16, DET, BT>(a, s);
        RSW_COL_CASE_E(float, 9, 16, 8) RSW_COL_CASE_E(float, 10, 4, col_c64(10))
        RSW_COL_CASE_E(float, 11, 4, col_c64(11)) RSW_COL_CASE(float, 12)
    default: return cudaErrorInvalidValue;
    }
}
#undef RSW_COL_CASE16
#undef RSW_COL_CASE_E
#undef RSW_COL_CASE
}  // namespace rsw
