// Row-pass dispatch by row length and samples per thread, shared by the
// instantiation units of the plain row passes (rsw_row_f32.cu, rsw_row_f64.cu)
// and of their batched variants (rsw_row_f32_batch.cu, rsw_row_f64_batch.cu).
#pragma once

#include "rsw_passes.cuh"

namespace rsw {
// two-level rows (chirp form): 2^7 .. 2^13 (c128) / 2^14 (c64), 16 or 32 elements per thread;
// single-level rows (per-sample form): 2^4 .. 2^13 / 2^14, 16 elements per thread
#define RSW_ROW_CASE(R, L) \
    case L: return chirp ? (e == 32 ? row_impl<R, L, 32, true, BT>(a, s) : row_impl<R, L, 16, true, BT>(a, s)) \
                         : row_impl<R, L, 16, false, BT>(a, s);
#define RSW_ROW_CASE16(R, L) \
    case L: return chirp ? row_impl<R, L, 16, true, BT>(a, s) : row_impl<R, L, 16, false, BT>(a, s);
// rows with 8 samples per thread (radix-8 stages, twice the threads)
#define RSW_ROW_CASE8(R, L) \
    case L: return chirp ? (e == 8 ? row_impl<R, L, 8, true, BT>(a, s) \
                                   : e == 32 ? row_impl<R, L, 32, true, BT>(a, s) : row_impl<R, L, 16, true, BT>(a, s)) \
                         : row_impl<R, L, 16, false, BT>(a, s);
#define RSW_ROW_CASE_S(R, L) \
    case L: return chirp ? cudaErrorInvalidValue : row_impl<R, L, 16, false, BT>(a, s);

// multi-level rows take the chirp form of the Fresnel kernel; the exact
// kernel and single-level rows evaluate the transfer function per sample.
// BT: the batched kernels (chirp form only; the others return an error)
template <bool BT> cudaError_t row_dispatch_f64(const PassArgs &a, int e, cudaStream_t s) {
    const bool chirp = a.log_n1 > 0 && !a.pr.exact;
    switch (a.log_n2) {
        RSW_ROW_CASE_S(double, 4) RSW_ROW_CASE_S(double, 5) RSW_ROW_CASE_S(double, 6)
        RSW_ROW_CASE16(double, 7) RSW_ROW_CASE16(double, 8) RSW_ROW_CASE(double, 9)
        RSW_ROW_CASE(double, 10) RSW_ROW_CASE8(double, 11) RSW_ROW_CASE8(double, 12) RSW_ROW_CASE8(double, 13)
    default: return cudaErrorInvalidValue;
    }
}
template <bool BT> cudaError_t row_dispatch_f32(const PassArgs &a, int e, cudaStream_t s) {
    const bool chirp = a.log_n1 > 0 && !a.pr.exact;
    switch (a.log_n2) {
        RSW_ROW_CASE_S(float, 4) RSW_ROW_CASE_S(float, 5) RSW_ROW_CASE_S(float, 6) RSW_ROW_CASE16(float, 7)
        RSW_ROW_CASE16(float, 8) RSW_ROW_CASE(float, 9) RSW_ROW_CASE(float, 10) RSW_ROW_CASE8(float, 11)
        RSW_ROW_CASE8(float, 12) RSW_ROW_CASE8(float, 13) RSW_ROW_CASE(float, 14)
    default: return cudaErrorInvalidValue;
    }
}
#undef RSW_ROW_CASE
#undef RSW_ROW_CASE16
#undef RSW_ROW_CASE8
#undef RSW_ROW_CASE_S
}  // namespace rsw
