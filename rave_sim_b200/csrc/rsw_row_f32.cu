// Row-pass kernels (float fields). Instantiations of rsw_passes.cuh.
#include "rsw_passes.cuh"

namespace rsw {
// two-level rows (chirp form): 2^7 .. 2^13 (c128) / 2^14 (c64), 16 or 32 elements per thread;
// single-level rows (per-sample form): 2^4 .. 2^13 / 2^14, 16 elements per thread
#define RSW_ROW_CASE(R, L) \
    case L: return chirp ? (e == 32 ? row_impl<R, L, 32, true>(a, s) : row_impl<R, L, 16, true>(a, s)) \
                         : row_impl<R, L, 16, false>(a, s);
#define RSW_ROW_CASE16(R, L) \
    case L: return chirp ? row_impl<R, L, 16, true>(a, s) : row_impl<R, L, 16, false>(a, s);
// rows with 8 samples per thread (radix-8 stages, twice the threads)
#define RSW_ROW_CASE8(R, L) \
    case L: return chirp ? (e == 8 ? row_impl<R, L, 8, true>(a, s) \
                                   : e == 32 ? row_impl<R, L, 32, true>(a, s) : row_impl<R, L, 16, true>(a, s)) \
                         : row_impl<R, L, 16, false>(a, s);
#define RSW_ROW_CASE_S(R, L) \
    case L: return chirp ? cudaErrorInvalidValue : row_impl<R, L, 16, false>(a, s);

cudaError_t launch_row_pass_f32(const PassArgs &a, int e, cudaStream_t s) {
    // multi-level rows take the chirp form of the Fresnel kernel; the exact
    // kernel and single-level rows evaluate the transfer function per sample
    const bool chirp = a.log_n1 > 0 && !a.pr.exact;
    switch (a.log_n2) {
        RSW_ROW_CASE_S(float, 4) RSW_ROW_CASE_S(float, 5) RSW_ROW_CASE_S(float, 6) RSW_ROW_CASE16(float, 7)
        RSW_ROW_CASE16(float, 8) RSW_ROW_CASE(float, 9) RSW_ROW_CASE(float, 10) RSW_ROW_CASE8(float, 11)
        RSW_ROW_CASE8(float, 12) RSW_ROW_CASE8(float, 13) RSW_ROW_CASE(float, 14)
    default: return cudaErrorInvalidValue;
        }
}
}  // namespace rsw
