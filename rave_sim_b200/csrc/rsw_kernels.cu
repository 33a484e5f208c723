// Split-step wavefront propagation kernels for B200 (sm_100a).
//
// The field of N = N1 * N2 samples is viewed as N1 rows of N2 contiguous
// samples. One split step (reference: big-wave/propagation.py:100-138 preceded
// by a transmission multiply, big-wave/optical_element.py:134-206/:432-476)
// is two passes over HBM:
//
//   column pass  one CTA per C adjacent columns: inverse column FFT of the
//                previous step, transmission multiply at x(n), forward column
//                FFT, four-step twiddle W_N^(n2*k1);
//   row pass     one CTA per row: forward row FFT, Fresnel transfer function
//                and frequency cutoff on the digit-reversed spectrum,
//                inverse row FFT, conjugate twiddle and 1/N.
//
// Between steps the buffer holds the "mid" representation (after the row
// pass); the field itself (natural order) only exists inside the column pass,
// where the transmission needs it. Small fields (N <= one block) use a single
// row pass per step.
#include <cuda_runtime.h>
#include <stdint.h>

#include "rsw_block_fft.cuh"
#include "rsw_internal.h"

namespace rsw {

// ---------------------------------------------------------------- counters
__device__ __forceinline__ double rint_d(double x) { return rint(x); }

// Range reduction of a phase to [-pi, pi] (Cody & Waite 1980, three-part
// constant; 2pi = P1 + P2 + P3 with P1, P2 of 29 significant bits so that
// k*P1 and k*P2 are exact for |k| < 2^24), then sincos of the remainder.
__device__ __forceinline__ void sincos_phase(double th, double *s, double *c) {
    const double P1 = 0x1.921fb54000000p+2;
    const double P2 = 0x1.10b4612000000p-28;
    const double P3 = -0x1.676733ae8fe48p-58;
    const double INV2PI = 0x1.45f306dc9c883p-3;
    const double k = rint_d(th * INV2PI);
    if (fabs(k) < 16777216.0) {
        double r = fma(-k, P1, th);
        r = fma(-k, P2, r);
        r = fma(-k, P3, r);
        sincos(r, s, c);
    } else {
        sincos(th, s, c);
    }
}
__device__ __forceinline__ double reduce_phase(double th) {
    const double P1 = 0x1.921fb54000000p+2;
    const double P2 = 0x1.10b4612000000p-28;
    const double P3 = -0x1.676733ae8fe48p-58;
    const double INV2PI = 0x1.45f306dc9c883p-3;
    const double k = rint_d(th * INV2PI);
    double r = fma(-k, P1, th);
    r = fma(-k, P2, r);
    return fma(-k, P3, r);
}

// ------------------------------------------------------------- transmission
__device__ __forceinline__ double grating_x(const TransArgs &t, int64_t n) {
    // np.linspace(x_start, x_stop, cnt, endpoint=False) of the chunk holding n:
    // x = fl(fl(l * step) + x_start)   (big-wave/optical_element.py:352-354)
    if (t.chunk_size <= 0) return __dadd_rn(__dmul_rn(double(n), t.step0), t.xstart0);
    const int64_t ch = n / t.chunk_size;
    const int64_t l = n - ch * t.chunk_size;
    return __dadd_rn(__dmul_rn(double(l), __ldg(t.chunk_step + ch)), __ldg(t.chunk_xstart + ch));
}

// np.mod(x / p + off, 1) < dc  (np.mod(a, 1) == a - floor(a) for finite a)
__device__ __forceinline__ bool mod_less(double x, double p, double off, double dc) {
    const double a = __dadd_rn(__ddiv_rn(x, p), off);
    return __dsub_rn(a, floor(a)) < dc;
}

__device__ __forceinline__ double sample_row_x(const TransArgs &t, int64_t j) {
    // row_x = np.arange(rowlen) * psx + x_pos - rowlen * psx * 0.5
    return __dsub_rn(__dadd_rn(__dmul_rn(double(j), t.psx), t.sample_xpos), t.sample_hw);
}

// Sample row factor at sample n: exp(i y * np.interp(x, row_x, row_db, 0, 0))
// (big-wave/optical_element.py:452-472). Returns false for vacuum (factor 1).
__device__ __forceinline__ bool sample_factor(const TransArgs &t, int64_t n, double2 *f) {
    const double x = __dmul_rn(double(n) - t.half_n, t.dx);
    const int64_t last = t.x_len - 1;
    const double x0 = sample_row_x(t, 0);
    const double xl = sample_row_x(t, last);
    if (x < x0 || x > xl) return false;
    int mi;
    if (x == xl) {
        mi = t.row_grid[last];
        if (mi == 0) return false;
        *f = t.mat_factor[mi];
        return true;
    }
    int64_t j = int64_t(floor((x - x0) * t.sample_inv_psx));
    j = j < 0 ? 0 : (j > last - 1 ? last - 1 : j);
    // move to the bracket row_x[j] <= x < row_x[j+1] (bounded)
    for (int it = 0; it < 4 && j > 0 && x < sample_row_x(t, j); ++it) --j;
    for (int it = 0; it < 4 && j < last - 1 && x >= sample_row_x(t, j + 1); ++it) ++j;
    const int m0 = t.row_grid[j];
    const int m1 = t.row_grid[j + 1];
    const double xj = sample_row_x(t, j);
    if (m0 == m1 || x == xj) {
        if (m0 == 0) return false;
        *f = t.mat_factor[m0];
        return true;
    }
    const double2 d0 = t.mat_db[m0], d1 = t.mat_db[m1];
    const double dxp = __dsub_rn(sample_row_x(t, j + 1), xj);
    const double sre = __ddiv_rn(__dsub_rn(d1.x, d0.x), dxp);
    const double sim = __ddiv_rn(__dsub_rn(d1.y, d0.y), dxp);
    const double xr = __dsub_rn(x, xj);
    const double dre = __dadd_rn(__dmul_rn(sre, xr), d0.x);
    const double dim = __dadd_rn(__dmul_rn(sim, xr), d0.y);
    // exp((0, y) * (dre, dim)) = exp(-y*dim) * (cos(y*dre), sin(y*dre))
    const double amp = exp(-__dmul_rn(t.sample_y, dim));
    double s, c;
    sincos(__dmul_rn(t.sample_y, dre), &s, &c);
    *f = make_double2(amp * c, amp * s);
    return true;
}

__device__ __forceinline__ double2 to_c(double2 a, double2) { return a; }
__device__ __forceinline__ float2 to_c(double2 a, float2) { return make_float2(float(a.x), float(a.y)); }

template <typename Cx> __device__ __forceinline__ Cx apply_trans(const TransArgs &t, int64_t n, Cx u) {
    switch (t.kind) {
    case TR_SCALAR: return cmul(u, to_c(t.fa, u));
    case TR_GRATING: {
        const double x = grating_x(t, n);
        const bool m = mod_less(x, t.pitch0, t.half_dc0, t.dc0);
        return cmul(u, to_c(m ? t.fa : t.fb, u));
    }
    case TR_DBA: {
        const double x = grating_x(t, n);
        const bool m = mod_less(x, t.pitch0, t.half_dc0, t.dc0) && mod_less(x, t.pitch1, 0.0, t.dc1);
        return cmul(u, to_c(m ? t.fa : t.fb, u));
    }
    case TR_SAMPLE: {
        double2 f;
        if (!sample_factor(t, n, &f)) return u;
        // computed in FP64, stored in the field's precision
        const double2 ud = make_double2(double(u.x), double(u.y));
        return to_c(cmul(ud, f), u);
    }
    default: return u;
    }
}

// ------------------------------------------------------------ propagator
// U *= exp(-i2pi dz/wl) * exp(i pi wl dz fx^2), fx = (ks * (1/N)) / dx, zero in
// the cutoff range (big-wave/propagation.py:74-97, :124-137).
__device__ __forceinline__ double2 prop_apply(const PropArgs &p, int64_t k, int64_t ks, double2 U) {
    if (p.has_cut && k >= p.cut_lo && k < p.cut_hi) return make_double2(0.0, 0.0);
    if (!p.has_h) return U;
    const double fx = __ddiv_rn(__dmul_rn(double(ks), p.fac), p.dx);
    const double th = __dmul_rn(p.c, __dmul_rn(fx, fx));
    double s, c;
    sincos_phase(th, &s, &c);
    const double2 H = make_double2(p.A.x * c - p.A.y * s, p.A.x * s + p.A.y * c);
    return cmul(U, H);
}
__device__ __forceinline__ float2 prop_apply(const PropArgs &p, int64_t k, int64_t ks, float2 U) {
    if (p.has_cut && k >= p.cut_lo && k < p.cut_hi) return make_float2(0.f, 0.f);
    if (!p.has_h) return U;
    const double fx = __ddiv_rn(__dmul_rn(double(ks), p.fac), p.dx);
    const double th = __dmul_rn(p.c, __dmul_rn(fx, fx));
    float s, c;
    sincosf(float(reduce_phase(th)), &s, &c);
    const float ax = float(p.A.x), ay = float(p.A.y);
    const float2 H = make_float2(ax * c - ay * s, ax * s + ay * c);
    return cmul(U, H);
}

template <typename Cx> __device__ __forceinline__ Cx one_c();
template <> __device__ __forceinline__ double2 one_c<double2>() { return make_double2(1.0, 0.0); }
template <> __device__ __forceinline__ float2 one_c<float2>() { return make_float2(1.f, 0.f); }

// ------------------------------------------------------------------ passes
template <typename Real, int LOG_L2>
__global__ void __launch_bounds__(Block<Real, LOG_L2, 1>::NT) row_pass_kernel(PassArgs a) {
    using B = Block<Real, LOG_L2, 1>;
    using Cx = typename B::Cx;
    extern __shared__ __align__(16) unsigned char smraw[];
    Cx *sm = reinterpret_cast<Cx *>(smraw);
    const int tp = threadIdx.x;
    const int64_t row = blockIdx.x;
    const Cx *__restrict__ gin = static_cast<const Cx *>(a.in) + (row << LOG_L2);
    Cx *__restrict__ gout = static_cast<Cx *>(a.out) + (row << LOG_L2);
    const Cx *twr = static_cast<const Cx *>(a.tw_row);
    const int flags = a.flags;
    Cx v[16];

    if (!(flags & PF_SPEC_IN)) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int p = B::first_pos(tp, r);
            v[r] = (flags & PF_ONES) ? one_c<Cx>() : gin[p];
        }
        if (flags & PF_TRANS) {
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = apply_trans(a.tr, (row << LOG_L2) + B::first_pos(tp, r), v[r]);
        }
        if (flags & PF_FWD) B::forward(sm, tp, v, twr);
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = gin[B::last_pos(tp, r)];
    }

    if (a.pr.has_h || a.pr.has_cut) {
        const int64_t k1 = digitrev_rt(row, a.log_n1);
        const int64_t half2 = int64_t(1) << (LOG_L2 - 1);
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int64_t k2 = digitrev_rt(B::last_pos(tp, r), LOG_L2);
            const int64_t k = k1 + (k2 << a.log_n1);
            const int64_t k2s = k2 >= half2 ? k2 - 2 * half2 : k2;
            const int64_t ks = k1 + k2s * (int64_t(1) << a.log_n1);
            v[r] = prop_apply(a.pr, k, ks, v[r]);
        }
    }

    if (flags & PF_INV) {
        B::inverse(sm, tp, v, twr);
        if (flags & PF_TW) {
            const int64_t k1 = digitrev_rt(row, a.log_n1);
            const Cx *lo = static_cast<const Cx *>(a.tw4_lo);
            const Cx *hi = static_cast<const Cx *>(a.tw4_hi_inv);
            const int64_t mask = (int64_t(1) << a.tw4_shift) - 1;
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int64_t m = int64_t(B::first_pos(tp, r)) * k1;
                v[r] = cmul(cmulc(v[r], __ldg(lo + (m & mask))), __ldg(hi + (m >> a.tw4_shift)));
            }
        } else if (flags & PF_SCALE) {
            const Real f = Real(a.pr.fac);
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = cscale(v[r], f);
        }
#pragma unroll
        for (int r = 0; r < 16; ++r) gout[B::first_pos(tp, r)] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) gout[B::last_pos(tp, r)] = v[r];
    }
}

template <typename Real, int LOG_L1, int C>
__global__ void __launch_bounds__(Block<Real, LOG_L1, C>::NT) col_pass_kernel(PassArgs a) {
    using B = Block<Real, LOG_L1, C>;
    using Cx = typename B::Cx;
    extern __shared__ __align__(16) unsigned char smraw[];
    const int t = threadIdx.x;
    const int c = t % C;
    const int tp = t / C;
    Cx *sm = reinterpret_cast<Cx *>(smraw) + c * B::PITCH;
    const int64_t col = int64_t(blockIdx.x) * C + c;
    const int log_n2 = a.log_n2;
    const Cx *__restrict__ gin = static_cast<const Cx *>(a.in) + col;
    Cx *__restrict__ gout = static_cast<Cx *>(a.out) + col;
    const Cx *twc = static_cast<const Cx *>(a.tw_col);
    const int flags = a.flags;
    Cx v[16];

    if (flags & PF_INV) {
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = gin[int64_t(B::last_pos(tp, r)) << log_n2];
        B::inverse(sm, tp, v, twc);
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r)
            v[r] = (flags & PF_ONES) ? one_c<Cx>() : gin[int64_t(B::first_pos(tp, r)) << log_n2];
    }
    if (flags & PF_TRANS) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
            v[r] = apply_trans(a.tr, (int64_t(B::first_pos(tp, r)) << log_n2) + col, v[r]);
    }
    if (flags & PF_FWD) {
        B::forward(sm, tp, v, twc);
        if (flags & PF_TW) {
            const Cx *lo = static_cast<const Cx *>(a.tw4_lo);
            const Cx *hi = static_cast<const Cx *>(a.tw4_hi);
            const int64_t mask = (int64_t(1) << a.tw4_shift) - 1;
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                const int64_t m = col * digitrev_rt(B::last_pos(tp, r), LOG_L1);
                v[r] = cmul(v[r], cmul(__ldg(lo + (m & mask)), __ldg(hi + (m >> a.tw4_shift))));
            }
        }
#pragma unroll
        for (int r = 0; r < 16; ++r) gout[int64_t(B::last_pos(tp, r)) << log_n2] = v[r];
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) gout[int64_t(B::first_pos(tp, r)) << log_n2] = v[r];
    }
}

// ---------------------------------------------------------- small kernels
// internal spectrum layout <-> natural frequency order
template <typename Cx>
__global__ void spec_to_natural_kernel(const Cx *__restrict__ in, Cx *__restrict__ out, int64_t n,
                                       int log_n1, int log_n2) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t mask1 = (int64_t(1) << log_n1) - 1;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int64_t k1 = k & mask1, k2 = k >> log_n1;
        const int64_t addr = (digitpos_rt(k1, log_n1) << log_n2) + digitpos_rt(k2, log_n2);
        out[k] = in[addr];
    }
}
template <typename Cx>
__global__ void natural_to_spec_kernel(const Cx *__restrict__ in, Cx *__restrict__ out, int64_t n,
                                       int log_n1, int log_n2) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t mask1 = (int64_t(1) << log_n1) - 1;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int64_t k1 = k & mask1, k2 = k >> log_n1;
        const int64_t addr = (digitpos_rt(k1, log_n1) << log_n2) + digitpos_rt(k2, log_n2);
        out[addr] = in[k];
    }
}

template <typename Cx>
__global__ void trans_kernel(Cx *__restrict__ u, int64_t n, TransArgs tr) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        u[i] = apply_trans(tr, i, u[i]);
}

template <typename Cx>
__global__ void copy_kernel(const Cx *__restrict__ in, Cx *__restrict__ out, int64_t n) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = in[i];
}

// exp(r * (-2 pi i / wl)) / sqrt(r), x = (i - N/2) dx - x_src, r = sqrt(x^2 + z^2)
// (big-wave/propagation.py:141-151)
template <typename Cx>
__global__ void point_source_kernel(Cx *__restrict__ u, int64_t n, double dx, double w, double z,
                                    double x_src) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const double half = double(n / 2);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = __dsub_rn(__dmul_rn(double(i) - half, dx), x_src);
        const double r = sqrt(__dadd_rn(__dmul_rn(x, x), __dmul_rn(z, z)));
        double s, c;
        sincos(__dmul_rn(r, w), &s, &c);
        const double scl = 1.0 / sqrt(r);
        u[i] = to_c(make_double2(c * scl, s * scl), u[i]);
    }
}

// Detector binning: pixel j sums |u|^2 over samples [bounds[j], bounds[j+1]),
// then (((sum * cos_j) * dx) * psy) / r_j; optional compensated accumulation
// acc[j] += weight * value.
template <typename Cx>
__global__ void detect_kernel(const Cx *__restrict__ u, const int64_t *__restrict__ bounds,
                              const double *__restrict__ cosv, const double *__restrict__ rv, double dx,
                              double psy, double *__restrict__ out, double *__restrict__ acc,
                              double *__restrict__ comp, double weight) {
    const int j = blockIdx.x;
    const int64_t lo = bounds[j], hi = bounds[j + 1];
    double s = 0.0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const Cx v = u[i];
        const double re = double(v.x), im = double(v.y);
        s += re * re + im * im;
    }
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        s = threadIdx.x < nw ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) {
            const double val = (((s * cosv[j]) * dx) * psy) / rv[j];
            if (out) out[j] = val;
            if (acc) {
                const double y = __dsub_rn(__dmul_rn(weight, val), comp[j]);
                const double t = __dadd_rn(acc[j], y);
                comp[j] = __dsub_rn(__dsub_rn(t, acc[j]), y);
                acc[j] = t;
            }
        }
    }
}

__global__ void zero_kernel(double *__restrict__ p, int64_t n) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = 0.0;
}

// ------------------------------------------------------------ launchers
static unsigned long long g_launches = 0;  // host-side count of kernel launches

template <typename K> static cudaError_t prep(K kernel, size_t smem) {
    if (smem > 48 * 1024) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    return cudaSuccess;
}

template <typename Real, int LG> static cudaError_t row_impl(const PassArgs &a, cudaStream_t s) {
    using B = Block<Real, LG, 1>;
    auto k = row_pass_kernel<Real, LG>;
    static cudaError_t attr = prep(k, B::SMEM);
    if (attr != cudaSuccess) return attr;
    const int64_t rows = a.n >> LG;
    k<<<dim3(unsigned(rows)), dim3(B::NT), B::SMEM, s>>>(a);
    ++g_launches;
    return cudaGetLastError();
}

template <typename Real, int LG, int C> static cudaError_t col_impl(const PassArgs &a, cudaStream_t s) {
    using B = Block<Real, LG, C>;
    auto k = col_pass_kernel<Real, LG, C>;
    static cudaError_t attr = prep(k, B::SMEM);
    if (attr != cudaSuccess) return attr;
    const int64_t tiles = (int64_t(1) << a.log_n2) / C;
    k<<<dim3(unsigned(tiles)), dim3(B::NT), B::SMEM, s>>>(a);
    ++g_launches;
    return cudaGetLastError();
}

#define RSW_ROW_CASE(R, L) \
    case L: return row_impl<R, L>(a, s);
#define RSW_COL_CASE(R, L, C) \
    case L: return col_impl<R, L, C>(a, s);

cudaError_t launch_row_pass(const PassArgs &a, bool dbl, cudaStream_t s) {
    if (dbl) {
        switch (a.log_n2) {
            RSW_ROW_CASE(double, 4) RSW_ROW_CASE(double, 5) RSW_ROW_CASE(double, 6) RSW_ROW_CASE(double, 7)
            RSW_ROW_CASE(double, 8) RSW_ROW_CASE(double, 9) RSW_ROW_CASE(double, 10) RSW_ROW_CASE(double, 11)
            RSW_ROW_CASE(double, 12) RSW_ROW_CASE(double, 13)
        default: return cudaErrorInvalidValue;
        }
    }
    switch (a.log_n2) {
        RSW_ROW_CASE(float, 4) RSW_ROW_CASE(float, 5) RSW_ROW_CASE(float, 6) RSW_ROW_CASE(float, 7)
        RSW_ROW_CASE(float, 8) RSW_ROW_CASE(float, 9) RSW_ROW_CASE(float, 10) RSW_ROW_CASE(float, 11)
        RSW_ROW_CASE(float, 12) RSW_ROW_CASE(float, 13) RSW_ROW_CASE(float, 14)
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_col_pass(const PassArgs &a, bool dbl, cudaStream_t s) {
    if (dbl) {
        switch (a.log_n1) {
            RSW_COL_CASE(double, 4, 4) RSW_COL_CASE(double, 5, 4) RSW_COL_CASE(double, 6, 4)
            RSW_COL_CASE(double, 7, 4) RSW_COL_CASE(double, 8, 4) RSW_COL_CASE(double, 9, 4)
            RSW_COL_CASE(double, 10, 4) RSW_COL_CASE(double, 11, 4)
        default: return cudaErrorInvalidValue;
        }
    }
    switch (a.log_n1) {
        RSW_COL_CASE(float, 4, 4) RSW_COL_CASE(float, 5, 4) RSW_COL_CASE(float, 6, 4)
        RSW_COL_CASE(float, 7, 4) RSW_COL_CASE(float, 8, 4) RSW_COL_CASE(float, 9, 4)
        RSW_COL_CASE(float, 10, 4) RSW_COL_CASE(float, 11, 4) RSW_COL_CASE(float, 12, 4)
    default: return cudaErrorInvalidValue;
    }
}

static unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    const int64_t cap = 148 * 32;
    return unsigned(b < 1 ? 1 : (b > cap ? cap : b));
}

cudaError_t launch_spec_to_natural(const void *in, void *out, int64_t n, int log_n1, int log_n2, bool dbl,
                                   cudaStream_t s) {
    ++g_launches;
    if (dbl)
        spec_to_natural_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)in, (double2 *)out, n,
                                                                          log_n1, log_n2);
    else
        spec_to_natural_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)in, (float2 *)out, n,
                                                                        log_n1, log_n2);
    return cudaGetLastError();
}
cudaError_t launch_natural_to_spec(const void *in, void *out, int64_t n, int log_n1, int log_n2, bool dbl,
                                   cudaStream_t s) {
    ++g_launches;
    if (dbl)
        natural_to_spec_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)in, (double2 *)out, n,
                                                                          log_n1, log_n2);
    else
        natural_to_spec_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)in, (float2 *)out, n,
                                                                        log_n1, log_n2);
    return cudaGetLastError();
}
cudaError_t launch_trans(void *u, int64_t n, const TransArgs &tr, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) trans_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((double2 *)u, n, tr);
    else trans_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((float2 *)u, n, tr);
    return cudaGetLastError();
}
cudaError_t launch_copy(const void *in, void *out, int64_t n, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) copy_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)in, (double2 *)out, n);
    else copy_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)in, (float2 *)out, n);
    return cudaGetLastError();
}
cudaError_t launch_point_source(void *u, int64_t n, double dx, double w, double z, double x_src, bool dbl,
                                cudaStream_t s) {
    ++g_launches;
    if (dbl) point_source_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((double2 *)u, n, dx, w, z, x_src);
    else point_source_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((float2 *)u, n, dx, w, z, x_src);
    return cudaGetLastError();
}
cudaError_t launch_detect(const void *u, const int64_t *bounds, const double *cosv, const double *rv,
                          int64_t n_pix, double dx, double psy, double *out, double *acc, double *comp,
                          double weight, bool dbl, cudaStream_t s) {
    if (n_pix <= 0) return cudaSuccess;
    ++g_launches;
    if (dbl)
        detect_kernel<double2><<<unsigned(n_pix), 256, 0, s>>>((const double2 *)u, bounds, cosv, rv, dx, psy, out,
                                                             acc, comp, weight);
    else
        detect_kernel<float2><<<unsigned(n_pix), 256, 0, s>>>((const float2 *)u, bounds, cosv, rv, dx, psy, out,
                                                           acc, comp, weight);
    return cudaGetLastError();
}
cudaError_t launch_zero(double *p, int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    ++g_launches;
    zero_kernel<<<grid_for(n, 256), 256, 0, s>>>(p, n);
    return cudaGetLastError();
}
unsigned long long launch_count() { return g_launches; }

}  // namespace rsw

namespace rsw {
template <typename Cx> __global__ void fill_ones_kernel(Cx *__restrict__ u, int64_t n) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) u[i] = one_c<Cx>();
}
cudaError_t launch_fill_ones(void *u, int64_t n, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) fill_ones_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((double2 *)u, n);
    else fill_ones_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((float2 *)u, n);
    return cudaGetLastError();
}
}  // namespace rsw
