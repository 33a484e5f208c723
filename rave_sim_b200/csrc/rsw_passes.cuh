// Split-step wavefront propagation kernels for B200 (sm_100a): device code
// shared by the translation units rsw_row_f64.cu, rsw_row_f32.cu, rsw_col.cu
// and rsw_kernels.cu.
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
// row pass per step. Three-level plans (N = N1 * Nb * Nr) add a middle pass
// over Nb between the two (the column kernel as a plain batched FFT), with
// the W_{N2} twiddles in the row pass. The row pass prefetches its next row
// into L2 while it transforms the current one. Both kernels also run over
// batches of transforms (n a multiple of one transform's length): rows and
// column tiles index within their own transform.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "rsw_block_fft.cuh"
#include "rsw_internal.h"

namespace rsw {

// ---------------------------------------------------------------- counters
__device__ __forceinline__ double rint_d(double x) { return rint(x); }

// L2 prefetch of [p, p + bytes): p 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
// L2 prefetch of the box of a 2-D TMA map at (x, y) (x in elements of the
// map; x times the element size a multiple of 16 bytes)
__device__ __forceinline__ void prefetch_l2_tile(const CUtensorMap *map, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y)
                 : "memory");
}

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

// Correctly rounded x / d from the correctly rounded reciprocal r = 1/d and
// one FMA correction (Markstein's theorem).
__device__ __forceinline__ double div_rn(double x, double d, double r) {
    const double q0 = x * r;
    return fma(fma(-q0, d, x), r, q0);
}

// np.mod(x / p + off, 1) < dc  (np.mod(a, 1) == a - floor(a) for finite a)
__device__ __forceinline__ bool mod_less(double x, double p, double rp, double off, double dc) {
    const double a = __dadd_rn(div_rn(x, p, rp), off);
    return __dsub_rn(a, floor(a)) < dc;
}

__device__ __forceinline__ double sample_row_x(const TransArgs &t, int64_t j) {
    // row_x = np.arange(rowlen) * psx + x_pos - rowlen * psx * 0.5
    return __dsub_rn(__dadd_rn(__dmul_rn(double(j), t.psx), t.sample_xpos), t.sample_hw);
}

static __device__ __noinline__ double2 sample_interp(const double2 *mat_db, double psx, double xpos, double hw,
                                                     double y, int64_t j, int m0, int m1, double x, double xj);

// Sample row factor at sample n: exp(i y * np.interp(x, row_x, row_db, 0, 0))
// (big-wave/optical_element.py:452-472). Returns false for vacuum (factor 1).
// The material tables and y are the instance's (t's own, or a batch entry's).
__device__ __forceinline__ bool sample_factor(const TransArgs &t, const double2 *mat_db, const double2 *mat_factor,
                                              double y, int64_t n, double2 *f) {
    const double x = __dmul_rn(double(n) - t.half_n, t.dx);
    const int64_t last = t.x_len - 1;
    const double x0 = sample_row_x(t, 0);
    const double xl = sample_row_x(t, last);
    if (x < x0 || x > xl) return false;
    int mi;
    if (x == xl) {
        mi = t.row_grid[last];
        if (mi == 0) return false;
        *f = mat_factor[mi];
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
        *f = mat_factor[m0];
        return true;
    }
    // scalars by value: a reference to the kernel parameter would force it into local memory
    *f = sample_interp(mat_db, t.psx, t.sample_xpos, t.sample_hw, y, j, m0, m1, x, xj);
    return true;
}

// Interpolated delta+i*beta between two different pixels and its factor
// exp(i y db); kept out of line (only samples at material boundaries get here).
static __device__ __noinline__ double2 sample_interp(const double2 *mat_db, double psx, double xpos, double hw,
                                                     double y, int64_t j, int m0, int m1, double x, double xj) {
    const double2 d0 = mat_db[m0], d1 = mat_db[m1];
    const double xj1 = __dsub_rn(__dadd_rn(__dmul_rn(double(j + 1), psx), xpos), hw);
    const double dxp = __dsub_rn(xj1, xj);
    const double sre = __ddiv_rn(__dsub_rn(d1.x, d0.x), dxp);
    const double sim = __ddiv_rn(__dsub_rn(d1.y, d0.y), dxp);
    const double xr = __dsub_rn(x, xj);
    const double dre = __dadd_rn(__dmul_rn(sre, xr), d0.x);
    const double dim = __dadd_rn(__dmul_rn(sim, xr), d0.y);
    // exp((0, y) * (dre, dim)) = exp(-y*dim) * (cos(y*dre), sin(y*dre))
    const double amp = exp(-__dmul_rn(y, dim));
    double s, c;
    sincos(__dmul_rn(y, dre), &s, &c);
    return make_double2(amp * c, amp * s);
}

__device__ __forceinline__ double2 to_c(double2 a, double2) { return a; }
__device__ __forceinline__ float2 to_c(double2 a, float2) { return make_float2(float(a.x), float(a.y)); }

// u * f for a transmission factor with every rounding explicit (one product
// rounded, one fused), so that every kernel variant that transmits (the
// plain and the batched passes) rounds the same way
__device__ __forceinline__ float2 tmul(float2 u, float2 f) {
    return make_float2(__fmaf_rn(u.x, f.x, -__fmul_rn(u.y, f.y)), __fmaf_rn(u.x, f.y, __fmul_rn(u.y, f.x)));
}
__device__ __forceinline__ double2 tmul(double2 u, double2 f) {
    return make_double2(__fma_rn(u.x, f.x, -__dmul_rn(u.y, f.y)), __fma_rn(u.x, f.y, __dmul_rn(u.y, f.x)));
}

template <typename Cx> __device__ __forceinline__ Cx apply_trans(const TransArgs &t, int64_t n, Cx u) {
    switch (t.kind) {
    case TR_SCALAR: return tmul(u, to_c(t.fa, u));
    case TR_GRATING: {
        const double x = grating_x(t, n);
        const bool m = mod_less(x, t.pitch0, t.inv_pitch0, t.half_dc0, t.dc0);
        return tmul(u, to_c(m ? t.fa : t.fb, u));
    }
    case TR_DBA: {
        const double x = grating_x(t, n);
        const bool m = mod_less(x, t.pitch0, t.inv_pitch0, t.half_dc0, t.dc0) &&
                       mod_less(x, t.pitch1, t.inv_pitch1, 0.0, t.dc1);
        return tmul(u, to_c(m ? t.fa : t.fb, u));
    }
    case TR_SAMPLE: {
        double2 f;
        if (!sample_factor(t, t.mat_db, t.mat_factor, t.sample_y, n, &f)) return u;
        // computed in FP64, stored in the field's precision
        const double2 ud = make_double2(double(u.x), double(u.y));
        return to_c(tmul(ud, f), u);
    }
    default: return u;
    }
}

// apply_trans to the E samples of a thread, sample r at index pos(r), with the
// kind of transmission decided once for all of them. In the column kernel
// this keeps the compiler from holding every kind's temporaries across the
// unrolled samples (the 2^11 complex128 kernel at 16 per thread spilled 204
// bytes per thread before, none after); the row kernel, which transmits only
// in single-level plans, keeps the per-sample form (its two-level code ran 6 %
// slower with this one).
template <int E, typename Cx, typename Pos>
__device__ __forceinline__ void apply_trans_e(const TransArgs &t, Pos pos, Cx *v) {
    switch (t.kind) {
    case TR_SCALAR: {
        const Cx f = to_c(t.fa, Cx{});
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = tmul(v[r], f);
        break;
    }
    case TR_GRATING:
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const double x = grating_x(t, pos(r));
            const bool m = mod_less(x, t.pitch0, t.inv_pitch0, t.half_dc0, t.dc0);
            v[r] = tmul(v[r], to_c(m ? t.fa : t.fb, Cx{}));
        }
        break;
    case TR_DBA:
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const double x = grating_x(t, pos(r));
            const bool m = mod_less(x, t.pitch0, t.inv_pitch0, t.half_dc0, t.dc0) &&
                           mod_less(x, t.pitch1, t.inv_pitch1, 0.0, t.dc1);
            v[r] = tmul(v[r], to_c(m ? t.fa : t.fb, Cx{}));
        }
        break;
    case TR_SAMPLE:
#pragma unroll
        for (int r = 0; r < E; ++r) {
            double2 f;
            if (sample_factor(t, t.mat_db, t.mat_factor, t.sample_y, pos(r), &f)) {
                const double2 ud = make_double2(double(v[r].x), double(v[r].y));
                v[r] = to_c(tmul(ud, f), Cx{});
            }
        }
        break;
    default: break;
    }
}

// apply_trans_e for one instance of a batched pass: the geometry from t, the
// wavelength-dependent factors from the instance's entry b (loaded once per
// tile, outside the unrolled samples)
template <int E, typename Cx, typename Pos>
__device__ __forceinline__ void apply_trans_batch(const TransArgs &t, const BatchTrans *__restrict__ b, Pos pos, Cx *v) {
    switch (t.kind) {
    case TR_SCALAR: {
        const Cx f = to_c(__ldg(&b->fa), Cx{});
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = tmul(v[r], f);
        break;
    }
    case TR_GRATING:
    case TR_DBA: {
        const Cx fa = to_c(__ldg(&b->fa), Cx{}), fb = to_c(__ldg(&b->fb), Cx{});
        const bool dba = t.kind == TR_DBA;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const double x = grating_x(t, pos(r));
            const bool m = mod_less(x, t.pitch0, t.inv_pitch0, t.half_dc0, t.dc0) &&
                           (!dba || mod_less(x, t.pitch1, t.inv_pitch1, 0.0, t.dc1));
            v[r] = tmul(v[r], m ? fa : fb);
        }
        break;
    }
    case TR_SAMPLE: {
        const double2 *mdb = b->mat_db, *mf = b->mat_factor;
        const double y = b->sample_y;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            double2 f;
            if (sample_factor(t, mdb, mf, y, pos(r), &f)) {
                const double2 ud = make_double2(double(v[r].x), double(v[r].y));
                v[r] = to_c(tmul(ud, f), Cx{});
            }
        }
        break;
    }
    default: break;
    }
}

// ------------------------------------------------------------ propagator
// U *= exp(-i2pi dz/wl) * exp(i pi wl dz fx^2), fx = (ks * (1/N)) / dx, zero in
// the cutoff range (big-wave/propagation.py:74-97, :124-137).
// (ks * 2^-n) / dx == 2^-n * (ks / dx) exactly; ks / dx is the correctly
// rounded quotient from the reciprocal and one FMA correction (Markstein).
__device__ __forceinline__ double prop_phase(const PropArgs &p, int64_t ks) {
    const double fx = __dmul_rn(div_rn(double(ks), p.dx, p.rdx), p.fac);
    return __dmul_rn(p.c, __dmul_rn(fx, fx));
}

// frac((hi + lo) * m) in [-0.5, 0.5] for an integer-valued m < 2^53, with the
// product error recovered by FMA (double-double argument, in turns).
__device__ __forceinline__ double frac_dd(double hi, double lo, double m) {
    const double p = hi * m;
    const double e = fma(hi, m, -p);
    double r = (p - rint(p)) + fma(lo, m, e);
    return r - rint(r);
}

// exp(2 pi i t) for t in turns
__device__ __forceinline__ double2 cis_turns(double t) {
    double s, c;
    sincospi(2.0 * t, &s, &c);
    return make_double2(c, s);
}
// Phase of the exact angular-spectrum kernel beyond the constant -2 pi dz / wl
// (carried in A): 2 pi dz (1/wl - sqrt(1/wl^2 - fx^2)) written without the
// cancellation as 2 pi dz fx^2 / (1/wl + sqrt(1/wl^2 - fx^2)), fx as in
// prop_phase. False for an evanescent component (fx^2 >= 1/wl^2).
__device__ __forceinline__ bool exact_phase(const PropArgs &p, int64_t ks, double *phi) {
    const double fx = __dmul_rn(div_rn(double(ks), p.dx, p.rdx), p.fac);
    const double f2 = __dmul_rn(fx, fx);
    const double d = __dsub_rn(p.inv_wl2, f2);
    if (!(d > 0.0)) return false;
    *phi = __ddiv_rn(__dmul_rn(p.z2pi, f2), __dadd_rn(p.inv_wl, __dsqrt_rn(d)));
    return true;
}
// the per-sample phase of the transfer function: Fresnel (the reference's) or
// exact; false: the component is zeroed
__device__ __forceinline__ bool prop_phase_any(const PropArgs &p, int64_t ks, double *phi) {
    if (p.exact) return exact_phase(p, ks, phi);
    *phi = prop_phase(p, ks);
    return true;
}
__device__ __forceinline__ double2 prop_apply(const PropArgs &p, int64_t k, int64_t ks, double2 U) {
    if (p.has_cut && k >= p.cut_lo && k < p.cut_hi) return make_double2(0.0, 0.0);
    if (!p.has_h) return U;
    double s, c, ph;
    if (!prop_phase_any(p, ks, &ph)) return make_double2(0.0, 0.0);
    sincos_phase(ph, &s, &c);
    const double2 H = make_double2(p.A.x * c - p.A.y * s, p.A.x * s + p.A.y * c);
    return cmul(U, H);
}
// complex64: the transfer function in FP64, applied by lifting (no
// amplitude bias from rounding H to FP32)
__device__ __forceinline__ float2 prop_apply(const PropArgs &p, int64_t k, int64_t ks, float2 U) {
    if (p.has_cut && k >= p.cut_lo && k < p.cut_hi) return make_float2(0.f, 0.f);
    if (!p.has_h) return U;
    double s, c, ph;
    if (!prop_phase_any(p, ks, &ph)) return make_float2(0.f, 0.f);
    sincos_phase(ph, &s, &c);
    return rot(U, lift_of(make_double2(p.A.x * c - p.A.y * s, p.A.x * s + p.A.y * c)));
}

template <typename Cx> __device__ __forceinline__ Cx one_c();
template <> __device__ __forceinline__ double2 one_c<double2>() { return make_double2(1.0, 0.0); }
template <> __device__ __forceinline__ float2 one_c<float2>() { return make_float2(1.f, 0.f); }

__device__ __forceinline__ double2 cvt(double2 a, double2) { return a; }
__device__ __forceinline__ float2 cvt(double2 a, float2) { return make_float2(float(a.x), float(a.y)); }

// W_N^m from the FP64 four-step tables (lo[m & mask] * hi[m >> shift]).
__device__ __forceinline__ double2 w4(const PassArgs &a, int64_t m) {
    const double2 *lo = static_cast<const double2 *>(a.tw4_lo);
    const double2 *hi = static_cast<const double2 *>(a.tw4_hi);
    const int64_t mask = (int64_t(1) << a.tw4_shift) - 1;
    return cmul(__ldg(lo + (m & mask)), __ldg(hi + (m >> a.tw4_shift)));
}

// digitrev_rt with the digit width as a compile-time constant (3 or 4)
__device__ __forceinline__ int64_t digitrev_w(int64_t p, int log_l, int rb) {
    return rb == 3 ? digitrev_rt(p, log_l, 3) : digitrev_rt(p, log_l, 4);
}

// ceil(x / 2^log_n1) clamped to [0, l]: the first row frequency k2 with
// k1 + k2 * 2^log_n1 >= k1 + x
__device__ __forceinline__ int k2_bound(int64_t x, int log_n1, int l) {
    const int64_t c = -((-x) >> log_n1);
    return c < 0 ? 0 : (c > l ? l : int(c));
}

// Layout of the column kernel's four-step factors (one copy per tile
// parity): per column, the thread-part factors X (2^LX, stride XP) and Y
// (2^LY, stride YP) in FP64, then the E register parts (stride E + 1) as
// 16-byte twiddle entries ({cos, sin} in FP64, or the complex64 lifting
// form). T = threads per column.
template <int T> struct ColTab {
    static constexpr int LOG_T = ilog2(T);
    static constexpr int LX = (LOG_T + 1) / 2, LY = LOG_T - LX;
    static constexpr int XP = (1 << LX) + 2, YP = (1 << LY) + 1;
    template <int C, int E, int CX> static constexpr size_t parity_bytes() {
        return (size_t(C) * (XP + YP) * 16 + size_t(C) * (E + 1) * CX + 15) / 16 * 16;
    }
    // bytes after the block's data and twiddles (16 of them for alignment)
    template <int C, int E, int CX> static constexpr size_t bytes() { return 16 + 2 * parity_bytes<C, E, CX>(); }
};

// ------------------------------------------------------------------ passes
// Persistent kernels: one CTA per SM loops over rows (column tiles); block
// twiddles are copied to shared memory once per CTA, four-step twiddles of a
// row (tile) are factored into 64 + len/64 entries built once per row (tile).
// CHIRP: transfer function in the factored chirp form (two-level plans), else
// the per-sample formula (single-level plans).
// Complex64 rows of 2^13 (512 threads) run two CTAs per SM at 64 registers:
// 8 % faster than one CTA at 121 registers.
template <typename Real, int LOG_L2, int E> constexpr int row_min_ctas() {
    return sizeof(Real) == 4 && LOG_L2 == 13 && E == 16 ? 2 : 1;
}
// TWF: the three-level variant with the W_{N2} twiddle before the forward
// transform (a separate kernel, so that the two-level one carries no code for it).
// BATCH: the batched variant (per-instance transfer functions, a.bpr; chirp
// form only), also a separate kernel so that the others carry no code for it.
template <typename Real, int LOG_L2, int E, bool CHIRP, bool TWF = false, bool BATCH = false>
__global__ void __launch_bounds__(Block<Real, LOG_L2, 1, E>::NT, row_min_ctas<Real, LOG_L2, E>()) row_pass_kernel(PassArgs a) {
    using B = Block<Real, LOG_L2, 1, E>;
    using Cx = typename B::Cx;
    constexpr int L = B::L;
    constexpr int NV = 64 + (L >> 6 > 0 ? L >> 6 : 1);
    using Tw = typename B::Tw;
    using Lf = typename LiftT<Real>::T;
    extern __shared__ __align__(16) unsigned char smraw[];
    Cx *sm = reinterpret_cast<Cx *>(smraw);
    Tw *tw = reinterpret_cast<Tw *>(smraw + B::DATA);
    Lf *const tabs = reinterpret_cast<Lf *>(smraw + (B::SMEM + 15) / 16 * 16);
    constexpr int NQ = (L >> 6) > 1 ? (L >> 6) : 2;  // k2s >> 6 spans [-NQ/2, NQ/2)
    constexpr int NCH = 64 + NQ + E;  // chirp factors per row: P, Q and the per-register R
    const int tp = threadIdx.x;
    const int flags = a.flags;
    const int64_t rows = a.n >> LOG_L2;
    B::load_twiddles(tw, static_cast<const Tw *>(a.tw_row));
    __syncthreads();
    const int64_t nmask = (int64_t(1) << a.tw_log) - 1;
    const double tw_scale = a.tw_scale;
    const int log_m = a.log_n1 + a.log_nb;  // spectrum index k = kbase + 2^log_m * k2
    // A forward + inverse row starts and ends with the stage-0 positions of
    // each thread, so the next row may overwrite the data buffer without a
    // barrier; every other flow ends its row with one.
    const bool paired = (flags & PF_FWD) && (flags & PF_INV) && !(flags & PF_SPEC_IN);

    const int fbase = B::freq_base(tp);  // per-thread part of the spectrum indices

    int parity = 0;
    for (int64_t row = blockIdx.x; row < rows; row += gridDim.x, parity ^= 1) {
        // per-row tables, double-buffered by row parity: the next row fills
        // the other copy while slower warps still read this one
        // 16-byte entries; complex64 keeps the lifting form {a, b, s, 0} of
        // each factor, except P and Q, kept in FP64 (their product is taken once
        // per row and thread before it is turned into a rotation)
        Lf *vec = tabs + parity * (NV + NCH);  // four-step factors: [0,64) low, [64, NV) high
        // chirp factors: [0,64) P[a], [64, 64+NQ) Q[b + NQ/2], [64+NQ, NCH) R[r]
        Lf *chp = vec + NV;
        // row -> (p1, pb): spectrum index base kbase = k1 + N1 kb; the
        // conjugate four-step twiddle of the innermost split uses tw_k
        // (rows beyond one transform belong to the next one of a batch)
        const int64_t k1 = digitrev_w((row >> a.log_nb) & ((int64_t(1) << a.log_n1) - 1), a.log_n1, a.rb_n1);
        const int64_t kb = digitrev_w(row & ((int64_t(1) << a.log_nb) - 1), a.log_nb, a.rb_nb);
        const int64_t kbase = k1 + (kb << a.log_n1);
        const int64_t tw_k = a.log_nb > 0 ? kb : k1;
        if (CHIRP && a.pr.has_h) {
            // phase of the row: G kbase^2 + g1 k2s with g1 = 2 M G kbase (turns),
            // M = 2^log_m; P[a] = A exp(2 pi i (G kbase^2 + g1 a)), Q[b] = exp(2 pi i 64 g1 b).
            // k2s = fbase + s_r splits into the thread's part (P[fbase & 63] Q[fbase >> 6],
            // taken once per row) and the register's part R[r] = exp(2 pi i g1 s_r),
            // s_r = freq_off(r) - L if the top frequency bit is set (all lanes read
            // the same R[r])
            // (a batched pass takes G and A of the row's instance)
            double g_hi = a.pr.g_hi, g_lo = a.pr.g_lo;
            double2 A = a.pr.A;
            if constexpr (BATCH) {
                const BatchProp *bp = a.bpr + (row >> log_m);
                g_hi = __ldg(&bp->g_hi);
                g_lo = __ldg(&bp->g_lo);
                A = __ldg(&bp->A);
            }
            const double m = double(int64_t(1) << log_m);
            const double gk = frac_dd(g_hi, g_lo, double(kbase * kbase));
            const double g1h = 2.0 * m * g_hi, g1l = 2.0 * m * g_lo;
            for (int idx = tp; idx < NCH; idx += B::NT) {
                double2 w;
                if (idx < 64) {
                    w = cmul(A, cis_turns(gk + frac_dd(g1h, g1l, double(kbase * idx))));
                } else if (idx < 64 + NQ) {
                    const int64_t b = int64_t(idx - 64) - NQ / 2;
                    w = cis_turns(frac_dd(g1h, g1l, double(kbase * 64 * b)));
                } else {
                    const int fo = B::freq_off(idx - 64 - NQ);
                    const int64_t sr = (fo & (L >> 1)) ? int64_t(fo) - L : int64_t(fo);
                    w = cis_turns(frac_dd(g1h, g1l, double(kbase * sr)));
                }
                if constexpr (B::LIFT) {
                    if (idx < 64 + NQ) reinterpret_cast<double2 *>(chp)[idx] = w;
                    else chp[idx] = lift_of(w);
                } else {
                    chp[idx] = w;
                }
            }
        }
        if (flags & (PF_TW | PF_TWF)) {
            // conj(W_M^{n2 tw_k}) * tw_scale = conj(A[n2 & 63]) * conj(B[n2 >> 6]) * tw_scale
            for (int idx = tp; idx < NV; idx += B::NT) {
                const int64_t m = ((idx < 64 ? int64_t(idx) : int64_t(idx - 64) << 6) * tw_k) & nmask;
                double2 w = w4(a, m);
                w = make_double2(w.x, -w.y);
                if constexpr (B::LIFT) {
                    vec[idx] = lift_of(w, idx >= 64 ? tw_scale : 1.0);
                } else {
                    if (idx >= 64) w = make_double2(w.x * tw_scale, w.y * tw_scale);
                    vec[idx] = w;
                }
            }
        }
        if constexpr (B::NS == 1) __syncthreads();  // no barrier inside a one-stage transform
        const Cx *__restrict__ gin = static_cast<const Cx *>(a.in) + (row << LOG_L2);
        Cx *__restrict__ gout = static_cast<Cx *>(a.out) + (row << LOG_L2);
        // this CTA's next row into L2 while this one is transformed, issued
        // after this row's own loads
        const auto prefetch_next = [&] {
            constexpr uint32_t chunk = uint32_t(L * sizeof(Cx) / 32);
            if constexpr (chunk >= 16 && chunk % 16 == 0) {
                if (!(flags & PF_ONES) && row + gridDim.x < rows && tp < 32)
                    prefetch_l2_bulk(reinterpret_cast<const unsigned char *>(gin + (int64_t(gridDim.x) << LOG_L2)) +
                                         tp * chunk,
                                     chunk);
            }
        };
        Cx v[E];
        if (!(flags & PF_SPEC_IN)) {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = (flags & PF_ONES) ? one_c<Cx>() : gin[B::first_pos(tp, r)];
            prefetch_next();
            if (TWF && (flags & PF_TWF)) {
                __syncthreads();  // this row's factor table is complete
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int n2 = B::first_pos(tp, r);
                    if constexpr (B::LIFT) {  // the exact inverse of the PF_TW rotations below
                        const Lf lo = vec[n2 & 63], hi = vec[64 + (n2 >> 6)];
                        v[r] = lift(lift(cscale(v[r], lo.z * hi.z), -hi.x, -hi.y), -lo.x, -lo.y);
                    } else {
                        v[r] = cmulc(cmulc(v[r], vec[n2 & 63]), vec[64 + (n2 >> 6)]);
                    }
                }
            }
            // Rows of multi-level plans never transmit (the column pass does).
            // Leaving the code out of the complex64 kernel frees registers
            // (5 % faster); the complex128 one ran 2 % slower without it.
            if constexpr (!(CHIRP && sizeof(Real) == 4)) {
                if (flags & PF_TRANS) {
#pragma unroll
                    for (int r = 0; r < E; ++r)
                        v[r] = apply_trans(a.tr, (row << LOG_L2) + B::first_pos(tp, r), v[r]);
                }
            }
            if (flags & PF_FWD) B::forward(sm, tp, v, tw);
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = gin[B::last_pos(tp, r)];
            prefetch_next();
        }

        if constexpr (CHIRP) {
          if (a.pr.has_h || a.pr.has_cut) {
            // cutoff: k = kbase + k2 2^log_m in [cut_lo, cut_hi)  <=>  k2 in [k2lo, k2hi)
            int k2lo = 0, k2hi = 0;
            if (a.pr.has_cut) {
                if constexpr (BATCH) {
                    const BatchProp *bp = a.bpr + (row >> log_m);
                    k2lo = k2_bound(__ldg(&bp->cut_lo) - kbase, log_m, L);
                    k2hi = k2_bound(__ldg(&bp->cut_hi) - kbase, log_m, L);
                } else {
                    k2lo = k2_bound(a.pr.cut_lo - kbase, log_m, L);
                    k2hi = k2_bound(a.pr.cut_hi - kbase, log_m, L);
                }
            }
            const unsigned cut_span = unsigned(k2hi - k2lo);
            if (a.pr.has_h) {
                // H = P[fbase & 63] * Q[fbase >> 6] * R[r] * h3[r][tp]; k2 >= L/2
                // (k2s = k2 - L) is decided by the compile-time part of the
                // frequency, so 0 <= fbase < L/2
                const Lf *h3 = static_cast<const Lf *>(BATCH ? a.bpr[row >> log_m].h3 : a.pr.h3);
                // rows without cut frequencies (cut_span 0, uniform per row)
                // take the loop without the per-sample test
                const auto zero_cut = [&](int r, Cx x) {
                    return unsigned((fbase | B::freq_off(r)) - k2lo) < cut_span ? Cx{} : x;
                };
                if constexpr (B::LIFT) {
                    // three rotations: the thread's P Q (FP64 product), R[r], h3
                    const double2 *chd = reinterpret_cast<const double2 *>(chp);
                    const Lf tl = lift_of(cmul(chd[fbase & 63], chd[64 + (fbase >> 6) + NQ / 2]));
                    const auto rotate = [&](auto cut) {
#pragma unroll
                        for (int r = 0; r < E; ++r) {
                            const Lf rr = chp[64 + NQ + r], g = __ldg(h3 + r * B::T + tp);
                            Cx x = cscale(v[r], tl.z * rr.z * g.z);
                            x = lift(lift(lift(x, tl.x, tl.y), rr.x, rr.y), g.x, g.y);
                            v[r] = decltype(cut)::value ? zero_cut(r, x) : x;
                            if (r % 4 == 3) asm volatile("" ::: "memory");
                        }
                    };
                    if (cut_span == 0) rotate(std::false_type{});
                    else rotate(std::true_type{});
                } else {
                const Cx tb = cmul(chp[fbase & 63], chp[64 + (fbase >> 6) + NQ / 2]);
                const auto multiply = [&](auto cut) {
#pragma unroll
                    for (int r = 0; r < E; ++r) {
                        const Cx h = cmul(cmul(tb, chp[64 + NQ + r]), __ldg(h3 + r * B::T + tp));
                        v[r] = decltype(cut)::value ? zero_cut(r, cmul(v[r], h)) : cmul(v[r], h);
                        // a compiler-only barrier per 4 samples: without it all E
                        // h3 loads were issued ahead and held live (the 2^14
                        // complex64 row spilled 132 bytes per thread instead of 52,
                        // 5 % slower)
                        if (r % 4 == 3) asm volatile("" ::: "memory");
                    }
                };
                if (cut_span == 0) multiply(std::false_type{});
                else multiply(std::true_type{});
                }
            } else {
#pragma unroll
                for (int r = 0; r < E; ++r)
                    if (unsigned((fbase | B::freq_off(r)) - k2lo) < cut_span) v[r] = Cx{};
            }
          }
        } else if (a.pr.has_h || a.pr.has_cut) {
            const int64_t half2 = int64_t(1) << (LOG_L2 - 1);
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int64_t k2 = B::last_freq(tp, r);
                const int64_t k = kbase + (k2 << log_m);
                const int64_t k2s = k2 >= half2 ? k2 - 2 * half2 : k2;
                const int64_t ks = kbase + k2s * (int64_t(1) << log_m);
                v[r] = prop_apply(a.pr, k, ks, v[r]);
            }
        }

        if (flags & PF_INV) {
            B::inverse(sm, tp, v, tw);
            if (flags & PF_TW) {
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int n2 = B::first_pos(tp, r);
                    if constexpr (B::LIFT) {
                        const Lf lo = vec[n2 & 63], hi = vec[64 + (n2 >> 6)];
                        v[r] = lift(lift(cscale(v[r], lo.z * hi.z), lo.x, lo.y), hi.x, hi.y);
                    } else {
                        v[r] = cmul(cmul(v[r], vec[n2 & 63]), vec[64 + (n2 >> 6)]);
                    }
                }
            } else if (flags & PF_SCALE) {
                const Real f = Real(a.pr.fac);
#pragma unroll
                for (int r = 0; r < E; ++r) v[r] = cscale(v[r], f);
            }
#pragma unroll
            for (int r = 0; r < E; ++r) gout[B::first_pos(tp, r)] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < E; ++r) gout[B::last_pos(tp, r)] = v[r];
        }
        if (!paired) __syncthreads();
    }
}

// ------------------------------------------------------- fused detection
// Pixel of sample n in [d.lo, d.hi): the linear guess is off by at most a
// sample or two for np.histogram bins on a uniform grid; bounded steps, then
// a bisection if they did not bracket it.
__device__ __forceinline__ int64_t pixel_of(const DetectArgs &d, int64_t n) {
    int64_t j = int64_t(double(n - d.lo) * d.inv_w);
    j = j < 0 ? 0 : (j >= d.n_pix ? d.n_pix - 1 : j);
    for (int it = 0; it < 4 && n < __ldg(d.bounds + j); ++it) --j;
    for (int it = 0; it < 4 && n >= __ldg(d.bounds + j + 1); ++it) ++j;
    if (n < __ldg(d.bounds + j) || n >= __ldg(d.bounds + j + 1)) {
        int64_t a = 0, b = d.n_pix - 1;  // last j with bounds[j] <= n
        while (a < b) {
            const int64_t m = (a + b + 1) / 2;
            if (__ldg(d.bounds + m) <= n) a = m; else b = m - 1;
        }
        j = a;
    }
    return j;
}

// |u|^2 of a thread's samples (column col, rows first_pos(tp, r)) into
// d.sum by pixel. The C lanes of one tp hold adjacent columns of the same
// rows; a group of G = min(C, 32) lanes whose samples share a pixel adds its
// group sum with one atomic, otherwise each lane adds its own.
template <typename B, typename Cx>
__device__ __forceinline__ void detect_bin(const DetectArgs &d, double *sum, int64_t col, int tp, const Cx *v,
                                           int log_n2) {
    constexpr int C = B::NT / B::T, G = C < 32 ? C : 32;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (lane & ~unsigned(G - 1));
#pragma unroll
    for (int r = 0; r < B::E; ++r) {
        const int64_t n = (int64_t(B::first_pos(tp, r)) << log_n2) + col;
        const bool in = n >= d.lo && n < d.hi;
        if (!__any_sync(0xffffffffu, in)) continue;
        int64_t j = -1;
        double s = 0.0;
        if (in) {
            j = pixel_of(d, n);
            const double re = double(v[r].x), im = double(v[r].y);
            s = re * re + im * im;
        }
        const int64_t lead = __shfl_sync(0xffffffffu, j, 0, G);
        const bool uniform = (__ballot_sync(0xffffffffu, j == lead) & gmask) == gmask;
        double g = s;
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o, G);
        if (uniform) {
            if ((lane & unsigned(G - 1)) == 0 && lead >= 0) atomicAdd(sum + lead, g);
        } else if (j >= 0) {
            atomicAdd(sum + j, s);
        }
    }
}

// End of a detection pass: the CTA that finishes last turns the sums into
// the pixel values of square_and_downsample, (((sum cos_j) dx) psy) / r_j,
// adds weight * value into the accumulator with Kahan compensation, and
// zeroes the sums and the count for the next pass. A batched pass adds its
// instances one after the other, in instance order: the order in which
// separate runs of the same sources would add them. With inst_out it also
// keeps each instance's own pixel values.
__device__ __forceinline__ void detect_finish(const DetectArgs &d) {
    __shared__ int last;
    __threadfence();  // this thread's atomics before the count
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(d.count, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int64_t j = threadIdx.x; j < d.n_pix; j += blockDim.x) {
        const double cj = __ldg(d.cosv + j), rj = __ldg(d.rv + j);
        double acc = d.acc[j], comp = d.comp[j];
        for (int b = 0; b < d.n_inst; ++b) {
            double *sum = d.sum + b * d.sum_stride + j;
            const double s = __ldcg(sum);
            const double val = (((s * cj) * d.dx) * d.psy) / rj;
            if (d.inst_out) d.inst_out[b * d.inst_stride + j] = val;
            const double w = d.bweight ? __ldg(d.bweight + b) : d.weight;
            const double y = __dsub_rn(__dmul_rn(w, val), comp);
            const double t = __dadd_rn(acc, y);
            comp = __dsub_rn(__dsub_rn(t, acc), y);
            acc = t;
            *sum = 0.0;
        }
        d.acc[j] = acc;
        d.comp[j] = comp;
    }
    if (threadIdx.x == 0) *d.count = 0u;
}

// DET: the detection variant, for the inverse-only pass that ends a phase
// step: each CTA takes a contiguous range of tiles (adjacent columns), bins
// |u|^2 after the inverse transform (detect_bin) and stores the field unless
// PF_NOSTORE; the last CTA finishes the detector row (detect_finish).
// BATCH: per-instance transmission factors (a.btr), a separate kernel. Its
// factors live in registers where the plain kernel reads them from the
// parameter bank, so some complex128 shapes hold fewer CTAs per SM
// (col_resident; the host then runs such sources one after the other).
template <typename Real, int LOG_L1, int C, int E, bool DET, bool BATCH>
__device__ __forceinline__ void col_pass(const PassArgs &a) {
    using B = Block<Real, LOG_L1, C, E>;
    using Cx = typename B::Cx;
    // Four-step factor W_M^(n2 k1) of column n2 = col0 + c at the frequency
    // k1 = freq_base(tp) | freq_off(r) held by register r: the thread's part
    // W^(n2 freq_base(tp)) times the register's part W^(n2 freq_off(r)) (E
    // per column, read by every lane of the column). freq_base is a bit
    // permutation, so the thread part is X[tp & (2^LX - 1)] * Y[tp >> LX] with
    // X[i] = W^(n2 freq_base(i)), Y[j] = W^(n2 freq_base(j 2^LX)), multiplied
    // in FP64. The strides put the C columns of a wavefront in different banks.
    // complex64 applies both parts as rotations by lifting (register parts
    // stored in the lifting form).
    using Tw = typename B::Tw;
    using Lf = typename LiftT<Real>::T;
    using CT = ColTab<B::T>;
    constexpr int LX = CT::LX, NX = 1 << LX, NXY = NX + (1 << CT::LY);
    constexpr int XP = CT::XP, YP = CT::YP, EP = E + 1;
    constexpr size_t PAR = CT::template parity_bytes<C, E, int(sizeof(Lf))>();
    extern __shared__ __align__(16) unsigned char smraw[];
    const int t = threadIdx.x;
    const int c = t % C;
    const int tp = t / C;
    Cx *sm = reinterpret_cast<Cx *>(smraw) + c * B::PITCH;
    Tw *tw = reinterpret_cast<Tw *>(smraw + B::DATA);
    const int log_n2 = a.log_n2;
    const int flags = a.flags;
    const int log_tb = log_n2 - ilog2(C);  // tiles per batch: 2^log_tb
    const int64_t tiles = (a.n >> LOG_L1) / C;
    const int64_t nmask = (int64_t(1) << a.tw_log) - 1;
    B::load_twiddles(tw, static_cast<const Tw *>(a.tw_col));
    __syncthreads();
    // An inverse + forward tile starts and ends with the last-stage positions
    // of each thread, so the next tile may overwrite the data buffer without
    // a barrier; every other flow ends its tile with one.
    const bool paired = (flags & PF_FWD) && (flags & PF_INV);

    unsigned char *tab0 = smraw + (B::SMEM + 15) / 16 * 16;

    int64_t t_first = blockIdx.x, t_end = tiles, t_step = gridDim.x;
    if constexpr (DET) {
        const int64_t per = (tiles + gridDim.x - 1) / gridDim.x;
        t_first = int64_t(blockIdx.x) * per;
        t_end = t_first + per < tiles ? t_first + per : tiles;
        t_step = 1;
    }
    // this CTA's next tile into L2 through the input's TMA map, one box of the
    // tile's C columns by up to 256 rows per thread of the first few, issued
    // right after the current tile's own loads (2^24 complex64 columns of
    // 2^11: 124 -> 112 us per launch alone; issued before the loads it gains
    // nothing)
    constexpr int PF_BOX = B::L < 256 ? B::L : 256;
    const auto prefetch_next = [&](int64_t tile) {
        if (!a.in_map_ok || tile + t_step >= t_end || t >= B::L / PF_BOX) return;
        const int64_t nt = tile + t_step;
        const int x = int((nt & ((int64_t(1) << log_tb) - 1)) * C) * int(sizeof(Cx) / 8);
        prefetch_l2_tile(&a.in_map, x, int(((nt >> log_tb) << LOG_L1) + int64_t(t) * PF_BOX));
    };
    int parity = 0;
    for (int64_t tile = t_first; tile < t_end; tile += t_step, parity ^= 1) {
        // factor tables, double-buffered by tile parity
        double2 *tx = reinterpret_cast<double2 *>(tab0 + parity * PAR);
        double2 *ty = tx + C * XP;
        Lf *vec = reinterpret_cast<Lf *>(ty + C * YP);
        const int64_t batch = tile >> log_tb;
        const int64_t col0 = (tile & ((int64_t(1) << log_tb) - 1)) * C;  // column within the batch
        const int64_t col = col0 + c;
        const int64_t base = batch << (LOG_L1 + log_n2);
        if (flags & (PF_TW | PF_TWI)) {
            for (int idx = t; idx < C * (NXY + E); idx += B::NT) {
                const int cc = idx / (NXY + E), e = idx % (NXY + E);
                const int64_t n2 = col0 + cc;
                if (e < NX)
                    tx[cc * XP + e] = w4(a, (int64_t(B::freq_base(e)) * n2) & nmask);
                else if (e < NXY)
                    ty[cc * YP + (e - NX)] = w4(a, (int64_t(B::freq_base((e - NX) << LX)) * n2) & nmask);
                else if constexpr (B::LIFT)
                    vec[cc * EP + (e - NXY)] = lift_of(w4(a, (int64_t(B::freq_off(e - NXY)) * n2) & nmask));
                else
                    vec[cc * EP + (e - NXY)] = w4(a, (int64_t(B::freq_off(e - NXY)) * n2) & nmask);
            }
        }
        if constexpr (B::NS == 1) __syncthreads();  // no barrier inside a one-stage transform
        const Cx *__restrict__ gin = static_cast<const Cx *>(a.in) + base + col;
        Cx *__restrict__ gout = static_cast<Cx *>(a.out) + base + col;
        Cx v[E];
        if (flags & PF_INV) {
#pragma unroll
            for (int r = 0; r < E; ++r) v[r] = gin[int64_t(B::last_pos(tp, r)) << log_n2];
            prefetch_next(tile);
            if (flags & PF_TWI) {
                __syncthreads();  // this tile's factor table is complete
                const Lf *vc = vec + c * EP;
                const double2 w64 = cmul(tx[c * XP + (tp & (NX - 1))], ty[c * YP + (tp >> LX)]);
                const Real s = Real(a.tw_scale);  // a power of two: exact
                if constexpr (B::LIFT) {
                    // the exact inverse of the PF_TW rotations (register part first)
                    const Lf wt = lift_of(w64);
#pragma unroll
                    for (int r = 0; r < E; ++r)
                        v[r] = lift(lift(cscale(v[r], wt.z * vc[r].z * s), -vc[r].x, -vc[r].y), -wt.x, -wt.y);
                } else {
                    const Cx w = cvt(w64, Cx{});
#pragma unroll
                    for (int r = 0; r < E; ++r) v[r] = cscale(cmulc(v[r], cmul(w, vc[r])), s);
                }
            }
            B::inverse(sm, tp, v, tw);
        } else if constexpr (!DET) {
#pragma unroll
            for (int r = 0; r < E; ++r)
                v[r] = (flags & PF_ONES) ? one_c<Cx>() : gin[int64_t(B::first_pos(tp, r)) << log_n2];
            prefetch_next(tile);
        }
        // the detection variant runs the inverse only: no transmission, no forward
        // (single-transform passes transmit at base 0; a batched pass at the
        // position within the tile's own transform)
        if (!DET && (flags & PF_TRANS)) {
            if constexpr (BATCH)
                apply_trans_batch<E>(a.tr, a.btr + batch,
                                     [&](int r) { return (int64_t(B::first_pos(tp, r)) << log_n2) + col; }, v);
            else
                apply_trans_e<E>(a.tr, [&](int r) { return base + (int64_t(B::first_pos(tp, r)) << log_n2) + col; }, v);
        }
        if (!DET && (flags & PF_FWD)) {
            B::forward(sm, tp, v, tw);
            if (flags & PF_TW) {
                const Lf *vc = vec + c * EP;
                const double2 w64 = cmul(tx[c * XP + (tp & (NX - 1))], ty[c * YP + (tp >> LX)]);
                if constexpr (B::LIFT) {
                    const Lf wt = lift_of(w64);
#pragma unroll
                    for (int r = 0; r < E; ++r)
                        v[r] = lift(lift(cscale(v[r], wt.z * vc[r].z), wt.x, wt.y), vc[r].x, vc[r].y);
                } else {
                    const Cx w = cvt(w64, Cx{});
#pragma unroll
                    for (int r = 0; r < E; ++r) v[r] = cmul(v[r], cmul(w, vc[r]));
                }
            }
#pragma unroll
            for (int r = 0; r < E; ++r) gout[int64_t(B::last_pos(tp, r)) << log_n2] = v[r];
        } else {
            if constexpr (DET) detect_bin<B>(a.det, a.det.sum + batch * a.det.sum_stride, col, tp, v, log_n2);
            if (!DET || !(flags & PF_NOSTORE)) {
#pragma unroll
                for (int r = 0; r < E; ++r) gout[int64_t(B::first_pos(tp, r)) << log_n2] = v[r];
            }
        }
        if (!paired) __syncthreads();
    }
    if constexpr (DET) detect_finish(a.det);
}

// The column kernel. Single-source complex128 tiles of 256 threads take a
// kernel held to two CTAs per SM: ptxas's default gave the 2^7 outer columns
// of 2^26 three-level plans 168 registers and one CTA per SM (1028 us per
// launch), two CTAs at 128 registers and a few spills run 774 us. (Their
// batched variants keep the default; rsw_sim_run_batch then runs such
// sources one by one.)
template <typename Real, int LOG_L1, int C, int E, bool DET = false, bool BATCH = false>
__global__ void __launch_bounds__(Block<Real, LOG_L1, C, E>::NT) col_pass_kernel(const __grid_constant__ PassArgs a) {
    col_pass<Real, LOG_L1, C, E, DET, BATCH>(a);
}
template <typename Real, int LOG_L1, int C, int E> constexpr bool col_two_ctas() {
    return sizeof(Real) == 8 && Block<Real, LOG_L1, C, E>::NT == 256;
}
template <typename Real, int LOG_L1, int C, int E, bool DET = false, bool BATCH = false>
__global__ void __launch_bounds__(Block<Real, LOG_L1, C, E>::NT, 2)
    col_pass_kernel_2cta(const __grid_constant__ PassArgs a) {
    col_pass<Real, LOG_L1, C, E, DET, BATCH>(a);
}

// exp(2 pi i G N1^2 k2s^2) for every register (r, tp) of the row kernel
// Block<Real, LOG_L2, 1, E>, stored at r * T + tp ({cos, sin} for complex128,
// the lifting form for complex64).
template <typename Real, int LOG_L2, int E>
__global__ void chirp_table_kernel(typename LiftT<Real>::T *__restrict__ out, double g3_hi, double g3_lo) {
    using B = Block<Real, LOG_L2, 1, E>;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B::L) return;
    const int r = idx / B::T, tp = idx % B::T;
    const int half2 = 1 << (LOG_L2 - 1);
    const int k2 = B::last_freq(tp, r);
    const double k2s = double(k2 >= half2 ? k2 - 2 * half2 : k2);
    const double2 w = cis_turns(frac_dd(g3_hi, g3_lo, k2s * k2s));
    if constexpr (sizeof(Real) == 4) out[idx] = lift_of(w);
    else out[idx] = w;
}

void count_launch();

template <typename K> static cudaError_t prep(K kernel, size_t smem) {
    if (smem > 48 * 1024) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    return cudaSuccess;
}

// persistent grid: as many CTAs as fit on the device at once, capped by the work
template <typename K> static int64_t resident_ctas(K kernel, int threads, size_t smem, int dev) {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    return int64_t(sms > 0 ? sms : 1) * (per_sm > 0 ? per_sm : 1);
}

// Launch set-up of one kernel, per device: the dynamic shared-memory limit is
// a per-device attribute of the kernel and the resident CTA count depends on
// the device, so both are taken once for each device the kernel launches on
// (the device current at the launch). cap[1] is the CTA count at the
// second shared-memory size (the column kernel without its factor tables).
constexpr int LAUNCH_MAX_DEVICES = 64;
struct LaunchSetup {
    cudaError_t attr = cudaSuccess;
    int64_t cap[2] = {1, 1};
};
template <typename K>
static const LaunchSetup *launch_setup(K kernel, int threads, size_t smem, size_t smem2, LaunchSetup *table,
                                       std::once_flag *once) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= LAUNCH_MAX_DEVICES) return nullptr;
    std::call_once(once[dev], [&] {
        LaunchSetup &st = table[dev];
        st.attr = prep(kernel, smem > smem2 ? smem : smem2);
        if (st.attr == cudaSuccess) {
            st.cap[0] = resident_ctas(kernel, threads, smem, dev);
            st.cap[1] = resident_ctas(kernel, threads, smem2, dev);
        }
    });
    return &table[dev];
}

template <int L> constexpr int n_vec() { return 64 + ((L >> 6) > 0 ? (L >> 6) : 1); }
template <int L, int E> constexpr int n_chirp() { return 64 + ((L >> 6) > 1 ? (L >> 6) : 2) + E; }

template <typename Real, int LG, int E, bool CH, bool TWF, bool BT>
static cudaError_t row_launch(const PassArgs &a, cudaStream_t s) {
    using B = Block<Real, LG, 1, E>;
    auto k = row_pass_kernel<Real, LG, E, CH, TWF, BT>;
    const size_t smem = (B::SMEM + 15) / 16 * 16 + 2 * size_t(n_vec<B::L>() + n_chirp<B::L, E>()) * 16;
    static LaunchSetup setup[LAUNCH_MAX_DEVICES];
    static std::once_flag once[LAUNCH_MAX_DEVICES];
    const LaunchSetup *st = launch_setup(k, B::NT, smem, smem, setup, once);
    if (!st) return cudaErrorInvalidDevice;
    if (st->attr != cudaSuccess) return st->attr;
    const int64_t cap = st->cap[0];
    const int64_t rows = a.n >> LG;
    k<<<dim3(unsigned(rows < cap ? rows : cap)), dim3(B::NT), smem, s>>>(a);
    count_launch();
    return cudaGetLastError();
}
// PF_TWF (rows of three-level plans) takes the TWF variant, for the chirp
// form and for the per-sample transfer function (exact kernel) alike; rows of
// multi-level plans hold at least 2^7 samples
// BT: the batched variant, chirp form only
template <typename Real, int LG, int E, bool CH, bool BT = false>
static cudaError_t row_impl(const PassArgs &a, cudaStream_t s) {
    if constexpr (BT && !CH) {
        return cudaErrorInvalidValue;
    } else {
        if constexpr (LG >= 7) {
            if (a.flags & PF_TWF) return row_launch<Real, LG, E, CH, true, BT>(a, s);
        }
        if (a.flags & PF_TWF) return cudaErrorInvalidValue;
        return row_launch<Real, LG, E, CH, false, BT>(a, s);
    }
}

// Columns per CTA of the column kernel (16 samples per thread): enough for
// 256-thread CTAs and 512-byte row segments on short columns, 4 (64-byte
// segments) from 2^10 up; capped so that the factor tables still fit.
constexpr int col_c(int log_l) {
    return log_l <= 5 ? 64 : log_l <= 7 ? 32 : log_l == 8 ? 16 : log_l == 9 ? 8 : 4;
}
// complex64 columns of 2^10 and 2^11: 16 and 8 (128- and 64-byte row
// segments, measured 26 % and 13 % faster than 32-byte ones at 2^28 and 2^24)
constexpr int col_c64(int log_l) { return log_l == 10 ? 16 : log_l == 11 ? 8 : col_c(log_l); }

// The input's TMA map for the column kernel's next-tile prefetch: rows of
// 2^log_n2 samples of words_per_sample 8-byte words, boxes of box_w words by
// box_h rows. False (no prefetch) when the input is not 16-byte aligned or
// the map cannot be encoded.
bool encode_col_map(CUtensorMap *map, const void *in, int64_t n, int log_n2, int words_per_sample, int box_w,
                    int box_h);

template <typename Real, int LG, int C, int E, bool DET = false, bool BT = false>
static cudaError_t col_impl(const PassArgs &a, cudaStream_t s) {
    using B = Block<Real, LG, C, E>;
    auto k = [] {
        if constexpr (col_two_ctas<Real, LG, C, E>() && !BT) return col_pass_kernel_2cta<Real, LG, C, E, DET, BT>;
        else return col_pass_kernel<Real, LG, C, E, DET, BT>;
    }();
    // the per-column factor tables only when the pass applies a four-step twiddle
    const size_t plain = B::SMEM;
    const size_t tab = (B::SMEM + 15) / 16 * 16 + ColTab<B::T>::template bytes<C, E, 16>();
    static LaunchSetup setup[LAUNCH_MAX_DEVICES];
    static std::once_flag once[LAUNCH_MAX_DEVICES];
    const LaunchSetup *st = launch_setup(k, B::NT, tab, plain, setup, once);
    if (!st) return cudaErrorInvalidDevice;
    if (st->attr != cudaSuccess) return st->attr;
    const bool tables = a.flags & (PF_TW | PF_TWI);
    const int64_t cap = tables ? st->cap[0] : st->cap[1];
    if (a.resident) {  // a query: the resident CTAs per device, no launch
        *a.resident = cap;
        return cudaSuccess;
    }
    const int64_t tiles = (a.n >> LG) / C;
    if ((int64_t(1) << a.log_n2) < C) return cudaErrorInvalidValue;  // fewer columns per batch than a tile
    int64_t grid = tiles < cap ? tiles : cap;
    if constexpr (DET) {  // contiguous tile ranges: no CTA without tiles
        const int64_t per = (tiles + grid - 1) / grid;
        grid = (tiles + per - 1) / per;
    }
    PassArgs b = a;
    constexpr int words = int(sizeof(typename B::Cx) / 8);
    b.in_map_ok = a.in && !(a.flags & PF_ONES) && tiles > grid &&
                  encode_col_map(&b.in_map, a.in, a.n, a.log_n2, words, C * words, B::L < 256 ? B::L : 256);
    k<<<dim3(unsigned(grid)), dim3(B::NT), tables ? tab : plain, s>>>(b);
    count_launch();
    return cudaGetLastError();
}

template <typename Real, int LG, int E> static cudaError_t chirp_impl(void *out, double hi, double lo, cudaStream_t s) {
    chirp_table_kernel<Real, LG, E><<<((1 << LG) + 255) / 256, 256, 0, s>>>(
        static_cast<typename LiftT<Real>::T *>(out), hi, lo);
    count_launch();
    return cudaGetLastError();
}
}  // namespace rsw
