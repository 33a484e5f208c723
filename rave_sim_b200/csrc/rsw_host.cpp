// Host side of the rsw engine: FFT plans, the numpy-exact host arithmetic of
// the reference's discrete decisions, the per-source schedule of
// big-wave/wavesim.py:84-298 on the fused two-pass engine, and the C ABI
// declared in include/rsw.h.
//
// Compiled with -ffp-contract=off: every scalar below is evaluated with the
// reference's operation order and one rounding per operation.
#include "rsw.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "rsw_internal.h"
#include "rsw_stages.h"

namespace rsw {
cudaError_t launch_row_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s);
cudaError_t launch_col_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s);
cudaError_t launch_col_detect(const PassArgs &a, bool dbl, int e, cudaStream_t s);
cudaError_t launch_spec_to_natural(const void *in, void *out, int64_t n, const SpecLevels &v, bool dbl,
                                   cudaStream_t s);
cudaError_t launch_natural_to_spec(const void *in, void *out, int64_t n, const SpecLevels &v, bool dbl,
                                   cudaStream_t s);
cudaError_t launch_trans(void *u, int64_t n, const TransArgs &tr, bool dbl, cudaStream_t s);
cudaError_t launch_retrieval(const double *data, int64_t n_pix, const RetrievalArgs &r, double *dabs, double *dphase,
                             double *dvis, double *chi2, cudaStream_t s);
cudaError_t launch_copy(const void *in, void *out, int64_t n, bool dbl, cudaStream_t s);
cudaError_t launch_transpose(const void *in, void *out, int64_t rows, int64_t cols, bool dbl, cudaStream_t s);
cudaError_t launch_ooc_twiddle(void *u, int64_t count, int log_len, int64_t row0, int log_n, bool inverse, bool dbl,
                               cudaStream_t s);
cudaError_t launch_point_source(void *u, int64_t n, double dx, double w, double z, double x_src, bool dbl,
                                cudaStream_t s);
cudaError_t launch_detect(const void *u, const int64_t *bounds, const double *cosv, const double *rv,
                          int64_t n_pix, double dx, double psy, double *out, double *acc, double *comp,
                          double weight, bool dbl, cudaStream_t s);
cudaError_t launch_zero(double *p, int64_t n, cudaStream_t s);
cudaError_t launch_fill_ones(void *u, int64_t n, bool dbl, cudaStream_t s);
cudaError_t launch_chirp_table(void *out, int log_n2, double hi, double lo, bool dbl, int e, cudaStream_t s);
cudaError_t launch_blue_pre(const void *in, void *w, int64_t n, int64_t m, const double2 *b, bool conj_in, bool dbl,
                            cudaStream_t s);
cudaError_t launch_blue_mul(void *w, const double2 *bh, int64_t m, bool dbl, cudaStream_t s);
cudaError_t launch_blue_post(const void *w, void *out, int64_t n, const double2 *b, double scale, bool conj_out,
                             bool dbl, cudaStream_t s);
cudaError_t launch_prop_natural(void *U, int64_t n, const PropArgs &p, bool dbl, cudaStream_t s);
unsigned long long launch_count();
}  // namespace rsw

using namespace rsw;
using cplx = std::complex<double>;

// ------------------------------------------------------------------ errors
static thread_local std::string t_last_error;

static rsw_status fail(rsw_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return st;
}

namespace rsw {
rsw_status set_error(rsw_status st, const char *msg) {
    t_last_error = msg;
    return st;
}
}  // namespace rsw

#define CU(call)                                                                               \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(e_ == cudaErrorMemoryAllocation ? RSW_ERR_NOMEM : RSW_ERR_CUDA,        \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define CHECK(expr)                   \
    do {                              \
        rsw_status s_ = (expr);       \
        if (s_ != RSW_OK) return s_;  \
    } while (0)

// -------------------------------------------------- reference host arithmetic
// big-wave/propagation.py:26-28, :69-71. The constants are evaluated the way
// the reference writes them (mantissa * 10 ** exponent, one rounding each):
// 1.602176634 * 10**-19 is one ulp away from the literal 1.602176634e-19, and
// at phases of 1e10 rad one ulp of the wavelength is 1e-6 rad.
static double wavelength(double energy_ev) {
    const double h_planck = 6.62607004 * std::pow(10.0, -34.0);
    const double c_0 = 299792458.0;
    const double ev_to_joule = 1.602176634 * std::pow(10.0, -19.0);
    return h_planck * c_0 / (energy_ev * ev_to_joule);
}

// Python float floor division `a // b` (CPython float_floor_div semantics).
static double py_floordiv(double a, double b) {
    double mod = std::fmod(a, b);
    double div = (a - mod) / b;
    if (mod != 0.0) {
        if ((b < 0) != (mod < 0)) div -= 1.0;
    }
    double fl;
    if (div != 0.0) {
        fl = std::floor(div);
        if (div - fl > 0.5) fl += 1.0;
    } else {
        fl = std::copysign(0.0, a / b);
    }
    return fl;
}

// material_factor(db, t, wl) = np.exp(2j*pi*t/wl * db) (big-wave/optical_element.py:36-39)
static cplx material_factor(double delta, double beta, double t, double wl) {
    const double y = (2.0 * M_PI * t) / wl;
    const double re = -(y * beta);
    const double im = y * delta;
    const double e = std::exp(re);
    return cplx(e * std::cos(im), e * std::sin(im));
}

// Propagator scalars of propagate() (big-wave/propagation.py:74-137).
// exact: the angular-spectrum kernel instead of the Fresnel one (opt-in, no
// counterpart in the reference): phi = 2 pi dz fx^2 / (1/wl + sqrt(1/wl^2 - fx^2))
// beyond the same constant -2 pi dz / wl.
static PropArgs make_prop(int64_t n, double dx, double wl, double dz, double cutoff_freq, bool apply_h,
                          bool exact = false) {
    PropArgs p{};
    p.has_h = apply_h ? 1 : 0;
    p.exact = exact ? 1 : 0;
    p.inv_wl = 1.0 / wl;
    p.inv_wl2 = p.inv_wl * p.inv_wl;
    p.z2pi = (2.0 * M_PI) * dz;
    p.c = (M_PI * wl) * dz;
    const double phi = ((-2.0 * M_PI) / wl) * dz;
    p.A = make_double2(std::cos(phi), std::sin(phi));
    p.fac = 1.0 / double(n);
    p.dx = dx;
    p.rdx = 1.0 / dx;
    const double frac = cutoff_freq * dx;
    const double start = std::ceil(double(n) * frac);
    if (!(start > double(n) / 2.0)) {
        p.has_cut = 1;
        p.cut_lo = int64_t(start);
        p.cut_hi = std::min<int64_t>(n - int64_t(start) + 1, n);
    }
    return p;
}

// Chirp form of the transfer-function phase for two-level plans: theta =
// c fx^2 with fx = ks / (N dx) exactly, i.e. G ks^2 turns with
// G = c / (2 pi N^2 dx^2), evaluated in long double and split into a
// double-double (c is the reference's rounded fl(fl(pi wl) dz)).
static void chirp_constant(const PropArgs &p, int64_t n, double *g_hi, double *g_lo) {
    const long double two_pi = 6.283185307179586476925286766559005768L;
    const long double ldx = (long double)p.dx;
    const long double nn = (long double)n;
    const long double g = (long double)p.c / (two_pi * nn * nn * ldx * ldx);
    *g_hi = double(g);
    *g_lo = double(g - (long double)(*g_hi));
}

// np.linspace chunk coordinates of generate_grating_chunk
// (big-wave/optical_element.py:341-357): per chunk (x_start, step).
static void chunk_coords(int64_t n, int64_t cs, double dx, double x_pos, std::vector<double> &xs,
                         std::vector<double> &st) {
    xs.clear();
    st.clear();
    if (cs <= 0 || cs > n) cs = n;
    for (int64_t idx = 0; idx < n; idx += cs) {
        const int64_t cnt = std::min(cs, n - idx);
        const int64_t start = idx - n / 2;
        const double x_start = double(start) * dx + x_pos;
        const double x_stop = x_start + double(cnt) * dx;
        const double delta = x_stop - x_start;
        xs.push_back(x_start);
        st.push_back(delta / double(cnt));
    }
}

// Detector geometry of square_and_downsample (big-wave/propagation.py:279-320):
// np.histogram bin membership turned into sample-index boundaries (positions
// (i - N/2)*dx are monotone in i), plus per-pixel cos(atan(x/z)) and r.
struct DetectorGeom {
    int64_t n_pix = 0;
    std::vector<int64_t> bounds;  // n_pix + 1
    std::vector<double> cosv, rv;
};

static rsw_status detector_geom(int64_t n, double dx, double det_size, double psx, double z, DetectorGeom &g) {
    if (!(psx > 0) || !(det_size > 0)) return fail(RSW_ERR_INVALID, "detector size and pixel size must be positive");
    const double nf = py_floordiv(det_size, psx);
    const int64_t outsize = int64_t(nf);
    // more pixels than samples is allowed (the pixels no sample reaches stay 0,
    // as in np.histogram); one CTA per pixel bounds the count by the grid
    if (!(nf <= 2147483647.0))
        return fail(RSW_ERR_UNSUPPORTED, "detector has %.0f pixels: at most 2^31 - 1", nf);
    g.n_pix = outsize;
    const double first = -(double(outsize) / 2.0) * psx;
    const double last = (double(outsize) / 2.0 + 1.0) * psx;
    const int64_t nb = outsize + 1;
    const double denom = last - first;
    const double step = denom / double(nb);
    auto edge = [&](int64_t i) { return i >= nb ? last : double(i) * step + first; };
    auto pos = [&](int64_t i) { return (double(i) - double(n) / 2.0) * dx; };  // the reference's N / 2
    auto bin = [&](double a) -> int64_t {
        const double f = ((a - first) / denom) * double(nb);
        int64_t idx = int64_t(f);
        if (idx == nb) idx -= 1;
        if (a < edge(idx)) idx -= 1;
        if (a >= edge(idx + 1) && idx != nb - 1) idx += 1;
        return idx;
    };
    // kept samples: first <= a <= last
    int64_t lo = 0, hi = n;  // first i with pos(i) >= first
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (pos(mid) >= first) hi = mid; else lo = mid + 1;
    }
    const int64_t n_lo = lo;
    lo = 0;
    hi = n;  // first i with pos(i) > last
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (pos(mid) > last) hi = mid; else lo = mid + 1;
    }
    const int64_t n_end = std::max(lo, n_lo);
    g.bounds.assign(outsize + 1, n_end);
    for (int64_t j = 0; j <= outsize; ++j) {
        int64_t a = n_lo, b = n_end;  // first i in [n_lo, n_end) with bin(pos(i)) >= j
        while (a < b) {
            int64_t mid = a + (b - a) / 2;
            if (bin(pos(mid)) >= j) b = mid; else a = mid + 1;
        }
        g.bounds[j] = a;
    }
    // x = (np.arange(n) - n // 2) * psx with n the float detector_size // psx (util.py:78-82)
    const double half = py_floordiv(nf, 2.0);
    g.cosv.resize(outsize);
    g.rv.resize(outsize);
    for (int64_t j = 0; j < outsize; ++j) {
        const double x = (double(j) - half) * psx;
        g.cosv[j] = std::cos(std::atan(x / z));
        g.rv[j] = std::sqrt(x * x + z * z);
    }
    return RSW_OK;
}

// ---------------------------------------------------------------- buffers
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes) {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    rsw_status alloc(size_t b) {
        if (bytes >= b && p) return RSW_OK;
        release();
        if (b == 0) return RSW_OK;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(RSW_ERR_NOMEM, "cudaMalloc(%zu): %s", b, cudaGetErrorString(e));
        }
        bytes = b;
        return RSW_OK;
    }
    template <typename T> rsw_status upload(const std::vector<T> &v) {
        CHECK(alloc(v.size() * sizeof(T)));
        if (!v.empty()) CU(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
        return RSW_OK;
    }
};

// -------------------------------------------------------------------- plan
static constexpr int ROW_MAX_C128 = 13, COL_MAX_C128 = 11;
// complex128 columns of 2^12 (two-column tiles): two-level plans only, for
// 2^25 (built in: 1.05 ms per split step against 1.31 ms for three levels)
// and for tunings
static constexpr int COL_TUNE_MAX_C128 = 12;
static constexpr int ROW_MAX_C64 = 14, COL_MAX_C64 = 12;
static std::atomic<uint64_t> g_api_calls{0};

struct rsw_plan_s {
    int64_t n = 0;
    int log_n = 0;
    int dtype = RSW_C128;
    int log_n1 = 0, log_n2 = 0;  // column level, row level: N = N1 * N2
    int log_nb = 0, log_nr = 0;  // N2 = Nb * Nr: middle level (0: two-level) and row-kernel length
    int device = 0;
    int row_e = 16, col_e = 16, mid_e = 16;  // elements per thread of the row / column / middle kernels
    int prop_mode = RSW_PROP_FRESNEL;        // transfer function of propagate and of simulations
    DevBuf tw_row, tw_col, tw_mid, tw4_lo, tw4_hi, tw4b_lo, tw4b_hi;
    int tw4_shift = 0, tw4b_shift = 0;
    DevBuf scratch;                                       // N samples, for the natural-order APIs
    DevBuf det_bounds, det_cos, det_r;                    // cached detector geometry
    double det_key[5] = {0, 0, 0, 0, 0};
    int64_t det_npix = -1;
    DevBuf chunk_xs, chunk_st;                            // per-call chunk tables
    DevBuf sample_grid, sample_db, sample_fac;            // per-call sample row data
    DevBuf h3_call;                                       // per-call chirp table
    // lengths that are not a power of two (Bluestein): the power-of-two plan
    // of length m >= 2n - 1, the chirp exp(i pi k^2 / n) (n entries, FP64), the
    // FP64 spectrum of the extended chirp (m entries) and m samples of work space
    bool blue = false;
    std::unique_ptr<rsw_plan_s> inner;
    int64_t m = 0;
    DevBuf bchirp, bhat, bwork;
    bool dbl() const { return dtype == RSW_C128; }
    size_t elem() const { return dbl() ? 16 : 8; }
    bool three() const { return log_nb > 0; }
};

// W_M^m = exp(-2 pi i m / M), accurate to < 1 ulp (long double evaluation)
static cplx twiddle(int64_t m, int64_t M) {
    m %= M;
    if (m < 0) m += M;
    const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)M;
    return cplx(double(cosl(ang)), double(sinl(ang)));
}

template <typename T> static void push_c(std::vector<T> &v, cplx c) {
    v.push_back(T(c.real()));
    v.push_back(T(c.imag()));
}

// Packed lifting form {a, b} of W_M^m = exp(-2 pi i m / M) for complex64
// block tables (rotation by three shears, rsw_block_fft.cuh), for the entry's
// tw_mode (rsw_stages.h): mode 0 rotates by the angle itself (below a quarter
// turn), mode 1 by the angle + pi/2 (the kernel adds the quarter turn); mode
// 2 reduces m to (-M/2, M/2] and beyond a quarter turn takes out a half
// turn, carried in the lowest mantissa bit of a (a is rounded to the nearest
// float whose low bit is the flag). Then t = -2 pi m' / M has |t| <= pi/2,
// a = -tan(t/2), b = sin(t).
static void push_lift(std::vector<float> &v, int64_t m, int64_t M, int mode) {
    m %= M;
    if (m < 0) m += M;
    unsigned flip = 0;
    if (mode == 1) {
        m -= M / 4;
    } else if (mode == 2) {
        if (m > M / 2) m -= M;
        if (4 * m > M) {
            m -= M / 2;
            flip = 1;
        } else if (4 * m < -M) {
            m += M / 2;
            flip = 1;
        }
    }
    const long double pi = 3.14159265358979323846264338327950288L;
    const long double t = -2.0L * pi * (long double)m / (long double)M;
    const long double a = -tanl(t / 2);
    float af = float(a);
    uint32_t bits;
    std::memcpy(&bits, &af, 4);
    if (mode == 2 && (bits & 1u) != flip) af = std::nextafter(af, (long double)af < a ? HUGE_VALF : -HUGE_VALF);
    v.push_back(af);
    v.push_back(float(sinl(t)));
}

// Block twiddle tables of a block of length 2^log_l in the shared-memory
// layout of the block FFT (rsw_stages.h): stages in order, entry k of stage s
// is W_{RS}^m with (m, RS) from stage_tw_entry; 16 bytes per entry ({cos, sin}
// in FP64, or the complex64 lifting form).
template <typename T> static std::vector<T> block_twiddles(int log_l, int rb) {
    std::vector<T> v;
    constexpr bool lift = sizeof(T) == 4;
    if (log_l >= 4) {
        const int max_ls = direct_max_ls(int(2 * sizeof(T)), log_l);
        for (int s = 0; s < stage_count(log_l, rb) - 1; ++s) {
            for (int64_t k = 0; k < stage_tw_entries(log_l, s, max_ls, rb); ++k) {
                int64_t m, mod;
                stage_tw_entry(log_l, s, max_ls, rb, k, &m, &mod);
                if constexpr (lift) push_lift(v, m, mod, stage_tw_mode(log_l, s, max_ls, rb, k));
                else push_c(v, twiddle(m, mod));
            }
        }
    }
    if (v.empty()) {
        if constexpr (lift) push_lift(v, 0, 1, 0);
        else push_c(v, cplx(1, 0));
    }
    return v;
}

// four-step twiddles W_M^m = lo[m & (2^h - 1)] * hi[m >> h] of M = 2^log_m in
// FP64 for both dtypes (rounded per tile on the device)
static rsw_status four_step_tables(int log_m, DevBuf &lo_buf, DevBuf &hi_buf, int *shift) {
    const int h = (log_m + 1) / 2;
    const int64_t m = int64_t(1) << log_m;
    *shift = h;
    std::vector<double> lo, hi;
    for (int64_t a = 0; a < (int64_t(1) << h); ++a) push_c(lo, twiddle(a, m));
    for (int64_t b = 0; b < (int64_t(1) << (log_m - h)); ++b) push_c(hi, twiddle(b << h, m));
    CHECK(lo_buf.upload(lo));
    return hi_buf.upload(hi);
}

template <typename T> static rsw_status plan_tables(rsw_plan_s *p) {
    CHECK(p->tw_row.upload(block_twiddles<T>(p->log_nr, digit_bits(p->row_e))));
    if (p->log_n1 > 0) {
        CHECK(p->tw_col.upload(block_twiddles<T>(p->log_n1, digit_bits(p->col_e))));
        CHECK(four_step_tables(p->log_n, p->tw4_lo, p->tw4_hi, &p->tw4_shift));
    }
    if (p->three()) {
        CHECK(p->tw_mid.upload(block_twiddles<T>(p->log_nb, digit_bits(p->mid_e))));
        CHECK(four_step_tables(p->log_n2, p->tw4b_lo, p->tw4b_hi, &p->tw4b_shift));
    }
    return RSW_OK;
}

// Level split of N = 2^lg: one row level up to the row kernel's limit; two
// levels (columns x rows) up to the column limit times the row limit; beyond
// that three levels, N = N1 x Nb x Nr, with rows of the row kernel's maximum
// length and the rest split evenly between the outer column level and the
// middle level (both run by the column kernel).
// A split from a tuning (levels 1..3): single level; columns of 2^log_rows
// and rows of the rest; columns, a middle level of 2^log_mid and rows.
static rsw_status tuned_split(int lg, int dtype, const rsw_tuning &t, int *l1, int *lb, int *lr) {
    const int row_max = dtype == RSW_C128 ? ROW_MAX_C128 : ROW_MAX_C64;
    const int col_max = dtype == RSW_C128 ? COL_MAX_C128 : COL_MAX_C64;
    *lb = 0;
    if (t.levels == 1) {
        if (lg > row_max) return fail(RSW_ERR_INVALID, "tuning: 2^%d is above the single-level limit 2^%d", lg, row_max);
        *l1 = 0;
        *lr = lg;
        return RSW_OK;
    }
    const int a = t.log_rows, b = t.levels == 3 ? t.log_mid : 0, c = lg - a - b;
    const int a_max = t.levels == 2 && dtype == RSW_C128 ? COL_TUNE_MAX_C128 : col_max;
    if (a < 4 || a > a_max || (t.levels == 3 && (b < 4 || b > col_max)) || c < 7 || c > row_max ||
        (t.levels != 2 && t.levels != 3))
        return fail(RSW_ERR_INVALID, "tuning: split %d levels, %d / %d / %d of 2^%d is not available", t.levels, a, b,
                    c, lg);
    *l1 = a;
    *lb = b;
    *lr = c;
    return RSW_OK;
}

static rsw_status plan_split(int64_t n, int dtype, int *log_n, int *l1, int *lb, int *lr, const rsw_tuning *t) {
    if (n < 16 || (n & (n - 1)) != 0)
        return fail(RSW_ERR_UNSUPPORTED, "N = %lld: this version supports powers of two >= 16", (long long)n);
    int lg = 0;
    while ((int64_t(1) << lg) < n) ++lg;
    const int row_max = dtype == RSW_C128 ? ROW_MAX_C128 : ROW_MAX_C64;
    const int col_max = dtype == RSW_C128 ? COL_MAX_C128 : COL_MAX_C64;
    *log_n = lg;
    *lb = 0;
    if (t && t->levels != 0) return tuned_split(lg, dtype, *t, l1, lb, lr);
    // RSW_SPLIT3 = "l1,lb,lr" forces a three-level split (tests and tuning sweeps)
    const char *ov3 = std::getenv("RSW_SPLIT3");
    if (ov3 && *ov3) {
        int a = 0, b = 0, c = 0;
        if (std::sscanf(ov3, "%d,%d,%d", &a, &b, &c) == 3 && a + b + c == lg && a >= 4 && a <= col_max &&
            b >= 4 && b <= col_max && c >= 7 && c <= row_max) {
            *l1 = a;
            *lb = b;
            *lr = c;
            return RSW_OK;
        }
    }
    // RSW_SPLIT = "l1" forces a two-level split with columns of 2^l1 when
    // valid, also for lengths that fit one row (tests and tuning sweeps)
    const char *ov = std::getenv("RSW_SPLIT");
    if (ov && *ov) {
        const int oa = std::atoi(ov), ob = lg - oa;
        if (oa >= 4 && oa <= col_max && ob >= 7 && ob <= row_max) {
            *l1 = oa;
            *lr = ob;
            return RSW_OK;
        }
    }
    if (lg <= row_max) {
        *l1 = 0;
        *lr = lg;
        return RSW_OK;
    }
    const int col2 = dtype == RSW_C128 ? COL_TUNE_MAX_C128 : col_max;  // two-level column limit
    if (lg > row_max + col2) {
        if (lg > row_max + 2 * col_max)
            return fail(RSW_ERR_UNSUPPORTED, "N = 2^%d exceeds the three-level limit 2^%d for this dtype", lg,
                        row_max + 2 * col_max);
        // long outer columns (the pass with the transmission and the factor
        // tables, which amortise over the column length); the middle level
        // runs plain FFTs of what is left, at least 2^4
        const int rest = lg - row_max;
        *lr = row_max;
        *l1 = std::min(std::min(col_max, 11), rest - 4);
        *lb = rest - *l1;
        if (*lb > col_max) {
            *lb = col_max;
            *l1 = rest - col_max;
        }
        return RSW_OK;
    }
    // prefer columns of at most 2^11 (the 2^12 c64 column kernel runs 1024
    // threads at 64 registers and spills); rows take the rest
    int a = std::min(std::min(col_max, 11), lg / 2);
    int b = lg - a;
    if (b > row_max) {
        a = lg - row_max;
        b = row_max;
    }
    if (b < 7) {  // rows of two-level plans hold at least 2^7 samples
        b = 7;
        a = lg - b;
    }
    if (b > row_max) {
        a = lg - row_max;
        b = row_max;
    }
    *l1 = a;
    *lr = b;
    return RSW_OK;
}

// Kernel variant per block size: elements per thread. complex128 columns of
// 2^8 .. 2^11 take 8 per thread (radix-8 stages, 512- or 1024-thread CTAs:
// two to four times the warps per SM of the 16-per-thread kernels, which
// hold up to 252 registers at 256 threads; measured 9-20 % faster), as do
// complex64 columns of 2^9 (16 per CTA, 6 %) and of 2^10 in two-level plans
// (at most 2^21 samples: too few tiles of 16 columns for 148 SMs). Other
// complex64 columns of 2^10 and 2^11 keep 16 per thread, which leaves room
// for 16 or 8 columns per CTA (128- or 64-byte row segments; 8 per thread
// with 4 columns measured 26-40 % slower). Everything else takes 16.
// RSW_ROW_E / RSW_COL_E (8, 16 or 32) override the choice (tuning sweeps).
static int env_int(const char *name, int dflt) {
    const char *v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}
// Samples per thread the kernels are built for: multi-level rows 16 from
// 2^7, 32 from 2^9, 8 for 2^11..2^13 (single-level rows 16); columns (and
// middle levels) 16, 8 for 2^8..2^11, 32 from 2^9.
static bool row_e_ok(int log_nr, bool multi, int e) {
    if (!multi) return e == 16;
    return (e == 16 && log_nr >= 7) || (e == 32 && log_nr >= 9) || (e == 8 && log_nr >= 11 && log_nr <= 13);
}
static bool col_e_ok(int log_l, int e, bool c128) {
    if (c128 && log_l == 12) return e == 8 || e == 16;
    return (e == 16 && log_l >= 4) || (e == 8 && log_l >= 8 && log_l <= 11) || (e == 32 && log_l >= 9);
}

static rsw_status choose_tuning(rsw_plan_s *p, const rsw_tuning *t) {
    auto pick = [](int log_l, int dflt) { return log_l >= 9 ? dflt : 16; };
    p->row_e = pick(p->log_nr, 16);
    const bool c128 = p->dtype == RSW_C128;
    const int l1 = p->log_n1;
    p->col_e = (c128 && l1 >= 8 && l1 <= 12) || (!c128 && (l1 == 9 || (l1 == 10 && p->log_nb == 0))) ? 8 : pick(l1, 16);
    p->mid_e = pick(p->log_nb, 16);
    if (t) {
        const bool multi = p->log_n1 > 0;
        if (t->row_e && !row_e_ok(p->log_nr, multi, t->row_e))
            return fail(RSW_ERR_INVALID, "tuning: rows of 2^%d have no kernel with %d samples per thread", p->log_nr,
                        t->row_e);
        if (t->col_e && (!multi || !col_e_ok(p->log_n1, t->col_e, c128)))
            return fail(RSW_ERR_INVALID, "tuning: no column kernel of 2^%d with %d samples per thread", p->log_n1,
                        t->col_e);
        if (t->mid_e && (!p->three() || !col_e_ok(p->log_nb, t->mid_e, c128)))
            return fail(RSW_ERR_INVALID, "tuning: no middle kernel of 2^%d with %d samples per thread", p->log_nb,
                        t->mid_e);
        if (t->row_e) p->row_e = t->row_e;
        if (t->col_e) p->col_e = t->col_e;
        if (t->mid_e) p->mid_e = t->mid_e;
        return RSW_OK;
    }
    const int re = env_int("RSW_ROW_E", 0), ce = env_int("RSW_COL_E", 0);
    if ((re == 16 || re == 32) && p->log_nr >= 9) p->row_e = re;
    if (ce == 16 || (ce == 32 && p->log_n1 >= 9)) p->col_e = ce;
    // 8 samples per thread: multi-level rows of 2^11..2^13, columns of 2^8..2^11
    if (re == 8 && p->log_n1 > 0 && p->log_nr >= 11 && p->log_nr <= 13) p->row_e = 8;
    if (ce == 8 && p->log_n1 >= 8 && p->log_n1 <= 11) p->col_e = 8;
    return RSW_OK;
}

// Tunings registered for later plans (rsw_set_tuning), per length and dtype.
struct TuningEntry {
    int64_t n;
    int dtype;
    rsw_tuning t;
};
static std::mutex g_tuning_mutex;
static std::vector<TuningEntry> g_tunings;
static bool registered_tuning(int64_t n, int dtype, rsw_tuning *t) {
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    for (const TuningEntry &e : g_tunings)
        if (e.n == n && e.dtype == dtype) {
            *t = e.t;
            return true;
        }
    return false;
}
// the tuning environment variables of tests and sweeps take precedence over
// registered tunings
static bool env_overrides() {
    for (const char *v : {"RSW_SPLIT", "RSW_SPLIT3", "RSW_ROW_E", "RSW_COL_E"}) {
        const char *x = std::getenv(v);
        if (x && *x) return true;
    }
    return false;
}

// Arguments of the outer column pass (and of single-level row passes).
//
// Between split steps the field is kept in the "mid" layout: the column
// spectrum (row p1 holds column frequency k1 = digitrev(p1)) with the row
// level already inverted. The column pass applies W_N^(n2 k1) after its
// forward (PF_TW). Two-level plans apply conj(W_N^(n2 k1)) / N at the end of
// the row pass (PF_TW of the row kernel). Three-level plans apply it in the
// column pass before the inverse (PF_TWI, from the same factor table) and
// W_{N2}^(nr kb) around the row transform (PF_TWF before, PF_TW after), so
// that their middle passes are plain FFTs.
static PassArgs base_args(const rsw_plan_s *p) {
    PassArgs a{};
    a.n = p->n;
    a.log_n1 = p->log_n1;
    a.log_n2 = p->log_n2;
    a.tw_row = p->tw_row.p;
    a.tw_col = p->tw_col.p;
    a.tw4_lo = p->tw4_lo.p;
    a.tw4_hi = p->tw4_hi.p;
    a.tw4_shift = p->tw4_shift;
    a.tw_log = p->log_n;
    a.tw_scale = 1.0 / double(p->n);
    a.rb_n1 = digit_bits(p->col_e);
    a.rb_nb = digit_bits(p->mid_e);
    a.pr.fac = 1.0 / double(p->n);
    a.tr.kind = TR_NONE;
    a.det.n_inst = 1;
    return a;
}
// detector sums of one instance of a batched detection pass: n_pix doubles
// rounded up to a 256-byte multiple
static int64_t batch_sum_stride(int64_t n_pix) { return (n_pix + 31) / 32 * 32; }
// The same arguments for the row kernel: rows of Nr samples; in three-level
// plans its twiddles are W_{N2}^(nr kb), unscaled.
static PassArgs row_level(const rsw_plan_s *p, PassArgs a) {
    a.log_n2 = p->log_nr;
    a.log_nb = p->log_nb;
    if (p->three()) {
        a.tw4_lo = p->tw4b_lo.p;
        a.tw4_hi = p->tw4b_hi.p;
        a.tw4_shift = p->tw4b_shift;
        a.tw_log = p->log_n2;
        a.tw_scale = 1.0;
    }
    return a;
}
// row-pass twiddle flags of a multi-level plan
static int row_tw(const rsw_plan_s *p, bool fwd, bool inv) {
    return p->three() ? ((fwd ? PF_TWF : 0) | (inv ? PF_TW : 0)) : (inv ? PF_TW : 0);
}
// column-pass flags of the inverse of the "mid" layout
static int col_inv(const rsw_plan_s *p) { return PF_INV | (p->three() ? PF_TWI : 0); }
// The middle level of three-level plans: the column kernel over N1 batches
// of Nb x Nr, a plain FFT over nb.
static PassArgs mid_level(const rsw_plan_s *p, PassArgs a) {
    a.log_n1 = p->log_nb;
    a.log_n2 = p->log_nr;
    a.log_nb = 0;
    a.tw_col = p->tw_mid.p;
    a.tr.kind = TR_NONE;
    return a;
}

// ------------------------------------------------------------ timing hooks
struct TimingLog {
    bool enabled = false;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    double ms[4] = {0, 0, 0, 0};  // row, column, detect, middle
    int64_t launches[4] = {0, 0, 0, 0};
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int kind, cudaStream_t s, Rec &r) {
        r.kind = kind;
        r.a = get();
        r.b = get();
        cudaEventRecord(r.a, s);
    }
    void end(Rec &r, cudaStream_t s) {
        cudaEventRecord(r.b, s);
        recs.push_back(r);
    }
    void collect() {
        for (auto &r : recs) {
            cudaEventSynchronize(r.b);
            float t = 0;
            cudaEventElapsedTime(&t, r.a, r.b);
            ms[r.kind] += t;
            launches[r.kind] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        recs.clear();
    }
    ~TimingLog() {
        for (auto &r : recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

static rsw_status run_row(const rsw_plan_s *p, const PassArgs &a, cudaStream_t s, TimingLog *tl = nullptr) {
    TimingLog::Rec r{};
    if (tl && tl->enabled) tl->begin(0, s, r);
    cudaError_t e = launch_row_pass(a, p->dbl(), p->row_e, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "row pass (2^%d): %s", a.log_n2, cudaGetErrorString(e));
    if (tl && tl->enabled) tl->end(r, s);
    return RSW_OK;
}
static rsw_status run_col(const rsw_plan_s *p, const PassArgs &a, cudaStream_t s, TimingLog *tl = nullptr) {
    TimingLog::Rec r{};
    if (tl && tl->enabled) tl->begin(1, s, r);
    cudaError_t e = launch_col_pass(a, p->dbl(), p->col_e, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "column pass (2^%d): %s", a.log_n1, cudaGetErrorString(e));
    if (tl && tl->enabled) tl->end(r, s);
    return RSW_OK;
}
// middle pass of a three-level plan
static rsw_status run_mid(const rsw_plan_s *p, const PassArgs &base, bool forward, cudaStream_t s,
                          TimingLog *tl = nullptr) {
    PassArgs a = mid_level(p, base);
    a.flags = forward ? PF_FWD : PF_INV;
    TimingLog::Rec r{};
    if (tl && tl->enabled) tl->begin(3, s, r);
    cudaError_t e = launch_col_pass(a, p->dbl(), p->mid_e, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "middle pass (2^%d): %s", a.log_n1, cudaGetErrorString(e));
    if (tl && tl->enabled) tl->end(r, s);
    return RSW_OK;
}

// Build the row-level chirp table of a transfer function into `table` (Nr
// samples) and switch `pr` to the chirp form. Multi-level plans only: the
// spectrum index of a row sample is kbase + M k2 with M = N1 Nb.
static rsw_status prepare_chirp(const rsw_plan_s *p, PropArgs &pr, void *table, cudaStream_t s) {
    if (p->log_n1 == 0 || !pr.has_h || pr.exact) return RSW_OK;
    double g_hi, g_lo;
    chirp_constant(pr, p->n, &g_hi, &g_lo);
    const double msq = std::ldexp(1.0, 2 * (p->log_n1 + p->log_nb));  // exact power of two
    cudaError_t e = launch_chirp_table(table, p->log_nr, g_hi * msq, g_lo * msq, p->dbl(), p->row_e, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "chirp table: %s", cudaGetErrorString(e));
    pr.chirp = 1;
    pr.g_hi = g_hi;
    pr.g_lo = g_lo;
    pr.h3 = table;
    return RSW_OK;
}

// The launches of one split step from `a.in` (NULL with ones: the plane
// wave) into `a.out`, with a.tr / a.pr set: multi-level plans run the column
// pass (the inverse of the previous step when the input is in the "mid"
// representation, transmission, forward), the middle passes of three-level
// plans around the row pass, and leave the "mid" representation; single-level
// plans run one row pass and leave the field in natural order.
static rsw_status launch_split_step(const rsw_plan_s *P, PassArgs a, bool mid_in, bool ones, cudaStream_t st,
                                    TimingLog *tl, bool *mid_out) {
    const bool trans = a.tr.kind != TR_NONE;
    if (P->log_n1 > 0) {
        const void *out = a.out;
        a.flags = (mid_in ? col_inv(P) : 0) | PF_FWD | PF_TW | (trans ? PF_TRANS : 0) | (ones ? PF_ONES : 0);
        const PropArgs keep = a.pr;
        a.pr = PropArgs{};
        CHECK(run_col(P, a, st, tl));
        a.in = out;
        a.tr.kind = TR_NONE;
        a.btr = nullptr;
        if (P->three()) CHECK(run_mid(P, a, true, st, tl));
        a.pr = keep;
        PassArgs r = row_level(P, a);
        r.flags = PF_FWD | PF_INV | row_tw(P, true, true);
        CHECK(run_row(P, r, st, tl));
        if (P->three()) {
            a.pr = PropArgs{};
            CHECK(run_mid(P, a, false, st, tl));
        }
        *mid_out = true;
    } else {
        a.flags = PF_FWD | PF_INV | PF_SCALE | (trans ? PF_TRANS : 0) | (ones ? PF_ONES : 0);
        CHECK(run_row(P, a, st, tl));
        *mid_out = false;
    }
    return RSW_OK;
}

// ================================================================== C ABI
extern "C" {

const char *rsw_last_error(void) { return t_last_error.c_str(); }
int rsw_abi_version(void) { return RSW_ABI_VERSION; }
uint64_t rsw_launch_count(void) { return uint64_t(launch_count()); }
double rsw_energy_to_wavelength(double energy_ev) { return wavelength(energy_ev); }
size_t rsw_struct_size(int which) {
    switch (which) {
    case 0: return sizeof(rsw_element);
    case 1: return sizeof(rsw_sim_desc);
    case 2: return sizeof(rsw_source);
    case 3: return sizeof(rsw_source_run);
    case 4: return sizeof(rsw_tuning);
    default: return 0;
    }
}

static rsw_status create_blue_plan(rsw_plan *out, int64_t n, int dtype);

static rsw_status create_plan(rsw_plan *out, int64_t n, int dtype, const rsw_tuning *t) {
    if (!out) return fail(RSW_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (dtype != RSW_C128 && dtype != RSW_C64) return fail(RSW_ERR_INVALID, "unknown dtype %d", dtype);
    // lengths that are not a power of two, and powers of two below 16
    if (n >= 1 && ((n & (n - 1)) != 0 || n < 16)) return create_blue_plan(out, n, dtype);
    int lg = 0, l1 = 0, lb = 0, lr = 0;
    CHECK(plan_split(n, dtype, &lg, &l1, &lb, &lr, t));
    std::unique_ptr<rsw_plan_s> p(new (std::nothrow) rsw_plan_s());
    if (!p) return fail(RSW_ERR_NOMEM, "host allocation failed");
    p->n = n;
    p->log_n = lg;
    p->dtype = dtype;
    p->log_n1 = l1;
    p->log_nb = lb;
    p->log_nr = lr;
    p->log_n2 = lb + lr;
    CU(cudaGetDevice(&p->device));
    CHECK(choose_tuning(p.get(), t));
    CHECK(p->dbl() ? plan_tables<double>(p.get()) : plan_tables<float>(p.get()));
    *out = p.release();
    return RSW_OK;
}

// A plan for a length that is not a power of two (Bluestein's algorithm over
// the power-of-two plan of length m >= 2n - 1). The extended chirp's spectrum
// is taken once with an FP64 plan of length m, also for complex64 plans.
static rsw_status create_blue_plan(rsw_plan *out, int64_t n, int dtype) {
    if (n > (int64_t(1) << 31)) return fail(RSW_ERR_UNSUPPORTED, "lengths that are not a power of two: at most 2^31");
    int64_t m = 16;
    while (m < 2 * n - 1) m <<= 1;
    std::unique_ptr<rsw_plan_s> p(new (std::nothrow) rsw_plan_s());
    if (!p) return fail(RSW_ERR_NOMEM, "host allocation failed");
    p->n = n;
    p->dtype = dtype;
    p->blue = true;
    p->m = m;
    CU(cudaGetDevice(&p->device));
    rsw_plan inner = nullptr;
    rsw_tuning reg{};
    const bool use = !env_overrides() && registered_tuning(m, dtype, &reg);
    CHECK(create_plan(&inner, m, dtype, use ? &reg : nullptr));
    p->inner.reset(inner);
    // chirp b[k] = exp(i pi k^2 / n), k^2 reduced mod 2n exactly
    const long double pi = 3.14159265358979323846264338327950288L;
    std::vector<double> b(size_t(2 * n)), bx(size_t(2 * m), 0.0);
    for (int64_t k = 0; k < n; ++k) {
        const uint64_t r = (uint64_t(k) * uint64_t(k)) % uint64_t(2 * n);
        const long double ang = pi * (long double)r / (long double)n;
        b[size_t(2 * k)] = double(cosl(ang));
        b[size_t(2 * k + 1)] = double(sinl(ang));
    }
    // extended chirp: b[j] at j and at m - j
    for (int64_t j = 0; j < n; ++j) {
        bx[size_t(2 * j)] = b[size_t(2 * j)];
        bx[size_t(2 * j + 1)] = b[size_t(2 * j + 1)];
        if (j > 0) {
            bx[size_t(2 * (m - j))] = b[size_t(2 * j)];
            bx[size_t(2 * (m - j) + 1)] = b[size_t(2 * j + 1)];
        }
    }
    CHECK(p->bchirp.upload(b));
    CHECK(p->bhat.upload(bx));
    rsw_plan p64 = inner;
    std::unique_ptr<rsw_plan_s> own;
    if (dtype != RSW_C128) {
        CHECK(create_plan(&p64, m, RSW_C128, nullptr));
        own.reset(p64);
    }
    CHECK(rsw_fft_forward(p64, p->bhat.p, p->bhat.p, nullptr));
    CU(cudaDeviceSynchronize());  // the spectrum is complete before the temporary plan goes
    CHECK(p->bwork.alloc(size_t(m) * p->elem()));
    *out = p.release();
    return RSW_OK;
}

// Natural-order DFT of a Bluestein plan (inverse: conj(DFT(conj X)) / n).
static rsw_status blue_transform(rsw_plan_s *p, const void *in, void *out, bool inverse, cudaStream_t s) {
    cudaError_t e = launch_blue_pre(in, p->bwork.p, p->n, p->m, (const double2 *)p->bchirp.p, inverse, p->dbl(), s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "bluestein: %s", cudaGetErrorString(e));
    CHECK(rsw_fft_forward(p->inner.get(), p->bwork.p, p->bwork.p, s));
    e = launch_blue_mul(p->bwork.p, (const double2 *)p->bhat.p, p->m, p->dbl(), s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "bluestein: %s", cudaGetErrorString(e));
    CHECK(rsw_fft_inverse(p->inner.get(), p->bwork.p, p->bwork.p, s));
    e = launch_blue_post(p->bwork.p, out, p->n, (const double2 *)p->bchirp.p, inverse ? 1.0 / double(p->n) : 1.0,
                         inverse, p->dbl(), s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "bluestein: %s", cudaGetErrorString(e));
    return RSW_OK;
}

// propagate() of a Bluestein plan: U = FFT(u) (unless given), transfer
// function and cutoff on the natural-order spectrum, u = iFFT(U).
static rsw_status blue_propagate(rsw_plan_s *p, void *u, void *U, const PropArgs &pr, bool skip_fft, cudaStream_t s) {
    void *spec = U;
    if (!spec) {
        CHECK(p->scratch.alloc(size_t(p->n) * p->elem()));
        spec = p->scratch.p;
    }
    if (!skip_fft) CHECK(blue_transform(p, u, spec, false, s));
    cudaError_t e = launch_prop_natural(spec, p->n, pr, p->dbl(), s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "transfer function: %s", cudaGetErrorString(e));
    return blue_transform(p, spec, u, true, s);
}

rsw_status rsw_plan_create(rsw_plan *out, int64_t n, int dtype) {
    rsw_tuning reg{};
    const bool use = !env_overrides() && registered_tuning(n, dtype, &reg);
    return create_plan(out, n, dtype, use ? &reg : nullptr);
}

rsw_status rsw_plan_create_tuned(rsw_plan *out, int64_t n, int dtype, const rsw_tuning *t) {
    return create_plan(out, n, dtype, t);
}

rsw_status rsw_plan_tuning(rsw_plan p, rsw_tuning *t) {
    if (!p || !t) return fail(RSW_ERR_INVALID, "NULL argument");
    if (p->blue) return rsw_plan_tuning(p->inner.get(), t);  // the transforms of length m do the work
    t->levels = p->log_n1 == 0 ? 1 : p->three() ? 3 : 2;
    t->log_rows = p->log_n1;
    t->log_mid = p->log_nb;
    t->row_e = p->row_e;
    t->col_e = p->log_n1 > 0 ? p->col_e : 0;
    t->mid_e = p->three() ? p->mid_e : 0;
    return RSW_OK;
}

rsw_status rsw_set_tuning(int64_t n, int dtype, const rsw_tuning *t) {
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    g_tunings.erase(std::remove_if(g_tunings.begin(), g_tunings.end(),
                                   [&](const TuningEntry &e) { return e.n == n && e.dtype == dtype; }),
                    g_tunings.end());
    if (t) g_tunings.push_back(TuningEntry{n, dtype, *t});
    return RSW_OK;
}

// The plan choice cuFFT makes inside cufftPlan1d (fast-wave/src/fft.cpp:8),
// made here by measurement: every split and samples-per-thread combination
// the kernels are built for is timed on one steady-state split step of a
// simulation (inverse column pass, grating transmission, forward column
// pass, [middle passes,] row pass with the chirp transfer function) over a
// field of n samples on the device, and the fastest is returned.
rsw_status rsw_autotune(int64_t n, int dtype, int reps, rsw_tuning *best, double *best_ms, rsw_tuning *tried,
                        double *tried_ms, int max_tried, int *n_tried, void *stream) {
    return rsw_autotune_batch(n, dtype, 1, reps, best, best_ms, tried, tried_ms, max_tried, n_tried, stream);
}

rsw_status rsw_autotune_batch(int64_t n, int dtype, int64_t fields, int reps, rsw_tuning *best, double *best_ms,
                              rsw_tuning *tried, double *tried_ms, int max_tried, int *n_tried, void *stream) {
    if (!best) return fail(RSW_ERR_INVALID, "best is NULL");
    if (fields < 1 || fields > RSW_BATCH_MAX) return fail(RSW_ERR_INVALID, "fields must be in [1, %d]", RSW_BATCH_MAX);
    if (dtype != RSW_C128 && dtype != RSW_C64) return fail(RSW_ERR_INVALID, "unknown dtype %d", dtype);
    if (n < 16 || (n & (n - 1)) != 0)
        return fail(RSW_ERR_UNSUPPORTED, "N = %lld: this version supports powers of two >= 16", (long long)n);
    if (reps < 1) reps = 1;
    int lg = 0;
    while ((int64_t(1) << lg) < n) ++lg;
    const int row_max = dtype == RSW_C128 ? ROW_MAX_C128 : ROW_MAX_C64;
    const int col_max = dtype == RSW_C128 ? COL_MAX_C128 : COL_MAX_C64;
    std::vector<rsw_tuning> cands;
    if (lg <= row_max) cands.push_back(rsw_tuning{1, 0, 0, 16, 0, 0});
    const bool c128 = dtype == RSW_C128;
    const int col_tune = c128 ? COL_TUNE_MAX_C128 : col_max;
    if (lg <= row_max + col_tune) {
        for (int l1 = 4; l1 <= col_tune; ++l1) {
            const int lr = lg - l1;
            if (lr < 7 || lr > row_max) continue;
            for (int re : {16, 32, 8})
                for (int ce : {16, 8, 32})
                    if (row_e_ok(lr, true, re) && col_e_ok(l1, ce, c128))
                        cands.push_back(rsw_tuning{2, l1, 0, re, ce, 0});
        }
    }
    if (lg > row_max + col_max) {
        // three levels: rows of the longest row kernel (fewest samples in
        // the two column levels), the column lengths and kernels varied
        for (int l1 = 4; l1 <= col_max; ++l1) {
            const int lb = lg - row_max - l1;
            if (lb < 4 || lb > col_max) continue;
            for (int ce : {16, 8})
                for (int me : {16, 8})
                    if (col_e_ok(l1, ce, c128) && col_e_ok(lb, me, c128))
                        cands.push_back(rsw_tuning{3, l1, lb, 16, ce, me});
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t elem = dtype == RSW_C128 ? 16 : 8;
    DevBuf field;
    CHECK(field.alloc(size_t(n) * size_t(fields) * elem));
    {
        cudaError_t e = launch_fill_ones(field.p, n * fields, dtype == RSW_C128, s);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "fill: %s", cudaGetErrorString(e));
    }
    // a grating sub-step at 46 keV on a 2 nm grid, 10 um thick, no cutoff
    const double dx = 2e-9, wl = 2.6953e-11, dz = 1e-5;
    TransArgs tr{};
    tr.kind = TR_GRATING;
    tr.fa = make_double2(0.9, 0.1);
    tr.fb = make_double2(1.0, 0.0);
    tr.pitch0 = 4.2e-6;
    tr.inv_pitch0 = 1.0 / tr.pitch0;
    tr.dc0 = 0.5;
    tr.half_dc0 = 0.25;
    tr.xstart0 = -double(n / 2) * dx;
    tr.step0 = dx;
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    struct Events {
        cudaEvent_t a, b;
        ~Events() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } ev{e0, e1};
    double best_t = 1e300;
    int count = 0;
    for (const rsw_tuning &c : cands) {
        rsw_plan raw = nullptr;
        if (create_plan(&raw, n, dtype, &c) != RSW_OK) continue;
        std::unique_ptr<rsw_plan_s> pl(raw);
        DevBuf h3;
        if (pl->log_n1 > 0 && h3.alloc(size_t(int64_t(1) << pl->log_nr) * 16) != RSW_OK) continue;
        PassArgs a = base_args(pl.get());
        a.n = n * fields;  // the passes over all fields, one launch each
        a.in = field.p;
        a.out = field.p;
        a.tr = tr;
        a.pr = make_prop(n, dx, wl, dz, 1e300, true);
        if (prepare_chirp(pl.get(), a.pr, h3.p, s) != RSW_OK) continue;
        bool mid = false, ok = true;
        for (int w = 0; w < 2 && ok; ++w) ok = launch_split_step(pl.get(), a, pl->log_n1 > 0, false, s, nullptr, &mid) == RSW_OK;
        if (!ok) continue;
        CU(cudaEventRecord(e0, s));
        for (int r = 0; r < reps && ok; ++r)
            ok = launch_split_step(pl.get(), a, pl->log_n1 > 0, false, s, nullptr, &mid) == RSW_OK;
        CU(cudaEventRecord(e1, s));
        CU(cudaEventSynchronize(e1));
        if (!ok) continue;
        float ms = 0;
        CU(cudaEventElapsedTime(&ms, e0, e1));
        const double per = double(ms) / reps;
        if (tried && tried_ms && count < max_tried) {
            tried[count] = c;
            tried_ms[count] = per;
        }
        ++count;
        if (per < best_t) {
            best_t = per;
            CHECK(rsw_plan_tuning(pl.get(), best));
        }
    }
    if (n_tried) *n_tried = count;
    if (count == 0) return fail(RSW_ERR_CUDA, "autotune: no candidate ran for N = 2^%d", lg);
    if (best_ms) *best_ms = best_t;
    return RSW_OK;
}

rsw_status rsw_plan_destroy(rsw_plan plan) {
    delete plan;
    return RSW_OK;
}

rsw_status rsw_plan_info(rsw_plan p, int64_t *n, int *dtype, int *log_rows, int *log_cols, int64_t *scratch) {
    if (!p) return fail(RSW_ERR_INVALID, "plan is NULL");
    if (n) *n = p->n;
    if (dtype) *dtype = p->dtype;
    if (log_rows) *log_rows = p->log_n1;
    if (log_cols) *log_cols = p->log_n2;
    if (scratch) *scratch = int64_t(p->scratch.bytes);
    return RSW_OK;
}

rsw_status rsw_plan_set_propagator(rsw_plan p, int mode) {
    if (!p) return fail(RSW_ERR_INVALID, "plan is NULL");
    if (mode != RSW_PROP_FRESNEL && mode != RSW_PROP_EXACT) return fail(RSW_ERR_INVALID, "unknown propagator %d", mode);
    // the exact kernel runs the per-sample row kernels (16 samples per thread)
    if (mode == RSW_PROP_EXACT && p->log_n1 > 0 && p->row_e != 16)
        return fail(RSW_ERR_UNSUPPORTED, "the exact propagator needs rows of 16 samples per thread");
    p->prop_mode = mode;
    return RSW_OK;
}

static rsw_status need_scratch(rsw_plan_s *p) { return p->scratch.alloc(size_t(p->n) * p->elem()); }

static SpecLevels spec_levels(const rsw_plan_s *p) {
    return SpecLevels{p->log_n1, p->log_nb, p->log_nr, digit_bits(p->col_e), digit_bits(p->mid_e),
                      digit_bits(p->row_e)};
}
static cudaError_t to_natural(const rsw_plan_s *p, const void *spec, void *nat, cudaStream_t s) {
    return launch_spec_to_natural(spec, nat, p->n, spec_levels(p), p->dbl(), s);
}
static cudaError_t to_spec(const rsw_plan_s *p, const void *nat, void *spec, cudaStream_t s) {
    return launch_natural_to_spec(nat, spec, p->n, spec_levels(p), p->dbl(), s);
}

rsw_status rsw_fft_forward(rsw_plan p, const void *in, void *out, void *stream) {
    if (!p || !in || !out) return fail(RSW_ERR_INVALID, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (p->blue) return blue_transform(p, in, out, false, s);
    CHECK(need_scratch(p));
    PassArgs a = base_args(p);
    a.in = in;
    a.out = p->scratch.p;
    if (p->log_n1 > 0) {
        a.flags = PF_FWD | PF_TW;
        CHECK(run_col(p, a, s));
        a.in = p->scratch.p;
        if (p->three()) CHECK(run_mid(p, a, true, s));
    }
    PassArgs r = row_level(p, a);
    r.flags = PF_FWD | row_tw(p, true, false);
    CHECK(run_row(p, r, s));
    cudaError_t e = to_natural(p, p->scratch.p, out, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_fft_inverse(rsw_plan p, const void *in, void *out, void *stream) {
    if (!p || !in || !out) return fail(RSW_ERR_INVALID, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (p->blue) return blue_transform(p, in, out, true, s);
    CHECK(need_scratch(p));
    cudaError_t e = to_spec(p, in, p->scratch.p, s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
    PassArgs a = base_args(p);
    a.in = p->scratch.p;
    if (p->log_n1 > 0) {
        PassArgs r = row_level(p, a);
        r.out = p->scratch.p;
        r.flags = PF_SPEC_IN | PF_INV | row_tw(p, false, true);
        CHECK(run_row(p, r, s));
        a.out = p->scratch.p;
        if (p->three()) CHECK(run_mid(p, a, false, s));
        a.out = out;
        a.flags = col_inv(p);
        CHECK(run_col(p, a, s));
    } else {
        a.out = out;
        a.flags = PF_SPEC_IN | PF_INV | PF_SCALE;
        CHECK(run_row(p, a, s));
    }
    return RSW_OK;
}

// ------------------------------------------------------------ out-of-core FFT
// Natural-order FFTs (inverse: scaled by 1/len) of `count` consecutive
// transforms of the plan's length, in -> out (out may equal in), with
// count * len samples of device work space. The passes of rsw_fft_forward /
// rsw_fft_inverse run over all transforms at once: the kernels index rows,
// column batches and spectrum positions within each transform.
static rsw_status fft_batch(rsw_plan_s *p, const void *in, void *out, int64_t count, bool inverse, void *work,
                            cudaStream_t s) {
    const int64_t total = count * p->n;
    PassArgs a = base_args(p);
    a.n = total;
    cudaError_t e;
    if (!inverse) {
        a.in = in;
        a.out = work;
        if (p->log_n1 > 0) {
            a.flags = PF_FWD | PF_TW;
            CHECK(run_col(p, a, s));
            a.in = work;
            if (p->three()) CHECK(run_mid(p, a, true, s));
        }
        PassArgs r = row_level(p, a);
        r.flags = PF_FWD | row_tw(p, true, false);
        CHECK(run_row(p, r, s));
        e = launch_spec_to_natural(work, out, total, spec_levels(p), p->dbl(), s);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
        return RSW_OK;
    }
    e = launch_natural_to_spec(in, work, total, spec_levels(p), p->dbl(), s);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
    a.in = work;
    if (p->log_n1 > 0) {
        PassArgs r = row_level(p, a);
        r.out = work;
        r.flags = PF_SPEC_IN | PF_INV | row_tw(p, false, true);
        CHECK(run_row(p, r, s));
        a.out = work;
        if (p->three()) CHECK(run_mid(p, a, false, s));
        a.out = out;
        a.flags = col_inv(p);
        CHECK(run_col(p, a, s));
    } else {
        a.out = out;
        a.flags = PF_SPEC_IN | PF_INV | PF_SCALE;
        CHECK(run_row(p, a, s));
    }
    return RSW_OK;
}

// The four-step of big-fourier's out-of-core fft (big-fourier/src/bfft.rs:27-100):
// x as q rows x r columns (q = 2^floor(l/2), r = 2^ceil(l/2), split_sizes,
// bfft.rs:11-24); column transforms of length q with the twiddle
// W_N^(j k1), then row transforms of length r, X[k1 + q k2]. The host arrays
// stream through device slabs: column slabs arrive by 2-D copies and are
// transposed on the device; step 1 writes its transforms contiguously to the
// scratch array (transform j at j q); step 2 gathers q-strided slabs of it and
// writes the result with q-strided 2-D copies.
rsw_status rsw_fft_host(const void *h_in, void *h_out, void *h_scratch, int64_t n, int dtype, int inverse,
                        int64_t device_bytes, void *stream) {
    if (!h_in || !h_out) return fail(RSW_ERR_INVALID, "NULL argument");
    if (dtype != RSW_C128 && dtype != RSW_C64) return fail(RSW_ERR_INVALID, "unknown dtype %d", dtype);
    if (n < 256 || (n & (n - 1)) != 0)
        return fail(RSW_ERR_UNSUPPORTED, "N = %lld: the out-of-core FFT takes powers of two >= 256", (long long)n);
    void *h_y = h_scratch ? h_scratch : h_out;
    if (h_y == h_in) return fail(RSW_ERR_INVALID, "the scratch array (or out, without one) must not be the input");
    int lg = 0;
    while ((int64_t(1) << lg) < n) ++lg;
    const int lq = lg / 2, lr = lg - lq;
    const int64_t q = int64_t(1) << lq, r = int64_t(1) << lr;
    const size_t el = dtype == RSW_C128 ? 16 : 8;
    // two pipelines of three slabs each, on the caller's stream and a second
    // one: consecutive slabs alternate, so that one slab's upload, transforms
    // and download overlap the other's
    int64_t slab = n;  // samples per device slab
    while (slab > r && int64_t(6) * slab * int64_t(el) > device_bytes) slab >>= 1;
    if (int64_t(6) * slab * int64_t(el) > device_bytes)
        return fail(RSW_ERR_INVALID, "device_bytes = %lld: at least 6 * 2^%d samples (%lld bytes) are needed",
                    (long long)device_bytes, lr, (long long)(6 * r * int64_t(el)));
    rsw_plan pq = nullptr, pr = nullptr;
    CHECK(rsw_plan_create(&pq, q, dtype));
    std::unique_ptr<rsw_plan_s, rsw_status (*)(rsw_plan)> gq(pq, rsw_plan_destroy);
    CHECK(rsw_plan_create(&pr, r, dtype));
    std::unique_ptr<rsw_plan_s, rsw_status (*)(rsw_plan)> gr(pr, rsw_plan_destroy);
    DevBuf A[2], B[2], W[2];
    for (int k = 0; k < 2; ++k) {
        CHECK(A[k].alloc(size_t(slab) * el));
        CHECK(B[k].alloc(size_t(slab) * el));
        CHECK(W[k].alloc(size_t(slab) * el));
    }
    const bool dbl = dtype == RSW_C128, inv = inverse != 0;
    cudaStream_t st[2] = {(cudaStream_t)stream, nullptr};
    CU(cudaStreamCreateWithFlags(&st[1], cudaStreamNonBlocking));
    std::unique_ptr<CUstream_st, cudaError_t (*)(cudaStream_t)> g1(st[1], cudaStreamDestroy);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto &e : ev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    std::unique_ptr<CUevent_st, cudaError_t (*)(cudaEvent_t)> ge0(ev[0], cudaEventDestroy), ge1(ev[1], cudaEventDestroy);
    // both streams start after the caller's prior work and meet between the steps
    auto join = [&]() -> rsw_status {
        CU(cudaEventRecord(ev[0], st[0]));
        CU(cudaEventRecord(ev[1], st[1]));
        CU(cudaStreamWaitEvent(st[1], ev[0], 0));
        CU(cudaStreamWaitEvent(st[0], ev[1], 0));
        return RSW_OK;
    };
    CHECK(join());
    const char *in_b = static_cast<const char *>(h_in);
    char *y_b = static_cast<char *>(h_y), *out_b = static_cast<char *>(h_out);
    // step 1: columns j0 .. j0 + c of x (q x r)
    const int64_t c = std::min(r, slab / q);
    for (int64_t j0 = 0, k = 0; j0 < r; j0 += c, k ^= 1) {
        cudaStream_t s = st[k];
        CU(cudaMemcpy2DAsync(A[k].p, c * el, in_b + j0 * el, r * el, c * el, q, cudaMemcpyHostToDevice, s));
        CU(launch_transpose(A[k].p, B[k].p, q, c, dbl, s));
        CHECK(fft_batch(pq, B[k].p, B[k].p, c, inv, W[k].p, s));
        CU(launch_ooc_twiddle(B[k].p, c, lq, j0, lg, inv, dbl, s));
        CU(cudaMemcpyAsync(y_b + j0 * q * el, B[k].p, size_t(c * q) * el, cudaMemcpyDeviceToHost, s));
    }
    CHECK(join());
    // step 2: frequencies k0 .. k0 + t of the r transforms (r x q in the scratch array)
    const int64_t t = std::min(q, slab / r);
    for (int64_t k0 = 0, k = 0; k0 < q; k0 += t, k ^= 1) {
        cudaStream_t s = st[k];
        CU(cudaMemcpy2DAsync(A[k].p, t * el, y_b + k0 * el, q * el, t * el, r, cudaMemcpyHostToDevice, s));
        CU(launch_transpose(A[k].p, B[k].p, r, t, dbl, s));
        CHECK(fft_batch(pr, B[k].p, B[k].p, t, inv, W[k].p, s));
        CU(launch_transpose(B[k].p, A[k].p, t, r, dbl, s));
        CU(cudaMemcpy2DAsync(out_b + k0 * el, q * el, A[k].p, t * el, t * el, r, cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(st[1]));
    CU(cudaStreamSynchronize(st[0]));
    return RSW_OK;
}

rsw_status rsw_propagate(rsw_plan p, void *u, void *U, double dx, double wl, double dz, double cutoff_freq,
                         int skip_fft, void *stream) {
    if (!p || !u) return fail(RSW_ERR_INVALID, "NULL argument");
    if (skip_fft && !U) return fail(RSW_ERR_INVALID, "skip_fft needs the spectrum U");
    if (!(dx > 0) || !(wl > 0)) return fail(RSW_ERR_INVALID, "dx and wl must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    PassArgs a = base_args(p);
    a.pr = make_prop(p->n, dx, wl, dz, cutoff_freq, dz != 0.0, p->prop_mode == RSW_PROP_EXACT);
    if (p->blue) return blue_propagate(p, u, U, a.pr, skip_fft != 0, s);
    const bool two = p->log_n1 > 0;
    if (two && a.pr.has_h && !a.pr.exact) {
        CHECK(p->h3_call.alloc(size_t(int64_t(1) << p->log_nr) * 16));  // 16-byte entries
        CHECK(prepare_chirp(p, a.pr, p->h3_call.p, s));
    }
    a.in = u;
    a.out = u;
    // 1. spectrum of u in the internal layout, in place in u
    if (skip_fft) {
        cudaError_t e = to_spec(p, U, u, s);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
    } else if (two) {
        PassArgs c = a;
        c.pr = PropArgs{};
        c.flags = PF_FWD | PF_TW;
        CHECK(run_col(p, c, s));
        if (p->three()) CHECK(run_mid(p, c, true, s));
    }
    PassArgs r = two ? row_level(p, a) : a;
    if (U) {
        // 2a. forward row level + transfer function, spectrum out; copy to U in natural order
        r.flags = skip_fft ? PF_SPEC_IN : (PF_FWD | row_tw(p, true, false));
        CHECK(run_row(p, r, s));
        cudaError_t e = to_natural(p, u, U, s);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reorder: %s", cudaGetErrorString(e));
        r.pr.has_h = 0;
        r.pr.has_cut = 0;
        r.flags = PF_SPEC_IN | PF_INV | (two ? row_tw(p, false, true) : PF_SCALE);
        CHECK(run_row(p, r, s));
    } else {
        r.flags = (skip_fft ? PF_SPEC_IN : (PF_FWD | row_tw(p, true, false))) | PF_INV |
                  (two ? row_tw(p, false, true) : PF_SCALE);
        CHECK(run_row(p, r, s));
    }
    if (two) {
        a.pr = PropArgs{};
        if (p->three()) CHECK(run_mid(p, a, false, s));
        a.flags = col_inv(p);
        CHECK(run_col(p, a, s));
    }
    return RSW_OK;
}

static rsw_status grating_trans(rsw_plan_s *p, TransArgs &tr, int64_t chunk_size, double dx, double x_pos,
                                cudaStream_t stream) {
    std::vector<double> xs, st;
    chunk_coords(p->n, chunk_size, dx, x_pos, xs, st);
    for (double v : st)
        if (v == 0.0) return fail(RSW_ERR_UNSUPPORTED, "grating coordinate step underflows to zero");
    tr.half_n_floor = p->n / 2;
    if (xs.size() == 1) {
        tr.chunk_size = 0;
        tr.xstart0 = xs[0];
        tr.step0 = st[0];
    } else {
        tr.chunk_size = chunk_size;
        // the plan's chunk tables may still be read by earlier work on this stream
        CU(cudaStreamSynchronize(stream));
        CHECK(p->chunk_xs.upload(xs));
        CHECK(p->chunk_st.upload(st));
        tr.chunk_xstart = (const double *)p->chunk_xs.p;
        tr.chunk_step = (const double *)p->chunk_st.p;
    }
    return RSW_OK;
}

rsw_status rsw_apply_grating_factors(rsw_plan p, void *u, double dx, int64_t chunk_size, double pitch, double dc,
                                     double x_position, const double fa[2], const double fb[2], void *stream) {
    if (!p || !u || !fa || !fb) return fail(RSW_ERR_INVALID, "NULL argument");
    if (!(pitch > 0)) return fail(RSW_ERR_INVALID, "pitch must be positive");
    TransArgs tr{};
    tr.kind = TR_GRATING;
    tr.pitch0 = pitch;
    tr.inv_pitch0 = 1.0 / pitch;
    tr.dc0 = dc;
    tr.half_dc0 = dc / 2;
    tr.fa = make_double2(fa[0], fa[1]);
    tr.fb = make_double2(fb[0], fb[1]);
    CHECK(grating_trans(p, tr, chunk_size, dx, x_position, (cudaStream_t)stream));
    cudaError_t e = launch_trans(u, p->n, tr, p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "grating: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_apply_dba_grating_factors(rsw_plan p, void *u, double dx, int64_t chunk_size, double pitch0,
                                         double pitch1, double dc0, double dc1, double x_position,
                                         const double fa[2], const double fb[2], void *stream) {
    if (!p || !u || !fa || !fb) return fail(RSW_ERR_INVALID, "NULL argument");
    if (!(pitch0 > 0) || !(pitch1 > 0)) return fail(RSW_ERR_INVALID, "pitches must be positive");
    TransArgs tr{};
    tr.kind = TR_DBA;
    tr.pitch0 = pitch0;
    tr.pitch1 = pitch1;
    tr.inv_pitch0 = 1.0 / pitch0;
    tr.inv_pitch1 = 1.0 / pitch1;
    tr.dc0 = dc0;
    tr.half_dc0 = dc0 / 2;
    tr.dc1 = dc1;
    tr.fa = make_double2(fa[0], fa[1]);
    tr.fb = make_double2(fb[0], fb[1]);
    CHECK(grating_trans(p, tr, chunk_size, dx, x_position, (cudaStream_t)stream));
    cudaError_t e = launch_trans(u, p->n, tr, p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "dba grating: %s", cudaGetErrorString(e));
    return RSW_OK;
}

// Sample row: the row's deltabeta values are turned into a per-pixel material
// table (each distinct value becomes one "material"), so the device code is
// the same as for a grid row.
static rsw_status sample_trans(rsw_plan_s *p, TransArgs &tr, double dx, double wl, double dz, double psx,
                               double x_pos, int64_t x_len, const int8_t *grid_row_host,
                               const std::vector<cplx> &mat_db /* [0] = vacuum */) {
    if (x_len < 2) return fail(RSW_ERR_UNSUPPORTED, "sample rows need at least 2 pixels");
    if (!(psx > 0)) return fail(RSW_ERR_INVALID, "pixel_size_x must be positive");
    tr.kind = TR_SAMPLE;
    tr.dx = dx;
    tr.half_n = double(p->n) / 2.0;
    tr.psx = psx;
    tr.sample_xpos = x_pos;
    tr.sample_hw = (double(x_len) * psx) * 0.5;
    tr.sample_inv_psx = 1.0 / psx;
    tr.x_len = x_len;
    tr.sample_y = (2.0 * M_PI * dz) / wl;
    std::vector<double> db, fac;
    for (const cplx &d : mat_db) {
        db.push_back(d.real());
        db.push_back(d.imag());
        const cplx f = material_factor(d.real(), d.imag(), dz, wl);
        fac.push_back(f.real());
        fac.push_back(f.imag());
    }
    CHECK(p->sample_db.upload(db));
    CHECK(p->sample_fac.upload(fac));
    CHECK(p->sample_grid.alloc(size_t(x_len)));
    CU(cudaMemcpy(p->sample_grid.p, grid_row_host, size_t(x_len), cudaMemcpyHostToDevice));
    tr.row_grid = (const int8_t *)p->sample_grid.p;
    tr.mat_db = (const double2 *)p->sample_db.p;
    tr.mat_factor = (const double2 *)p->sample_fac.p;
    return RSW_OK;
}

rsw_status rsw_apply_sample_row(rsw_plan p, void *u, double dx, double wl, double dz, double psx, double x_pos,
                                int64_t x_len, const double *h_row_db, void *stream) {
    if (!p || !u || !h_row_db) return fail(RSW_ERR_INVALID, "NULL argument");
    if (x_len > 127 * 1024 * 1024) return fail(RSW_ERR_INVALID, "row too long");
    // distinct values -> material indices (0 = vacuum)
    std::vector<cplx> mats{cplx(0, 0)};
    std::vector<int8_t> grid(size_t(std::max<int64_t>(x_len, 0)));
    for (int64_t j = 0; j < x_len; ++j) {
        const cplx d(h_row_db[2 * j], h_row_db[2 * j + 1]);
        size_t m = 0;
        while (m < mats.size() && !(mats[m] == d)) ++m;
        if (m == mats.size()) {
            if (mats.size() >= 127) return fail(RSW_ERR_UNSUPPORTED, "more than 126 distinct values in a row");
            mats.push_back(d);
        }
        grid[j] = int8_t(m);
    }
    TransArgs tr{};
    // the plan's row buffers may still be read by earlier work on this stream
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    CHECK(sample_trans(p, tr, dx, wl, dz, psx, x_pos, x_len, grid.data(), mats));
    cudaError_t e = launch_trans(u, p->n, tr, p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "sample: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_scale(rsw_plan p, void *u, const double f[2], void *stream) {
    if (!p || !u || !f) return fail(RSW_ERR_INVALID, "NULL argument");
    TransArgs tr{};
    tr.kind = TR_SCALAR;
    tr.fa = make_double2(f[0], f[1]);
    cudaError_t e = launch_trans(u, p->n, tr, p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "scale: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_point_source(rsw_plan p, void *u, double dx, double wl, double z, double x_src, void *stream) {
    if (!p || !u) return fail(RSW_ERR_INVALID, "NULL argument");
    const double w = (-2.0 * M_PI) / wl;
    cudaError_t e = launch_point_source(u, p->n, dx, w, z, x_src, p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "point source: %s", cudaGetErrorString(e));
    return RSW_OK;
}

static rsw_status plan_detector(rsw_plan_s *p, double dx, double det, double psx, double z) {
    const double key[5] = {dx, det, psx, z, double(p->n)};
    if (p->det_npix >= 0 && std::memcmp(key, p->det_key, sizeof key) == 0) return RSW_OK;
    DetectorGeom g;
    CHECK(detector_geom(p->n, dx, det, psx, z, g));
    CHECK(p->det_bounds.upload(g.bounds));
    CHECK(p->det_cos.upload(g.cosv));
    CHECK(p->det_r.upload(g.rv));
    std::memcpy(p->det_key, key, sizeof key);
    p->det_npix = g.n_pix;
    return RSW_OK;
}

rsw_status rsw_square_and_downsample(rsw_plan p, const void *u, double dx, double det, double psx, double psy,
                                     double z, double *out, int64_t *n_pix_out, void *stream) {
    if (!p) return fail(RSW_ERR_INVALID, "plan is NULL");
    CHECK(plan_detector(p, dx, det, psx, z));
    if (n_pix_out) *n_pix_out = p->det_npix;
    if (!out) return n_pix_out ? RSW_OK : fail(RSW_ERR_INVALID, "out is NULL");
    if (!u) return fail(RSW_ERR_INVALID, "u is NULL");
    cudaError_t e = launch_detect(u, (const int64_t *)p->det_bounds.p, (const double *)p->det_cos.p,
                                  (const double *)p->det_r.p, p->det_npix, dx, psy, out, nullptr, nullptr, 0.0,
                                  p->dbl(), (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "detect: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_detector_geometry(int64_t n, double dx, double det, double psx, double z, int64_t *n_pix,
                                 int64_t *bounds, double *cosv, double *rv) {
    if (!n_pix) return fail(RSW_ERR_INVALID, "n_pix is NULL");
    if (n < 1) return fail(RSW_ERR_INVALID, "n must be positive");
    DetectorGeom g;
    CHECK(detector_geom(n, dx, det, psx, z, g));
    *n_pix = g.n_pix;
    if (bounds) std::copy(g.bounds.begin(), g.bounds.end(), bounds);
    if (cosv) std::copy(g.cosv.begin(), g.cosv.end(), cosv);
    if (rv) std::copy(g.rv.begin(), g.rv.end(), rv);
    return RSW_OK;
}

rsw_status rsw_signal_retrieval(const double *d_data, int64_t n_pix, int nsteps, double period, double *d_abs,
                                double *d_phase, double *d_vis, double *d_chi2, void *stream) {
    if (!d_data) return fail(RSW_ERR_INVALID, "d_data is NULL");
    if (n_pix < 0) return fail(RSW_ERR_INVALID, "n_pix < 0");
    if (nsteps < 3 || nsteps > RSW_RETRIEVAL_MAX)
        return fail(RSW_ERR_INVALID, "nsteps = %d: need 3 <= nsteps <= %d", nsteps, RSW_RETRIEVAL_MAX);
    if (!(period > 0)) return fail(RSW_ERR_INVALID, "period must be positive");
    // design matrix [sin, cos, 1] at phi_k = k * step, step = (2 pi nsteps / period) / nsteps
    RetrievalArgs r{};
    r.k = nsteps;
    const double step = (2.0 * M_PI * double(nsteps) / period) / double(nsteps);
    long double g[3][3] = {{0}};
    for (int k = 0; k < nsteps; ++k) {
        const double phi = double(k) * step;
        r.sn[k] = std::sin(phi);
        r.cs[k] = std::cos(phi);
        const long double m[3] = {r.sn[k], r.cs[k], 1.0L};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) g[i][j] += m[i] * m[j];
    }
    // pseudo-inverse (M^T M)^-1 M^T from the adjugate of the 3 x 3 Gram matrix
    long double inv[3][3];
    inv[0][0] = g[1][1] * g[2][2] - g[1][2] * g[2][1];
    inv[0][1] = g[0][2] * g[2][1] - g[0][1] * g[2][2];
    inv[0][2] = g[0][1] * g[1][2] - g[0][2] * g[1][1];
    inv[1][0] = g[1][2] * g[2][0] - g[1][0] * g[2][2];
    inv[1][1] = g[0][0] * g[2][2] - g[0][2] * g[2][0];
    inv[1][2] = g[0][2] * g[1][0] - g[0][0] * g[1][2];
    inv[2][0] = g[1][0] * g[2][1] - g[1][1] * g[2][0];
    inv[2][1] = g[0][1] * g[2][0] - g[0][0] * g[2][1];
    inv[2][2] = g[0][0] * g[1][1] - g[0][1] * g[1][0];
    const long double det = g[0][0] * inv[0][0] + g[0][1] * inv[1][0] + g[0][2] * inv[2][0];
    if (!(std::fabs(double(det)) > 1e-12)) return fail(RSW_ERR_INVALID, "phase steps do not determine the fit");
    for (int k = 0; k < nsteps; ++k) {
        const long double m[3] = {r.sn[k], r.cs[k], 1.0L};
        for (int i = 0; i < 3; ++i) {
            long double acc = 0;
            for (int j = 0; j < 3; ++j) acc += inv[i][j] * m[j];
            r.p[i * RSW_RETRIEVAL_MAX + k] = double(acc / det);
        }
    }
    cudaError_t e = launch_retrieval(d_data, n_pix, r, d_abs, d_phase, d_vis, d_chi2, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "signal retrieval: %s", cudaGetErrorString(e));
    return RSW_OK;
}

}  // extern "C"

// ============================================================ simulations
struct SimElement {
    rsw_element d{};
    std::vector<double> x_positions;
    std::vector<int8_t> grid;
    DevBuf grid_dev;
    // grating chunk tables per phase-step position (when several chunks)
    std::vector<std::unique_ptr<DevBuf>> chunk_xs, chunk_st;
    std::vector<double> xs0, st0;  // single-chunk values per position
    int64_t steps() const {
        return d.type == RSW_EL_SAMPLE ? d.grid_z : int64_t(d.nr_steps) + (d.substrate_thickness > 0 ? 1 : 0);
    }
    double total_thickness() const {
        return d.type == RSW_EL_SAMPLE ? d.pixel_size_z * double(d.grid_z) : d.thickness + d.substrate_thickness;
    }
};

// transfer-function tables of one (dz, cutoff) for the instances of a batch
struct BatchPropTables {
    DevBuf entries, h3;
    std::vector<BatchProp> host;
    bool any_cut = false;
};

struct rsw_sim_s {
    rsw_plan_s *plan = nullptr;
    rsw_sim_desc d{};
    std::vector<SimElement> els;
    std::vector<double> cutoff_angles;
    int64_t nr_phase_steps = 1;
    int snap_el = -1;
    DetectorGeom geom;
    DevBuf bounds, cosv, rv;
    DevBuf acc, comp;
    DevBuf dsum;  // fused detection: n_pix raw sums, then the CTA counter (kept zero between passes)
    DevBuf buf[2];
    DevBuf mat_db, mat_fac;  // per-run sample material tables
    std::vector<std::unique_ptr<DevBuf>> h3_pool;  // chirp tables, one per distinct dz of a run
    int last_field = -1;
    TimingLog tl;
    int64_t split_steps = 0;
    // history recording (big-wave/history.py): detector images at the z
    // points of the first phase-step pass, stored [entry][n_pix] on the device
    double hist_dz = 0.0;
    DevBuf hbuf;  // third field buffer: history views and intermediate points
    DevBuf hist, hist_cos, hist_r;
    int64_t hist_cap = 0;
    std::vector<double> hist_z;
    // keypoints (big-wave/wavesim.py:35-55): caller buffers for the field
    // before / after each element of the first pass, NULL entries skipped
    std::vector<void *> keypoints;
    // final fields (big-wave's save_u): caller buffers for the field at the
    // detector of each phase step, NULL entries skipped
    std::vector<void *> final_fields;
    // lockstep batches (rsw_sim_run_batch), sized for the largest batch so far:
    // field buffers of nb * N samples, per-instance transmission entries
    // [element][grating, substrate][instance], sample material tables
    // [instance][element][128], transfer-function tables per (dz, cutoff),
    // detector sums [instance][sum_stride] then the CTA counter, weights
    int64_t batch_cap = 0;
    DevBuf bbuf[2], btab, bmat_db, bmat_fac, bsum, bweight;
    std::vector<std::unique_ptr<BatchPropTables>> bprop;
    ~rsw_sim_s() { rsw_plan_destroy(plan); }
};

// z offsets of big-wave's propagate_with_history (big-wave/history.py:90-97):
// np.arange(0, dz, hdz), the last one moved to dz when closer than hdz / 2,
// else dz appended
static std::vector<double> history_zs(double dz, double hdz) {
    const int64_t len = std::max<int64_t>(int64_t(std::ceil(dz / hdz)), 0);
    std::vector<double> zs;
    for (int64_t i = 0; i < len; ++i) zs.push_back(double(i) * hdz);
    if (zs.empty()) zs.push_back(0.0);
    if (dz - zs.back() < hdz / 2.0 && zs.size() > 1)
        zs.back() = dz;
    else
        zs.push_back(dz);
    return zs;
}

namespace {

struct Runner {
    rsw_sim_s *S;
    rsw_plan_s *P;
    cudaStream_t st;
    double wl;
    std::vector<double> cut;
    // field state
    int cur = 0;            // buffer index holding the field (or -1 when plane_pending)
    bool mid = false;       // field in the row-pass ("mid") representation
    bool ones = false;      // field is the plane wave u = 1, not yet materialised
    int readonly = -1;      // buffer that must not be written (snapshot)
    // per-run material factors: per element [fa? ...]
    std::vector<std::vector<cplx>> db;  // deltabeta per element (gratings: a,b,sub; samples: materials 1..)
    std::vector<double> chirp_dz;       // dz of each built chirp table of this run (slot = index)
    // Lockstep batches (rsw_sim_run_batch): nb instances of the same field
    // length in consecutive N-sample slices of the batch buffers; instance 0's
    // values stand in the common arguments, the wavelength-dependent ones of
    // every instance come from device tables
    int nb = 1;
    DevBuf *fbuf = nullptr;                // field buffers: the sim's own, or its batch buffers
    std::vector<double> wls;               // wavelength per instance
    std::vector<std::vector<double>> cuts; // cutoff frequency per instance and cutoff index
    const BatchTrans *btr = nullptr;       // entries of the element being applied
    std::vector<std::pair<double, int>> prop_keys;  // (dz, cutoff index) of each transfer-function table
    // optional: each source's own detector values (unweighted), instance b's
    // [phase][pix] at each + b * nr_phase_steps * n_pix
    double *each = nullptr;

    // chirp table for a distance dz at this run's wavelength (built on first use)
    rsw_status chirp_for(PropArgs &pr, double dz) {
        if (P->log_n1 == 0 || !pr.has_h || pr.exact) return RSW_OK;
        size_t slot = 0;
        while (slot < chirp_dz.size() && chirp_dz[slot] != dz) ++slot;
        const bool fresh = slot == chirp_dz.size();
        if (fresh) {
            chirp_dz.push_back(dz);
            if (S->h3_pool.size() <= slot) S->h3_pool.emplace_back(new DevBuf());
            CHECK(S->h3_pool[slot]->alloc(size_t(int64_t(1) << P->log_nr) * 16));  // 16-byte entries
            CHECK(prepare_chirp(P, pr, S->h3_pool[slot]->p, st));
            return RSW_OK;
        }
        double g_hi, g_lo;
        chirp_constant(pr, P->n, &g_hi, &g_lo);
        pr.chirp = 1;
        pr.g_hi = g_hi;
        pr.g_lo = g_lo;
        pr.h3 = S->h3_pool[slot]->p;
        return RSW_OK;
    }

    int target() const {
        if (cur < 0) return readonly == 0 ? 1 : 0;
        return cur == readonly ? 1 - cur : cur;
    }
    // field buffers 0 and 1 hold the state; 2 is the history buffer
    void *bp(int i) const { return i == 2 ? S->hbuf.p : fbuf[i].p; }

    // batch: the instances' transmission entries of element ei (sub 0: the
    // grating or sample, 1: the substrate)
    const BatchTrans *btab_at(int ei, int sub) const {
        return static_cast<const BatchTrans *>(S->btab.p) + (size_t(ei) * 2 + size_t(sub)) * size_t(nb);
    }
    // batch: the instances' transfer functions of a split step over dz with
    // cutoff ci (built on first use in a run: the scalars of make_prop and
    // chirp_constant per instance and one chirp table each); pr keeps
    // instance 0's common values and covers every instance's cutoff
    rsw_status batch_prop(PropArgs &pr, double dz, int ci, const BatchProp **out) {
        size_t slot = 0;
        while (slot < prop_keys.size() && !(prop_keys[slot].first == dz && prop_keys[slot].second == ci)) ++slot;
        const bool chirp = pr.has_h && !pr.exact;
        const size_t nr = size_t(1) << P->log_nr;
        if (slot == prop_keys.size()) {
            prop_keys.emplace_back(dz, ci);
            if (S->bprop.size() <= slot) S->bprop.emplace_back(new BatchPropTables());
            BatchPropTables &t = *S->bprop[slot];
            CHECK(t.entries.alloc(size_t(nb) * sizeof(BatchProp)));
            if (chirp) CHECK(t.h3.alloc(size_t(nb) * nr * 16));
            t.host.assign(size_t(nb), BatchProp{});
            t.any_cut = false;
            for (int b = 0; b < nb; ++b) {
                PropArgs q = make_prop(P->n, S->d.dx, wls[size_t(b)], dz, cuts[size_t(b)][size_t(ci)], dz != 0.0);
                BatchProp &e = t.host[size_t(b)];
                e.A = q.A;
                if (q.has_cut) {
                    e.cut_lo = q.cut_lo;
                    e.cut_hi = q.cut_hi;
                    t.any_cut = true;
                }
                if (chirp) {
                    void *h3 = static_cast<char *>(t.h3.p) + size_t(b) * nr * 16;
                    CHECK(prepare_chirp(P, q, h3, st));
                    e.g_hi = q.g_hi;
                    e.g_lo = q.g_lo;
                    e.h3 = h3;
                }
            }
            // pageable source: staged before the call returns
            CU(cudaMemcpyAsync(t.entries.p, t.host.data(), t.host.size() * sizeof(BatchProp), cudaMemcpyHostToDevice,
                               st));
        }
        const BatchPropTables &t = *S->bprop[slot];
        pr.has_cut = t.any_cut ? 1 : 0;
        if (chirp) pr.chirp = 1;
        *out = static_cast<const BatchProp *>(t.entries.p);
        return RSW_OK;
    }

    rsw_status split_step(const TransArgs &tr, double dz, int ci) { return step_to(tr, dz, ci, target(), true); }

    // One split step from the current state into buffer dst; commit = false
    // leaves the state untouched (history points reached from a gap start).
    // ci: the cutoff's index (the element the step belongs to, 0 before the
    // first one).
    rsw_status step_to(const TransArgs &tr, double dz, int ci, int dst, bool commit) {
        PassArgs a = base_args(P);
        a.tr = tr;
        a.pr = make_prop(P->n, S->d.dx, wl, dz, cut[size_t(ci)], dz != 0.0, P->prop_mode == RSW_PROP_EXACT);
        if (nb > 1) {
            a.n = P->n * nb;
            CHECK(batch_prop(a.pr, dz, ci, &a.bpr));
            a.btr = tr.kind != TR_NONE ? btr : nullptr;
        } else {
            CHECK(chirp_for(a.pr, dz));
        }
        a.in = ones ? nullptr : bp(cur);
        a.out = bp(dst);
        bool now_mid = false;
        if (P->blue) {
            // any length: transmission and propagate on the natural-order field
            void *d = bp(dst);
            cudaError_t e = cudaSuccess;
            if (ones) e = launch_fill_ones(d, P->n, P->dbl(), st);
            else if (cur != dst)
                e = cudaMemcpyAsync(d, bp(cur), size_t(P->n) * P->elem(), cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess && tr.kind != TR_NONE) e = launch_trans(d, P->n, tr, P->dbl(), st);
            if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "split step: %s", cudaGetErrorString(e));
            CHECK(blue_propagate(P, d, nullptr, a.pr, false, st));
        } else {
            CHECK(launch_split_step(P, a, mid, ones, st, &S->tl, &now_mid));
        }
        if (commit) {
            cur = dst;
            ones = false;
            mid = now_mid;
        }
        S->split_steps += nb;
        return RSW_OK;
    }

    // ---------------------------------------------------------- history
    bool hist_on = false;

    rsw_status hist_reserve() {
        const int64_t np = S->geom.n_pix;
        const int64_t n = int64_t(S->hist_z.size());
        if (n < S->hist_cap) return RSW_OK;
        const int64_t cap = std::max<int64_t>(64, 2 * S->hist_cap);
        const size_t bytes = size_t(cap * std::max<int64_t>(np, 1)) * sizeof(double);
        DevBuf nb, nc, nr;  // images, and per-entry cos / r of the detector geometry
        CHECK(nb.alloc(bytes));
        CHECK(nc.alloc(bytes));
        CHECK(nr.alloc(bytes));
        if (n > 0) CU(cudaMemcpyAsync(nb.p, S->hist.p, size_t(n * np) * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CU(cudaStreamSynchronize(st));  // the old buffers are freed below
        S->hist = std::move(nb);
        S->hist_cos = std::move(nc);
        S->hist_r = std::move(nr);
        S->hist_cap = cap;
        return RSW_OK;
    }
    // detector image of a natural-order field at z (square_and_downsample)
    rsw_status hist_detect(const void *field, double z) {
        CHECK(hist_reserve());
        DetectorGeom g;
        CHECK(detector_geom(P->n, S->d.dx, S->d.detector_size, S->d.pixel_size_x, z, g));
        const int64_t off = int64_t(S->hist_z.size()) * S->geom.n_pix;
        double *cosv = (double *)S->hist_cos.p + off, *rv = (double *)S->hist_r.p + off;
        // pageable sources: the copies are staged before the calls return
        CU(cudaMemcpyAsync(cosv, g.cosv.data(), g.cosv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(rv, g.rv.data(), g.rv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        double *out = (double *)S->hist.p + off;
        cudaError_t e = launch_detect(field, (const int64_t *)S->bounds.p, cosv, rv, S->geom.n_pix, S->d.dx,
                                      S->d.pixel_size_y, out, nullptr, nullptr, 1.0, P->dbl(), st);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "history detect: %s", cudaGetErrorString(e));
        S->hist_z.push_back(z);
        return RSW_OK;
    }
    // history entry of the current state at z
    rsw_status hist_push(double z) {
        if (ones) {
            cudaError_t e = launch_fill_ones(bp(2), P->n, P->dbl(), st);
            if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "fill: %s", cudaGetErrorString(e));
            return hist_detect(bp(2), z);
        }
        if (mid) {
            PassArgs a = base_args(P);
            a.in = bp(cur);
            a.out = bp(2);
            a.flags = col_inv(P);
            CHECK(run_col(P, a, st, &S->tl));
            return hist_detect(bp(2), z);
        }
        return hist_detect(bp(cur), z);
    }
    // host-computed entry (analytic point-source history)
    rsw_status hist_host(const std::vector<double> &img, double z) {
        CHECK(hist_reserve());
        double *out = (double *)S->hist.p + int64_t(S->hist_z.size()) * S->geom.n_pix;
        if (!img.empty()) CU(cudaMemcpyAsync(out, img.data(), img.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        CU(cudaStreamSynchronize(st));  // img is a temporary
        S->hist_z.push_back(z);
        return RSW_OK;
    }
    // propagate_with_history (big-wave/history.py:67-135): every history point
    // is reached from the state at the start of the gap; the last one is the
    // gap's own propagation
    rsw_status gap(double dz, int ci, double z_from) {
        if (dz == 0.0) return RSW_OK;
        if (!hist_on) return split_step(TransArgs{}, dz, ci);
        const std::vector<double> zs = history_zs(dz, S->hist_dz);
        for (size_t i = 1; i + 1 < zs.size(); ++i) {
            CHECK(step_to(TransArgs{}, zs[i] - zs[0], ci, 2, false));
            if (P->log_n1 > 0) {  // "mid" -> natural, in place
                PassArgs a = base_args(P);
                a.in = bp(2);
                a.out = bp(2);
                a.flags = col_inv(P);
                CHECK(run_col(P, a, st, &S->tl));
            }
            CHECK(hist_detect(bp(2), zs[i] + z_from));
        }
        CHECK(split_step(TransArgs{}, zs.back() - zs[0], ci));
        return hist_push(zs.back() + z_from);
    }

    // save_keypoint (big-wave/wavesim.py:35-55): the current field in natural
    // order into a caller buffer; the state is left as it is
    rsw_status keypoint(void *dst) {
        if (!dst) return RSW_OK;
        cudaError_t e = cudaSuccess;
        if (ones) {
            e = launch_fill_ones(dst, P->n, P->dbl(), st);
        } else if (mid) {
            PassArgs a = base_args(P);
            a.in = bp(cur);
            a.out = dst;
            a.flags = col_inv(P);
            return run_col(P, a, st);
        } else {
            e = cudaMemcpyAsync(dst, bp(cur), size_t(P->n) * P->elem(), cudaMemcpyDeviceToDevice, st);
        }
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "keypoint: %s", cudaGetErrorString(e));
        return RSW_OK;
    }

    rsw_status finalize() {
        if (ones) {
            const int dst = target();
            cudaError_t e = launch_fill_ones(S->buf[dst].p, P->n, P->dbl(), st);
            if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "fill: %s", cudaGetErrorString(e));
            cur = dst;
            ones = false;
            mid = false;
        }
        if (mid) {
            const int dst = target();
            PassArgs a = base_args(P);
            a.in = S->buf[cur].p;
            a.out = S->buf[dst].p;
            a.flags = col_inv(P);
            CHECK(run_col(P, a, st, &S->tl));
            cur = dst;
            mid = false;
        }
        return RSW_OK;
    }

    // The end of a phase step: the field's last inverse column pass with the
    // detector binning fused in (the field is written only when `keep`, for
    // the final field of a run); the plain inverse and the binning kernel
    // where the field is not in the multi-level "mid" representation.
    rsw_status finish_phase(int64_t phase, double weight, bool keep) {
        const int64_t np = S->geom.n_pix;
        // the caller's buffer for this phase step's final field, if any
        void *fin = size_t(phase) < S->final_fields.size() ? S->final_fields[size_t(phase)] : nullptr;
        if (!(mid && P->log_n1 > 0 && np > 0)) {
            CHECK(finalize());
            if (fin) CU(cudaMemcpyAsync(fin, bp(cur), size_t(P->n) * P->elem(), cudaMemcpyDeviceToDevice, st));
            return detect(phase, weight, each ? each + phase * np : nullptr);
        }
        const int dst = target();
        PassArgs a = base_args(P);
        a.n = P->n * nb;
        a.in = bp(cur);
        a.out = fin && !keep ? fin : bp(dst);
        a.flags = col_inv(P) | (keep || fin ? 0 : PF_NOSTORE);
        DetectArgs &d = a.det;
        d.bounds = (const int64_t *)S->bounds.p;
        d.cosv = (const double *)S->cosv.p;
        d.rv = (const double *)S->rv.p;
        d.n_pix = np;
        d.lo = S->geom.bounds[0];
        d.hi = S->geom.bounds[size_t(np)];
        d.inv_w = d.hi > d.lo ? double(np) / double(d.hi - d.lo) : 0.0;
        d.dx = S->d.dx;
        d.psy = S->d.pixel_size_y;
        d.weight = weight;
        d.sum = (double *)S->dsum.p;
        d.count = (unsigned *)((double *)S->dsum.p + np);
        d.acc = (double *)S->acc.p + phase * np;
        d.comp = (double *)S->comp.p + phase * np;
        if (nb > 1) {
            d.sum_stride = batch_sum_stride(np);
            d.sum = (double *)S->bsum.p;
            d.count = (unsigned *)(d.sum + nb * d.sum_stride);
            d.bweight = (const double *)S->bweight.p;
            d.n_inst = nb;
        }
        if (each) {
            d.inst_out = each + phase * np;
            d.inst_stride = S->nr_phase_steps * np;
        }
        TimingLog::Rec r{};
        if (S->tl.enabled) S->tl.begin(2, st, r);
        cudaError_t e = launch_col_detect(a, P->dbl(), P->col_e, st);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "detection pass (2^%d): %s", a.log_n1, cudaGetErrorString(e));
        if (S->tl.enabled) S->tl.end(r, st);
        if (keep) {
            cur = dst;
            mid = false;
            if (fin) CU(cudaMemcpyAsync(fin, bp(cur), size_t(P->n) * P->elem(), cudaMemcpyDeviceToDevice, st));
        }
        return RSW_OK;
    }

    // out: also the phase step's pixel values (unweighted), or NULL
    rsw_status detect(int64_t phase, double weight, double *out = nullptr) {
        TimingLog::Rec r{};
        if (S->tl.enabled) S->tl.begin(2, st, r);
        double *acc = (double *)S->acc.p + phase * S->geom.n_pix;
        double *comp = (double *)S->comp.p + phase * S->geom.n_pix;
        cudaError_t e = launch_detect(S->buf[cur].p, (const int64_t *)S->bounds.p, (const double *)S->cosv.p,
                                      (const double *)S->rv.p, S->geom.n_pix, S->d.dx, S->d.pixel_size_y, out,
                                      acc, comp, weight, P->dbl(), st);
        if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "detect: %s", cudaGetErrorString(e));
        if (S->tl.enabled) S->tl.end(r, st);
        return RSW_OK;
    }

    rsw_status apply(int ei, int64_t step, int ci) {
        SimElement &el = S->els[ei];
        const rsw_element &e = el.d;
        const std::vector<cplx> &m = db[ei];
        if (e.type == RSW_EL_GRATING || e.type == RSW_EL_DBA_GRATING) {
            const double z_step = e.thickness / double(e.nr_steps);
            const cplx fa = material_factor(m[0].real(), m[0].imag(), z_step, wl);
            const cplx fb = material_factor(m[1].real(), m[1].imag(), z_step, wl);
            for (int i = 0; i < e.nr_steps; ++i) {
                const double zf = double(i) / double(e.nr_steps);
                TransArgs tr{};
                tr.kind = e.type == RSW_EL_GRATING ? TR_GRATING : TR_DBA;
                tr.fa = make_double2(fa.real(), fa.imag());
                tr.fb = make_double2(fb.real(), fb.imag());
                tr.pitch0 = e.pitch;
                tr.pitch1 = e.pitch1;
                tr.inv_pitch0 = 1.0 / e.pitch;
                tr.inv_pitch1 = e.pitch1 > 0 ? 1.0 / e.pitch1 : 0.0;
                tr.dc0 = (1.0 - zf) * e.dc[0] + zf * e.dc[1];
                tr.half_dc0 = tr.dc0 / 2;
                tr.dc1 = (1.0 - zf) * e.dc1[0] + zf * e.dc1[1];
                if (el.chunk_xs.empty()) {
                    tr.chunk_size = 0;
                    tr.xstart0 = el.xs0[step];
                    tr.step0 = el.st0[step];
                } else {
                    tr.chunk_size = S->d.chunk_size;
                    tr.chunk_xstart = (const double *)el.chunk_xs[step]->p;
                    tr.chunk_step = (const double *)el.chunk_st[step]->p;
                }
                if (nb > 1) btr = btab_at(ei, 0);
                CHECK(split_step(tr, z_step, ci));
                if (hist_on) CHECK(hist_push(e.z_start + double(i + 1) * z_step));
            }
            if (e.substrate_thickness > 0) {
                const cplx fs = material_factor(m[2].real(), m[2].imag(), e.substrate_thickness, wl);
                TransArgs tr{};
                tr.kind = TR_SCALAR;
                tr.fa = make_double2(fs.real(), fs.imag());
                if (nb > 1) btr = btab_at(ei, 1);
                CHECK(split_step(tr, e.substrate_thickness, ci));
            }
            return RSW_OK;
        }
        // sample
        const double psz = e.pixel_size_z;
        TransArgs tr{};
        tr.kind = TR_SAMPLE;
        tr.dx = S->d.dx;
        tr.half_n = double(P->n) / 2.0;
        tr.psx = e.pixel_size_x;
        tr.sample_xpos = el.x_positions[step];
        tr.sample_hw = (double(e.grid_x) * e.pixel_size_x) * 0.5;
        tr.sample_inv_psx = 1.0 / e.pixel_size_x;
        tr.x_len = e.grid_x;
        tr.sample_y = (2.0 * M_PI * psz) / wl;
        const size_t off = size_t(ei) * 128;
        tr.mat_db = (const double2 *)S->mat_db.p + off;
        tr.mat_factor = (const double2 *)S->mat_fac.p + off;
        for (int64_t r = 0; r < e.grid_z; ++r) {
            if (hist_on) CHECK(hist_push(e.z_start + double(r) * psz));
            tr.row_grid = (const int8_t *)el.grid_dev.p + r * e.grid_x;
            if (nb > 1) btr = btab_at(ei, 0);
            CHECK(split_step(tr, psz, ci));
        }
        return RSW_OK;
    }
};

}  // namespace

extern "C" {

rsw_status rsw_sim_create(rsw_sim *out, const rsw_sim_desc *desc) {
    if (!out || !desc) return fail(RSW_ERR_INVALID, "NULL argument");
    *out = nullptr;
    if (desc->n_elements < 0 || (desc->n_elements > 0 && !desc->elements))
        return fail(RSW_ERR_INVALID, "bad element list");
    if (!desc->cutoff_angles) return fail(RSW_ERR_INVALID, "cutoff_angles is NULL");
    if (!(desc->dx > 0)) return fail(RSW_ERR_INVALID, "dx must be positive");
    std::unique_ptr<rsw_sim_s> S(new (std::nothrow) rsw_sim_s());
    if (!S) return fail(RSW_ERR_NOMEM, "host allocation failed");
    CHECK(rsw_plan_create(&S->plan, desc->n, desc->dtype));
    S->d = *desc;
    S->d.elements = nullptr;
    S->cutoff_angles.assign(desc->cutoff_angles, desc->cutoff_angles + desc->n_elements + 1);
    for (double a : S->cutoff_angles)
        if (!(a >= 0 && a <= M_PI / 2 + 1e-12)) return fail(RSW_ERR_INVALID, "cutoff angles must be in [0, pi/2]");
    const double z_tol = 1e-8;
    double last_z = 0;
    S->els.resize(desc->n_elements);
    for (int i = 0; i < desc->n_elements; ++i) {
        const rsw_element &e = desc->elements[i];
        SimElement &el = S->els[i];
        el.d = e;
        if (e.n_x_positions < 1 || !e.x_positions) return fail(RSW_ERR_INVALID, "element %d: no x_positions", i);
        el.x_positions.assign(e.x_positions, e.x_positions + e.n_x_positions);
        el.d.x_positions = nullptr;
        if (e.type == RSW_EL_GRATING || e.type == RSW_EL_DBA_GRATING) {
            if (e.nr_steps < 1 || !(e.thickness > 0) || e.substrate_thickness < 0 || !(e.pitch > 0) ||
                (e.type == RSW_EL_DBA_GRATING && !(e.pitch1 > 0)))
                return fail(RSW_ERR_INVALID, "element %d: invalid grating", i);
            const bool multi = desc->chunk_size > 0 && desc->chunk_size < desc->n;
            for (double xp : el.x_positions) {
                std::vector<double> xs, st;
                chunk_coords(desc->n, desc->chunk_size, desc->dx, xp, xs, st);
                for (double v : st)
                    if (v == 0.0) return fail(RSW_ERR_UNSUPPORTED, "grating coordinate step underflows");
                if (multi) {
                    el.chunk_xs.emplace_back(new DevBuf());
                    el.chunk_st.emplace_back(new DevBuf());
                    CHECK(el.chunk_xs.back()->upload(xs));
                    CHECK(el.chunk_st.back()->upload(st));
                } else {
                    el.xs0.push_back(xs[0]);
                    el.st0.push_back(st[0]);
                }
            }
        } else if (e.type == RSW_EL_SAMPLE) {
            if (e.grid_z < 1 || e.grid_x < 2 || !e.grid || !(e.pixel_size_x > 0) || !(e.pixel_size_z > 0))
                return fail(RSW_ERR_INVALID, "element %d: invalid sample", i);
            if (e.n_materials < 0 || e.n_materials > 126) return fail(RSW_ERR_INVALID, "element %d: materials", i);
            el.grid.assign(e.grid, e.grid + size_t(e.grid_z * e.grid_x));
            for (int8_t g : el.grid)
                if (g < 0 || g > e.n_materials) return fail(RSW_ERR_INVALID, "element %d: grid index %d", i, int(g));
            el.d.grid = nullptr;
            CHECK(el.grid_dev.alloc(el.grid.size()));
            CU(cudaMemcpy(el.grid_dev.p, el.grid.data(), el.grid.size(), cudaMemcpyHostToDevice));
        } else {
            return fail(RSW_ERR_INVALID, "element %d: unknown type %d", i, e.type);
        }
        // check_validity (fast-wave/src/simulation.cpp:237-274)
        if (e.z_start < last_z - z_tol) return fail(RSW_ERR_INVALID, "element %d starts before the previous ends", i);
        last_z = e.z_start + el.total_thickness();
        const int64_t k = e.n_x_positions;
        if (k > 1) {
            if (S->nr_phase_steps != 1 && S->nr_phase_steps != k)
                return fail(RSW_ERR_INVALID, "inconsistent number of phase steps");
            S->nr_phase_steps = k;
            if (S->snap_el < 0) S->snap_el = i;
        }
    }
    if (last_z > desc->z_detector + z_tol) return fail(RSW_ERR_INVALID, "detector before the last element");
    CHECK(detector_geom(desc->n, desc->dx, desc->detector_size, desc->pixel_size_x, desc->z_detector, S->geom));
    CHECK(S->bounds.upload(S->geom.bounds));
    CHECK(S->cosv.upload(S->geom.cosv));
    CHECK(S->rv.upload(S->geom.rv));
    const size_t nacc = size_t(S->nr_phase_steps * S->geom.n_pix);
    CHECK(S->acc.alloc(std::max<size_t>(nacc, 1) * sizeof(double)));
    CHECK(S->comp.alloc(std::max<size_t>(nacc, 1) * sizeof(double)));
    CU(cudaMemset(S->acc.p, 0, nacc * sizeof(double)));
    CU(cudaMemset(S->comp.p, 0, nacc * sizeof(double)));
    const size_t dsum_bytes = size_t(S->geom.n_pix) * sizeof(double) + 16;
    CHECK(S->dsum.alloc(dsum_bytes));
    CU(cudaMemset(S->dsum.p, 0, dsum_bytes));
    const size_t fb = size_t(desc->n) * S->plan->elem();
    CHECK(S->buf[0].alloc(fb));
    if (S->nr_phase_steps > 1) CHECK(S->buf[1].alloc(fb));
    CHECK(S->mat_db.alloc(size_t(std::max(desc->n_elements, 1)) * 128 * sizeof(double2)));
    CHECK(S->mat_fac.alloc(size_t(std::max(desc->n_elements, 1)) * 128 * sizeof(double2)));
    *out = S.release();
    return RSW_OK;
}

rsw_status rsw_sim_destroy(rsw_sim s) {
    delete s;
    return RSW_OK;
}

rsw_status rsw_sim_shape(rsw_sim S, int64_t *nps, int64_t *npix, int64_t *steps) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    if (nps) *nps = S->nr_phase_steps;
    if (npix) *npix = S->geom.n_pix;
    if (steps) *steps = S->split_steps;
    return RSW_OK;
}

rsw_status rsw_sim_reset(rsw_sim S, void *stream) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    const int64_t n = S->nr_phase_steps * S->geom.n_pix;
    cudaError_t e = launch_zero((double *)S->acc.p, n, (cudaStream_t)stream);
    if (e == cudaSuccess) e = launch_zero((double *)S->comp.p, n, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(RSW_ERR_CUDA, "reset: %s", cudaGetErrorString(e));
    return RSW_OK;
}

rsw_status rsw_sim_read(rsw_sim S, double *h, void *stream) {
    if (!S || !h) return fail(RSW_ERR_INVALID, "NULL argument");
    const size_t n = size_t(S->nr_phase_steps * S->geom.n_pix);
    CU(cudaMemcpyAsync(h, S->acc.p, n * sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CU(cudaStreamSynchronize((cudaStream_t)stream));
    return RSW_OK;
}

rsw_status rsw_sim_read_device(rsw_sim S, double *d, void *stream) {
    if (!S || !d) return fail(RSW_ERR_INVALID, "NULL argument");
    const size_t n = size_t(S->nr_phase_steps * S->geom.n_pix);
    CU(cudaMemcpyAsync(d, S->acc.p, n * sizeof(double), cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
    return RSW_OK;
}

rsw_status rsw_sim_accumulator(rsw_sim S, double **d) {
    if (!S || !d) return fail(RSW_ERR_INVALID, "NULL argument");
    *d = (double *)S->acc.p;
    return RSW_OK;
}

rsw_status rsw_sim_final_field(rsw_sim S, void *dst, void *stream) {
    if (!S || !dst) return fail(RSW_ERR_INVALID, "NULL argument");
    if (S->last_field < 0) return fail(RSW_ERR_INVALID, "no run yet");
    CU(cudaMemcpyAsync(dst, S->buf[S->last_field].p, size_t(S->d.n) * S->plan->elem(), cudaMemcpyDeviceToDevice,
                       (cudaStream_t)stream));
    return RSW_OK;
}

rsw_status rsw_sim_set_timing(rsw_sim S, int enable) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    S->tl.collect();
    S->tl.enabled = enable != 0;
    for (int k = 0; k < 4; ++k) {
        S->tl.ms[k] = 0;
        S->tl.launches[k] = 0;
    }
    return RSW_OK;
}

rsw_status rsw_sim_timing(rsw_sim S, int kind, double *ms, int64_t *launches) {
    if (!S || kind < 0 || kind > 3) return fail(RSW_ERR_INVALID, "bad argument");
    S->tl.collect();
    if (ms) *ms = S->tl.ms[kind];
    if (launches) *launches = S->tl.launches[kind];
    return RSW_OK;
}

rsw_status rsw_sim_set_propagator(rsw_sim S, int mode) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    return rsw_plan_set_propagator(S->plan, mode);
}

rsw_status rsw_sim_set_history(rsw_sim S, double history_dz) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    if (!(history_dz >= 0)) return fail(RSW_ERR_INVALID, "history_dz must be >= 0");
    S->hist_dz = history_dz;
    return RSW_OK;
}

rsw_status rsw_sim_set_keypoints(rsw_sim S, void *const *dst, int64_t n_dst) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    if (n_dst == 0) {
        S->keypoints.clear();
        return RSW_OK;
    }
    if (!dst || n_dst != 2 * int64_t(S->els.size()))
        return fail(RSW_ERR_INVALID, "keypoints: %lld buffers for %zu elements (2 per element)", (long long)n_dst,
                    S->els.size());
    S->keypoints.assign(dst, dst + n_dst);
    return RSW_OK;
}

rsw_status rsw_sim_set_final_fields(rsw_sim S, void *const *dst, int64_t n_dst) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    if (n_dst == 0) {
        S->final_fields.clear();
        return RSW_OK;
    }
    if (!dst || n_dst != S->nr_phase_steps)
        return fail(RSW_ERR_INVALID, "final fields: %lld buffers for %lld phase steps", (long long)n_dst,
                    (long long)S->nr_phase_steps);
    S->final_fields.assign(dst, dst + n_dst);
    return RSW_OK;
}

rsw_status rsw_sim_history(rsw_sim S, double *h_out, double *h_z, int64_t *n_entries, void *stream) {
    if (!S) return fail(RSW_ERR_INVALID, "sim is NULL");
    const int64_t n = int64_t(S->hist_z.size()), np = S->geom.n_pix;
    if (n_entries) *n_entries = n;
    if (h_z) std::copy(S->hist_z.begin(), S->hist_z.end(), h_z);
    if (h_out && n > 0) {
        std::vector<double> tmp(size_t(n * np));
        CU(cudaMemcpyAsync(tmp.data(), S->hist.p, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost,
                           (cudaStream_t)stream));
        CU(cudaStreamSynchronize((cudaStream_t)stream));
        for (int64_t e = 0; e < n; ++e)
            for (int64_t j = 0; j < np; ++j) h_out[j * n + e] = tmp[size_t(e * np + j)];
    }
    return RSW_OK;
}

}  // extern "C"

namespace {

// The deltabeta values of one run per element (gratings: a, b, substrate;
// samples: materials 1..n), and the host images of its sample material tables
// (deltabeta and exp(i y db) at [element * 128 + material], [0] = vacuum).
static rsw_status load_deltabeta(const rsw_sim_s &S, const rsw_source_run *run, double wl,
                                 std::vector<std::vector<cplx>> &db, double *dbh, double *fch) {
    int64_t k = 0;
    db.assign(S.els.size(), {});
    for (size_t i = 0; i < S.els.size(); ++i) {
        const rsw_element &e = S.els[i].d;
        const int cnt = e.type == RSW_EL_SAMPLE ? e.n_materials : 3;
        if (k + cnt > run->n_deltabeta || (cnt > 0 && !run->deltabeta))
            return fail(RSW_ERR_INVALID, "deltabeta table too short (%lld values)", (long long)run->n_deltabeta);
        for (int m = 0; m < cnt; ++m, ++k) db[i].push_back(cplx(run->deltabeta[2 * k], run->deltabeta[2 * k + 1]));
        if (e.type == RSW_EL_SAMPLE) {
            const double psz = e.pixel_size_z;
            for (int m = 0; m < cnt; ++m) {
                const cplx d = db[i][m];
                const cplx f = material_factor(d.real(), d.imag(), psz, wl);
                dbh[(i * 128 + m + 1) * 2] = d.real();
                dbh[(i * 128 + m + 1) * 2 + 1] = d.imag();
                fch[(i * 128 + m + 1) * 2] = f.real();
                fch[(i * 128 + m + 1) * 2 + 1] = f.imag();
            }
            fch[(i * 128) * 2] = 1.0;
        }
    }
    return RSW_OK;
}

static double run_wavelength(const rsw_source_run *run) {
    return run->wavelength_m > 0 ? run->wavelength_m : wavelength(run->energy_ev);
}

// The per-source schedule of big-wave/wavesim.py:84-298 on R's instances:
// source, elements (phase-step snapshot before the first stepped element),
// detector, then the remaining phase steps from the snapshot.
// srcs: one source for every instance (n_srcs 1) or one per instance
// (n_srcs R.nb), all of one type and z; point positions and vector fields
// may differ between instances.
static rsw_status run_schedule(Runner &R, const rsw_source *srcs, int64_t n_srcs, double weight) {
    const rsw_source *src = srcs;  // type, z (and everything of a single source)
    const auto src_of = [&](int b) { return n_srcs > 1 ? srcs + b : srcs; };
    rsw_sim_s &s = *R.S;
    const double z_tol = 1e-8;
    const int nel = int(s.els.size());
    // ---- source (big-wave/source.py:46-101)
    int ci = 0;  // cutoff index: R.cut[ci]
    double z = nel > 0 ? s.els[0].d.z_start : s.d.z_detector;
    R.cur = 0;
    R.readonly = -1;
    R.mid = false;
    R.ones = false;
    s.hist_z.clear();
    R.hist_on = s.hist_dz > 0;
    if (R.hist_on) CHECK(s.hbuf.alloc(size_t(s.d.n) * R.P->elem()));
    const size_t fbytes = size_t(s.d.n) * R.P->elem();
    if (src->type == RSW_SRC_POINT) {
        // grid_density_check (big-wave/propagation.py:31-45), per instance
        const double dzs = z - src->z;
        for (int b = 0; b < R.nb; ++b) {
            const double xs = src_of(b)->x;
            auto dist_x = [&](double idx) {
                const double a = (double(s.d.n) / 2.0 - idx) * s.d.dx + std::fabs(xs);
                return std::sqrt(a * a + dzs * dzs);
            };
            const double wl = R.wls[size_t(b)];
            if (!(std::fabs(dist_x(0.0) - dist_x(1.0)) <= wl / 2.0))
                return fail(RSW_ERR_INVALID, "Nyquist not satisfied, dx too large for the point source at dz = %g",
                            dzs);
            CHECK(rsw_point_source(R.P, static_cast<char *>(R.bp(0)) + size_t(b) * fbytes, s.d.dx, wl, z - src->z,
                                   xs, (void *)R.st));
        }
        CHECK(R.split_step(TransArgs{}, 0.0, ci));
        if (R.hist_on) {
            // generate_analytic_history (big-wave/history.py:43-64) at
            // np.arange(0, z, hdz)[1:]
            const double psx = s.d.pixel_size_x, psy = s.d.pixel_size_y;
            const double nd = py_floordiv(s.d.detector_size, psx);
            const int64_t npx = int64_t(nd);
            const double gradient = R.cut[0] * R.wl;
            const int64_t len = std::max<int64_t>(int64_t(std::ceil(z / s.hist_dz)), 0);
            for (int64_t k = 1; k < len; ++k) {
                const double zh = double(k) * s.hist_dz;
                std::vector<double> img(static_cast<size_t>(npx));
                for (int64_t j = 0; j < npx; ++j) {
                    const double x = (double(j) - py_floordiv(nd, 2.0)) * psx - src->x;
                    const double ang = std::atan(x / zh);
                    const double r2 = x * x + zh * zh;
                    img[size_t(j)] = std::fabs(x) > gradient * zh ? 0.0 : psx * psy * std::cos(ang) / r2;
                }
                CHECK(R.hist_host(img, zh));
            }
        }
    } else if (src->type == RSW_SRC_PLANE || src->type == RSW_SRC_VECTOR) {
        if (src->type == RSW_SRC_PLANE) {
            R.ones = true;
            R.cur = -1;
        } else {
            // each instance's input field (or the one field of all of them)
            for (int b = 0; b < R.nb; ++b) {
                const rsw_source *sb = src_of(b);
                if (!sb->d_field && !sb->h_field) return fail(RSW_ERR_INVALID, "vector source without a field");
                const cudaMemcpyKind kind = sb->d_field ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
                const void *from = sb->d_field ? sb->d_field : sb->h_field;
                CU(cudaMemcpyAsync(static_cast<char *>(R.bp(0)) + size_t(b) * fbytes, from, fbytes, kind, R.st));
            }
        }
        const double dz = z - src->z;
        if (dz != 0.0) CHECK(R.gap(dz, ci, src->z));
    } else {
        return fail(RSW_ERR_INVALID, "unknown source type %d", src->type);
    }

    // ---- element loop (big-wave/wavesim.py:159-219)
    struct Snap {
        double z;
        int cur;
        bool mid, ones;
    } snap{0, -1, false, false};
    for (int i = 0; i < nel; ++i) {
        const rsw_element &e = s.els[i].d;
        if (z < e.z_start) CHECK(R.gap(e.z_start - z, ci, z));
        z = e.z_start;
        if (i == s.snap_el) {
            snap = Snap{z, R.cur, R.mid, R.ones};
            R.readonly = R.cur;
        }
        ci = i + 1;
        const bool kp = s.keypoints.size() == size_t(2 * nel);
        if (kp) CHECK(R.keypoint(s.keypoints[size_t(2 * i)]));
        CHECK(R.apply(i, 0, ci));
        if (kp) CHECK(R.keypoint(s.keypoints[size_t(2 * i + 1)]));
        z = e.z_start + s.els[i].total_thickness();
    }
    if (z < s.d.z_detector - z_tol) CHECK(R.gap(s.d.z_detector - z, ci, z));
    const bool batched = R.nb > 1;  // batches keep no final field
    CHECK(R.finish_phase(0, weight, s.nr_phase_steps == 1 && !batched));
    R.hist_on = false;  // phase steps from the snapshot record no history (big-wave/wavesim.py:234-237)

    // ---- remaining phase steps from the snapshot (big-wave/wavesim.py:238-296)
    for (int64_t step = 1; step < s.nr_phase_steps; ++step) {
        R.cur = snap.cur;
        R.mid = snap.mid;
        R.ones = snap.ones;
        z = snap.z;
        ci = s.snap_el;
        for (int i = s.snap_el; i < nel; ++i) {
            const rsw_element &e = s.els[i].d;
            if (z < e.z_start) CHECK(R.split_step(TransArgs{}, e.z_start - z, ci));
            z = e.z_start;
            ci = i + 1;
            CHECK(R.apply(i, e.n_x_positions > 1 ? step : 0, ci));
            z = e.z_start + s.els[i].total_thickness();
        }
        if (z < s.d.z_detector - z_tol) CHECK(R.split_step(TransArgs{}, s.d.z_detector - z, ci));
        CHECK(R.finish_phase(step, weight, step == s.nr_phase_steps - 1 && !batched));
    }
    s.last_field = batched ? -1 : R.cur;
    return RSW_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

// One source (rsw_sim_run); each: also its own detector values, or NULL.
static rsw_status run_one(rsw_sim_s *S, const rsw_source *src, const rsw_source_run *run, void *stream,
                          double *each) {
    if (!S || !src || !run) return fail(RSW_ERR_INVALID, "NULL argument");
    if (!(run->energy_ev > 0) && !(run->wavelength_m > 0))
        return fail(RSW_ERR_INVALID, "energy or wavelength must be positive");
    ++g_api_calls;
    Runner R;
    R.S = S;
    R.P = S->plan;
    R.st = (cudaStream_t)stream;
    R.fbuf = S->buf;
    R.each = each;
    R.wl = run_wavelength(run);
    R.wls.assign(1, R.wl);
    for (double a : S->cutoff_angles) R.cut.push_back(std::sin(a) / R.wl);
    std::vector<double> dbh(size_t(std::max<int64_t>(S->d.n_elements, 1)) * 128 * 2, 0.0);
    std::vector<double> fch(dbh.size(), 0.0);
    CHECK(load_deltabeta(*S, run, R.wl, R.db, dbh.data(), fch.data()));
    CU(cudaMemcpyAsync(S->mat_db.p, dbh.data(), dbh.size() * sizeof(double), cudaMemcpyHostToDevice, R.st));
    CU(cudaMemcpyAsync(S->mat_fac.p, fch.data(), fch.size() * sizeof(double), cudaMemcpyHostToDevice, R.st));
    return run_schedule(R, src, 1, run->weight);
}

extern "C" {

rsw_status rsw_sim_run(rsw_sim S, const rsw_source *src, const rsw_source_run *run, void *stream) {
    return run_one(S, src, run, stream, nullptr);
}

}  // extern "C"

// Whether the batched column kernel of the plan's transmitting pass holds as
// many CTAs per SM as the plain one. Its per-instance factors take registers
// that the plain kernel does not need; where that costs resident CTAs (some
// complex128 column shapes of 64 to 256 threads), a batch is slower than the
// same sources one after the other (2^26 complex128, three levels with
// columns of 2^7: 24.1 against 27.5 G samples*steps/s on B200).
static bool batch_keeps_occupancy(const rsw_plan_s *P) {
    PassArgs a = base_args(P);
    a.flags = PF_FWD | PF_INV | PF_TW | PF_TRANS | (P->three() ? PF_TWI : 0);
    int64_t plain = 0, batched = 0;
    a.resident = &plain;
    if (launch_col_pass(a, P->dbl(), P->col_e, nullptr) != cudaSuccess) return false;
    BatchTrans dummy{};
    a.btr = &dummy;
    a.resident = &batched;
    if (launch_col_pass(a, P->dbl(), P->col_e, nullptr) != cudaSuccess) return false;
    return batched >= plain;
}

extern "C" {

// Sources per lockstep chunk: as many as fit, with their batch buffers, in
// four fifths of the device memory that is free or already held by the
// sim's batch buffers.
static int64_t batch_chunk(const rsw_sim_s *S, int64_t count) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return count;
    }
    const size_t held = S->bbuf[0].bytes + S->bbuf[1].bytes;
    const size_t per = size_t(S->d.n) * S->plan->elem() * (S->nr_phase_steps > 1 ? 2 : 1);
    const size_t budget = (free_b + held) / 5 * 4;
    int64_t k = std::max<int64_t>(1, std::min<int64_t>(count, per ? int64_t(budget / per) : count));
    // RSW_BATCH_CHUNK caps the chunk (tests)
    const int cap = env_int("RSW_BATCH_CHUNK", 0);
    if (cap > 0) k = std::min<int64_t>(k, cap);
    return k;
}

// One lockstep batch of nb >= 2 sources (rsw_sim_run_batch).
static rsw_status run_lockstep(rsw_sim_s *S, const rsw_source *srcs, int64_t n_srcs, const rsw_source_run *runs,
                               int nb, cudaStream_t st, double *each) {
    rsw_plan_s *P = S->plan;
    const size_t nel = S->els.size();
    const int64_t np = S->geom.n_pix;
    const int64_t stride = batch_sum_stride(np);
    if (S->batch_cap < nb) {
        // sums and counter start at zero and are left at zero by every pass;
        // the capacity counts only once every buffer is in place
        S->batch_cap = 0;
        const size_t fb = size_t(S->d.n) * P->elem() * size_t(nb);
        CHECK(S->bbuf[0].alloc(fb));
        if (S->nr_phase_steps > 1) CHECK(S->bbuf[1].alloc(fb));
        CHECK(S->btab.alloc(nel * 2 * size_t(nb) * sizeof(BatchTrans)));
        CHECK(S->bmat_db.alloc(size_t(nb) * nel * 128 * sizeof(double2)));
        CHECK(S->bmat_fac.alloc(size_t(nb) * nel * 128 * sizeof(double2)));
        const size_t sum_bytes = size_t(nb * stride) * sizeof(double) + 16;
        CHECK(S->bsum.alloc(sum_bytes));
        CU(cudaMemsetAsync(S->bsum.p, 0, sum_bytes, st));
        CHECK(S->bweight.alloc(size_t(nb) * sizeof(double)));
        S->batch_cap = nb;
    }
    Runner R;
    R.S = S;
    R.P = P;
    R.st = st;
    R.nb = nb;
    R.fbuf = S->bbuf;
    R.each = each;
    R.cuts.resize(size_t(nb));
    std::vector<double> dbh(size_t(nb) * nel * 128 * 2, 0.0), fch(dbh.size(), 0.0);
    std::vector<BatchTrans> tab(nel * 2 * size_t(nb));
    std::vector<double> weights(static_cast<size_t>(nb));
    const double2 *mdb = static_cast<const double2 *>(S->bmat_db.p);
    const double2 *mfc = static_cast<const double2 *>(S->bmat_fac.p);
    for (int b = 0; b < nb; ++b) {
        const rsw_source_run *run = runs + b;
        const double wl = run_wavelength(run);
        R.wls.push_back(wl);
        for (double a : S->cutoff_angles) R.cuts[size_t(b)].push_back(std::sin(a) / wl);
        std::vector<std::vector<cplx>> db;
        const size_t off = size_t(b) * nel * 128 * 2;
        CHECK(load_deltabeta(*S, run, wl, db, dbh.data() + off, fch.data() + off));
        // the wavelength-dependent transmission values of each element
        // (Runner::apply computes the same for one source)
        for (size_t i = 0; i < nel; ++i) {
            const rsw_element &e = S->els[i].d;
            BatchTrans &t0 = tab[(i * 2) * size_t(nb) + size_t(b)];
            BatchTrans &t1 = tab[(i * 2 + 1) * size_t(nb) + size_t(b)];
            if (e.type == RSW_EL_SAMPLE) {
                t0.mat_db = mdb + (size_t(b) * nel + i) * 128;
                t0.mat_factor = mfc + (size_t(b) * nel + i) * 128;
                t0.sample_y = (2.0 * M_PI * e.pixel_size_z) / wl;
            } else {
                const double z_step = e.thickness / double(e.nr_steps);
                const cplx fa = material_factor(db[i][0].real(), db[i][0].imag(), z_step, wl);
                const cplx fb = material_factor(db[i][1].real(), db[i][1].imag(), z_step, wl);
                t0.fa = make_double2(fa.real(), fa.imag());
                t0.fb = make_double2(fb.real(), fb.imag());
                const cplx fs = material_factor(db[i][2].real(), db[i][2].imag(), e.substrate_thickness, wl);
                t1.fa = make_double2(fs.real(), fs.imag());
            }
        }
        weights[size_t(b)] = run->weight;
        if (b == 0) {
            R.wl = wl;
            R.cut = R.cuts[0];
            R.db = db;
        }
    }
    // pageable sources: staged before the calls return
    CU(cudaMemcpyAsync(S->bmat_db.p, dbh.data(), dbh.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(S->bmat_fac.p, fch.data(), fch.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(S->btab.p, tab.data(), tab.size() * sizeof(BatchTrans), cudaMemcpyHostToDevice, st));
    CU(cudaMemcpyAsync(S->bweight.p, weights.data(), weights.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    return run_schedule(R, srcs, n_srcs, 0.0);
}

rsw_status rsw_sim_run_batch(rsw_sim S, const rsw_source *srcs, int64_t n_sources, const rsw_source_run *runs,
                             int64_t count, double *d_each, void *stream) {
    if (!S || !srcs || (!runs && count > 0)) return fail(RSW_ERR_INVALID, "NULL argument");
    if (count < 0 || count > RSW_BATCH_MAX)
        return fail(RSW_ERR_INVALID, "batch of %lld sources (at most %d)", (long long)count, RSW_BATCH_MAX);
    if (n_sources != 1 && n_sources != count)
        return fail(RSW_ERR_INVALID, "%lld source descriptions for %lld runs (1 or one per run)",
                    (long long)n_sources, (long long)count);
    const auto src_of = [&](int64_t b) { return n_sources > 1 ? srcs + b : srcs; };
    bool same_kind = true;  // one type and z: lockstep possible
    for (int64_t b = 1; b < n_sources; ++b)
        same_kind = same_kind && srcs[b].type == srcs[0].type && srcs[b].z == srcs[0].z;
    for (int64_t b = 0; b < count; ++b)
        if (!(runs[b].energy_ev > 0) && !(runs[b].wavelength_m > 0))
            return fail(RSW_ERR_INVALID, "source %lld: energy or wavelength must be positive", (long long)b);
    const rsw_plan_s *P = S->plan;
    // lockstep needs the two- or three-level passes with the chirp form of the
    // Fresnel kernel and the fused detection; everything else runs the
    // sources one after the other, with the same results
    const bool lockstep = count > 1 && P->log_n1 > 0 && !P->blue && P->prop_mode == RSW_PROP_FRESNEL &&
                          S->hist_dz == 0.0 && S->keypoints.empty() && S->final_fields.empty() &&
                          !S->els.empty() && S->geom.n_pix > 0 && same_kind &&
                          batch_keeps_occupancy(P);
    // consecutive chunks keep the order in which every (phase step, pixel)
    // accumulator receives the sources
    const int64_t chunk = lockstep ? batch_chunk(S, count) : 1;
    const int64_t per_source = S->nr_phase_steps * S->geom.n_pix;  // d_each values of one source
    for (int64_t b = 0; b < count; b += chunk) {
        const int64_t k = std::min(chunk, count - b);
        double *each = d_each ? d_each + b * per_source : nullptr;
        if (k > 1) {
            ++g_api_calls;
            CHECK(run_lockstep(S, src_of(b), n_sources > 1 ? k : 1, runs + b, int(k), (cudaStream_t)stream, each));
        } else {
            CHECK(run_one(S, src_of(b), runs + b, stream, each));
        }
    }
    return RSW_OK;
}

}  // extern "C"
