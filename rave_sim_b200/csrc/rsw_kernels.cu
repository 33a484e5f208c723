// Small kernels of the split-step engine: spectrum reordering, per-call
// transmission, point source, detector binning, fills; launch counter and
// row-pass dispatch.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "rsw_passes.cuh"

namespace rsw {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda), looked up once
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

bool encode_col_map(CUtensorMap *map, const void *in, int64_t n, int log_n2, int words_per_sample, int box_w,
                    int box_h) {
    const EncodeTiledFn fn = encode_tiled_fn();
    if (!fn || (reinterpret_cast<uintptr_t>(in) & 15) != 0 || box_w > 256 || box_h > 256) return false;
    const int64_t row_words = (int64_t(1) << log_n2) * words_per_sample;
    const int64_t rows = n >> log_n2;
    if (rows < box_h || row_words < box_w || rows > (int64_t(1) << 31) || row_words > (int64_t(1) << 31))
        return false;
    cuuint64_t dims[2] = {cuuint64_t(row_words), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(row_words * 8)};
    cuuint32_t box[2] = {cuuint32_t(box_w), cuuint32_t(box_h)};
    cuuint32_t elem_strides[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void *>(in), dims, strides, box, elem_strides,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static std::atomic<unsigned long long> g_launches{0};  // host-side count of kernel launches
void count_launch() { ++g_launches; }

cudaError_t launch_row_pass_f64(const PassArgs &a, int e, cudaStream_t s);
cudaError_t launch_row_pass_f32(const PassArgs &a, int e, cudaStream_t s);
cudaError_t launch_row_pass_f64_batch(const PassArgs &a, int e, cudaStream_t s);
cudaError_t launch_row_pass_f32_batch(const PassArgs &a, int e, cudaStream_t s);
// per-instance transfer functions take the batched kernels
cudaError_t launch_row_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s) {
    if (a.bpr) return dbl ? launch_row_pass_f64_batch(a, e, s) : launch_row_pass_f32_batch(a, e, s);
    return dbl ? launch_row_pass_f64(a, e, s) : launch_row_pass_f32(a, e, s);
}

// ---------------------------------------------------------- small kernels
// internal spectrum layout <-> natural frequency order. Frequency
// k = k1 + N1 (kb + Nb kr) sits at ((p1 Nb + pb) Nr + pr), p = digitpos of
// each level's index (log_nb = 0 for two-level and single-level plans).
// Position in the spectrum layout of natural frequency k; indices at and
// above one transform's length address consecutive transforms (batches).
__device__ __forceinline__ int64_t spec_addr(int64_t k, const SpecLevels &v) {
    const int log_len = v.log_n1 + v.log_nb + v.log_nr;
    const int64_t seq = k >> log_len << log_len;
    const int64_t k1 = k & ((int64_t(1) << v.log_n1) - 1);
    const int64_t kb = (k >> v.log_n1) & ((int64_t(1) << v.log_nb) - 1);
    const int64_t kr = (k >> (v.log_n1 + v.log_nb)) & ((int64_t(1) << v.log_nr) - 1);
    return seq + ((((digitpos_rt(k1, v.log_n1, v.rb_n1) << v.log_nb) + digitpos_rt(kb, v.log_nb, v.rb_nb))
                   << v.log_nr) +
                  digitpos_rt(kr, v.log_nr, v.rb_nr));
}
template <typename Cx>
__global__ void spec_to_natural_kernel(const Cx *__restrict__ in, Cx *__restrict__ out, int64_t n, SpecLevels v) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        out[k] = in[spec_addr(k, v)];
}
template <typename Cx>
__global__ void natural_to_spec_kernel(const Cx *__restrict__ in, Cx *__restrict__ out, int64_t n, SpecLevels v) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride)
        out[spec_addr(k, v)] = in[k];
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
    const double half = double(n) / 2.0;  // the reference's N / 2 (a float for odd N)
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = __dsub_rn(__dmul_rn(double(i) - half, dx), x_src);
        const double r = sqrt(__dadd_rn(__dmul_rn(x, x), __dmul_rn(z, z)));
        double s, c;
        sincos(__dmul_rn(r, w), &s, &c);
        const double scl = 1.0 / sqrt(r);
        u[i] = to_c(make_double2(c * scl, s * scl), Cx{});
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

// out (cols x rows) = transpose of in (rows x cols), row-major, through
// 32 x 32 tiles in shared memory (padded rows: conflict-free columns)
template <typename Cx>
__global__ void __launch_bounds__(256) transpose_kernel(const Cx *__restrict__ in, Cx *__restrict__ out,
                                                        int64_t rows, int64_t cols) {
    __shared__ Cx tile[32][33];
    const int64_t tx = (cols + 31) / 32, ty = (rows + 31) / 32;
    for (int64_t t = blockIdx.x; t < tx * ty; t += gridDim.x) {
        const int64_t r0 = (t / tx) * 32, c0 = (t % tx) * 32;
        for (int i = threadIdx.y; i < 32; i += 8) {
            const int64_t r = r0 + i, c = c0 + threadIdx.x;
            if (r < rows && c < cols) tile[i][threadIdx.x] = in[r * cols + c];
        }
        __syncthreads();
        for (int i = threadIdx.y; i < 32; i += 8) {
            const int64_t c = c0 + i, r = r0 + threadIdx.x;
            if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][i];
        }
        __syncthreads();
    }
}

// Four-step twiddle of the out-of-core FFT: u[j len + k] *= exp(sign 2 pi i
// ((row0 + j) k mod n) / n) for j < count, k < len (FP64 phase, exact index).
template <typename Cx>
__global__ void ooc_twiddle_kernel(Cx *__restrict__ u, int64_t count, int log_len, int64_t row0, int log_n,
                                   double sign) {
    const int64_t total = count << log_len;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t nmask = (int64_t(1) << log_n) - 1;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int64_t j = row0 + (i >> log_len), k = i & ((int64_t(1) << log_len) - 1);
        const double t = ldexp(double((j * k) & nmask), 1 - log_n);  // 2 m / n, exact
        double sn, cs;
        sincospi(t, &sn, &cs);
        const double2 w = make_double2(cs, sign * sn);
        const double2 v = make_double2(double(u[i].x), double(u[i].y));
        u[i] = to_c(make_double2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x), Cx{});
    }
}

static unsigned grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    const int64_t cap = 148 * 32;
    return unsigned(b < 1 ? 1 : (b > cap ? cap : b));
}

cudaError_t launch_spec_to_natural(const void *in, void *out, int64_t n, const SpecLevels &v, bool dbl,
                                   cudaStream_t s) {
    ++g_launches;
    if (dbl)
        spec_to_natural_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)in, (double2 *)out, n, v);
    else
        spec_to_natural_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)in, (float2 *)out, n, v);
    return cudaGetLastError();
}
cudaError_t launch_natural_to_spec(const void *in, void *out, int64_t n, const SpecLevels &v, bool dbl,
                                   cudaStream_t s) {
    ++g_launches;
    if (dbl)
        natural_to_spec_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)in, (double2 *)out, n, v);
    else
        natural_to_spec_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)in, (float2 *)out, n, v);
    return cudaGetLastError();
}
cudaError_t launch_trans(void *u, int64_t n, const TransArgs &tr, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) trans_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((double2 *)u, n, tr);
    else trans_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((float2 *)u, n, tr);
    return cudaGetLastError();
}
cudaError_t launch_transpose(const void *in, void *out, int64_t rows, int64_t cols, bool dbl, cudaStream_t s) {
    ++g_launches;
    const int64_t tiles = ((rows + 31) / 32) * ((cols + 31) / 32);
    const unsigned g = unsigned(tiles < 148 * 16 ? tiles : 148 * 16);
    if (dbl) transpose_kernel<double2><<<g, dim3(32, 8), 0, s>>>((const double2 *)in, (double2 *)out, rows, cols);
    else transpose_kernel<float2><<<g, dim3(32, 8), 0, s>>>((const float2 *)in, (float2 *)out, rows, cols);
    return cudaGetLastError();
}
cudaError_t launch_ooc_twiddle(void *u, int64_t count, int log_len, int64_t row0, int log_n, bool inverse, bool dbl,
                               cudaStream_t s) {
    ++g_launches;
    const int64_t total = count << log_len;
    const double sign = inverse ? 1.0 : -1.0;
    if (dbl) ooc_twiddle_kernel<double2><<<grid_for(total, 256), 256, 0, s>>>((double2 *)u, count, log_len, row0, log_n, sign);
    else ooc_twiddle_kernel<float2><<<grid_for(total, 256), 256, 0, s>>>((float2 *)u, count, log_len, row0, log_n, sign);
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
unsigned long long launch_count() { return g_launches.load(); }

// ------------------------------------------------------- Bluestein (any N)
// A length-N DFT as a circular convolution of length M >= 2N - 1 (a power of
// two), with the chirp b[k] = exp(i pi k^2 / N):
//   X[k] = conj(b[k]) sum_j (x[j] conj(b[j])) b[k - j].
// The pointwise products are taken in FP64 for both field types (the tables
// are FP64), so the fields round once per product.
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(double(a.x), double(a.y)); }
template <typename Cx>
__global__ void blue_pre_kernel(const Cx *__restrict__ in, Cx *__restrict__ w, int64_t n, int64_t m,
                                const double2 *__restrict__ b, int conj_in) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += stride) {
        if (k < n) {
            double2 x = to_d(in[k]);
            if (conj_in) x.y = -x.y;
            w[k] = to_c(cmulc(x, b[k]), Cx{});
        } else {
            w[k] = to_c(make_double2(0.0, 0.0), Cx{});
        }
    }
}
template <typename Cx>
__global__ void blue_mul_kernel(Cx *__restrict__ w, const double2 *__restrict__ bh, int64_t m) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < m; k += stride)
        w[k] = to_c(cmul(to_d(w[k]), bh[k]), Cx{});
}
template <typename Cx>
__global__ void blue_post_kernel(const Cx *__restrict__ w, Cx *__restrict__ out, int64_t n,
                                 const double2 *__restrict__ b, double scale, int conj_out) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
        double2 y = cmulc(to_d(w[k]), b[k]);
        y = make_double2(y.x * scale, (conj_out ? -y.y : y.y) * scale);
        out[k] = to_c(y, Cx{});
    }
}
// Transfer function and cutoff on a natural-order spectrum of any length:
// ks = k or k - N (np.fft.fftfreq's order), fx = (ks * (1/N)) / dx in the
// reference's order (big-wave/propagation.py:154-175, :124-128), applied in FP64.
template <typename Cx>
__global__ void prop_natural_kernel(Cx *__restrict__ U, int64_t n, PropArgs p) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t pos_end = (n - 1) / 2 + 1;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
        if (p.has_cut && k >= p.cut_lo && k < p.cut_hi) {
            U[k] = to_c(make_double2(0.0, 0.0), Cx{});
            continue;
        }
        if (!p.has_h) continue;
        const int64_t ks = k < pos_end ? k : k - n;
        const double fx = __ddiv_rn(__dmul_rn(double(ks), p.fac), p.dx);
        double ph;
        if (p.exact) {
            const double f2 = __dmul_rn(fx, fx);
            const double d = __dsub_rn(p.inv_wl2, f2);
            if (!(d > 0.0)) {
                U[k] = to_c(make_double2(0.0, 0.0), Cx{});
                continue;
            }
            ph = __ddiv_rn(__dmul_rn(p.z2pi, f2), __dadd_rn(p.inv_wl, __dsqrt_rn(d)));
        } else {
            ph = __dmul_rn(p.c, __dmul_rn(fx, fx));
        }
        double sn, cs;
        sincos_phase(ph, &sn, &cs);
        const double2 H = make_double2(p.A.x * cs - p.A.y * sn, p.A.x * sn + p.A.y * cs);
        U[k] = to_c(cmul(to_d(U[k]), H), Cx{});
    }
}

cudaError_t launch_blue_pre(const void *in, void *w, int64_t n, int64_t m, const double2 *b, bool conj_in, bool dbl,
                            cudaStream_t s) {
    ++g_launches;
    if (dbl)
        blue_pre_kernel<double2><<<grid_for(m, 256), 256, 0, s>>>((const double2 *)in, (double2 *)w, n, m, b, conj_in);
    else
        blue_pre_kernel<float2><<<grid_for(m, 256), 256, 0, s>>>((const float2 *)in, (float2 *)w, n, m, b, conj_in);
    return cudaGetLastError();
}
cudaError_t launch_blue_mul(void *w, const double2 *bh, int64_t m, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) blue_mul_kernel<double2><<<grid_for(m, 256), 256, 0, s>>>((double2 *)w, bh, m);
    else blue_mul_kernel<float2><<<grid_for(m, 256), 256, 0, s>>>((float2 *)w, bh, m);
    return cudaGetLastError();
}
cudaError_t launch_blue_post(const void *w, void *out, int64_t n, const double2 *b, double scale, bool conj_out,
                             bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl)
        blue_post_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((const double2 *)w, (double2 *)out, n, b, scale,
                                                                  conj_out);
    else
        blue_post_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((const float2 *)w, (float2 *)out, n, b, scale,
                                                                 conj_out);
    return cudaGetLastError();
}
cudaError_t launch_prop_natural(void *U, int64_t n, const PropArgs &p, bool dbl, cudaStream_t s) {
    ++g_launches;
    if (dbl) prop_natural_kernel<double2><<<grid_for(n, 256), 256, 0, s>>>((double2 *)U, n, p);
    else prop_natural_kernel<float2><<<grid_for(n, 256), 256, 0, s>>>((float2 *)U, n, p);
    return cudaGetLastError();
}

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

namespace rsw {
// Phase-step signal retrieval: per pixel j the least-squares fit of
// I_k = a sin(phi_k) + b cos(phi_k) + c over the K phase steps, as
// (a, b, c) = P I with the 3 x K pseudo-inverse P of [sin, cos, 1] (built on
// the host); outputs as signal_retrieval_least_squares of the reference's
// crack-simulation notebook: abs = K c, phase = -atan2(a, b),
// vis = sqrt(a^2 + b^2) / c, chi2 = squared residual norm.
__global__ void retrieval_kernel(const double *__restrict__ data, int64_t n_pix, RetrievalArgs r,
                                 double *__restrict__ dabs, double *__restrict__ dphase,
                                 double *__restrict__ dvis, double *__restrict__ chi2) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n_pix; j += stride) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int k = 0; k < r.k; ++k) {
            const double v = data[int64_t(k) * n_pix + j];
            a = fma(r.p[k], v, a);
            b = fma(r.p[RSW_RETRIEVAL_MAX + k], v, b);
            c = fma(r.p[2 * RSW_RETRIEVAL_MAX + k], v, c);
        }
        if (chi2) {
            double e2 = 0.0;
            for (int k = 0; k < r.k; ++k) {
                const double e = data[int64_t(k) * n_pix + j] - (a * r.sn[k] + b * r.cs[k] + c);
                e2 = fma(e, e, e2);
            }
            chi2[j] = e2;
        }
        if (dabs) dabs[j] = c * double(r.k);
        if (dphase) dphase[j] = -atan2(a, b);
        if (dvis) dvis[j] = sqrt(a * a + b * b) / c;
    }
}
cudaError_t launch_retrieval(const double *data, int64_t n_pix, const RetrievalArgs &r, double *dabs, double *dphase,
                             double *dvis, double *chi2, cudaStream_t s) {
    if (n_pix <= 0) return cudaSuccess;
    ++g_launches;
    retrieval_kernel<<<grid_for(n_pix, 256), 256, 0, s>>>(data, n_pix, r, dabs, dphase, dvis, chi2);
    return cudaGetLastError();
}
}  // namespace rsw
