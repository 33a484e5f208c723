// rsw_fft_forward_noalloc: the natural-order forward FFT of rsw_fft_forward
// for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc/cudaFree on the path
// where they need an FFT: a process whose device memory is entirely managed
// by another allocator (a framework's caching allocator that owns the free
// memory, so a raw cudaMalloc fails or fragments it), or a latency-sensitive
// loop that must not pay the device-wide synchronisation of cudaFree. The
// plan-based entry points allocate (twiddle tables and an N-sample scratch
// buffer per plan); this entry point does not.
//
// Its scratch is the file-scope array g_noalloc_scratch below (1.5 MiB): the
// intermediate spectrum of up to RSW_NOALLOC_MAX_N samples plus the twiddle
// tables of the current length. Every GPU that loads the library holds the
// array until the process exits. Host code never dereferences the symbol: on
// the first call on each device (with that device current) the device address
// is taken once with cudaGetSymbolAddress and passed to the kernels.
//
// All calls share the array and it keeps the last call's contents: the
// tables are rebuilt (by a small kernel on the caller's stream) whenever the
// length or dtype differs from the previous call on that device, and every
// scratch sample a call reads was written earlier in the same call, so
// nothing needs clearing. Calls whose work overlaps on the GPU (different
// streams without ordering, or several host threads) race on the array and
// must be serialised by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>

#include "rsw.h"
#include "rsw_passes.cuh"

namespace rsw {
rsw_status set_error(rsw_status st, const char *msg);  // message for rsw_last_error()
cudaError_t launch_row_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s);
cudaError_t launch_col_pass(const PassArgs &a, bool dbl, int e, cudaStream_t s);
cudaError_t launch_spec_to_natural(const void *in, void *out, int64_t n, const SpecLevels &v, bool dbl,
                                   cudaStream_t s);
}  // namespace rsw

using namespace rsw;

namespace {

constexpr int64_t MAX_N = RSW_NOALLOC_MAX_N;
constexpr size_t SPEC_BYTES = size_t(MAX_N) * 16;  // intermediate spectrum, complex128 worst case
constexpr size_t BLOCK_TW_ENTRIES = 8192;           // per level, >= the block twiddles of 2^8 (both dtypes)
constexpr size_t TW4_ENTRIES = 256;                 // 2^ceil(16/2)
constexpr size_t OFF_TWROW = SPEC_BYTES;
constexpr size_t OFF_TWCOL = OFF_TWROW + BLOCK_TW_ENTRIES * 16;
constexpr size_t OFF_TW4LO = OFF_TWCOL + BLOCK_TW_ENTRIES * 16;
constexpr size_t OFF_TW4HI = OFF_TW4LO + TW4_ENTRIES * 16;
constexpr size_t SCRATCH_BYTES = OFF_TW4HI + TW4_ENTRIES * 16;
static_assert(SCRATCH_BYTES <= 1536 * 1024, "scratch layout exceeds the array");

}  // namespace

// The scratch array of rsw_fft_forward_noalloc (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[1536 * 1024];

namespace {

// Block twiddles of a block of length 2^log_l into `out` in the layout of
// the block FFT (rsw_stages.h): W_M^m = exp(-2 pi i m / M) as {cos, sin}
// (FP64) from sincospi of an exact argument, or for complex64 the packed
// lifting form {a, b}: m reduced to (-M/2, M/2], a half turn taken out beyond
// a quarter turn, a = -tan(t/2), b = sin(t) of the remaining angle
// t = -2 pi m' / M, and a rounded to the nearest float whose lowest mantissa
// bit is the half-turn flag (the rule of the host-built tables).
template <typename T>
__device__ void block_tables(T *out, int log_l, int idx, int stride) {
    int off = 0;
    const int max_ls = direct_max_ls(int(2 * sizeof(T)), log_l);
    for (int s = 0; s < stage_count(log_l) - 1; ++s) {
        const int count = stage_tw_entries(log_l, s, max_ls);
        for (int k = idx; k < count; k += stride) {
            int64_t m, mod;
            stage_tw_entry(log_l, s, max_ls, 4, k, &m, &mod);
            if constexpr (sizeof(T) == 8) {
                double sn, cs;
                sincospi(-2.0 * double(m % mod) / double(mod), &sn, &cs);
                out[2 * (off + k)] = T(cs);
                out[2 * (off + k) + 1] = T(sn);
            } else {
                m %= mod;
                if (m > mod / 2) m -= mod;
                unsigned flip = 0;
                if (4 * m > mod) {
                    m -= mod / 2;
                    flip = 1;
                } else if (4 * m < -mod) {
                    m += mod / 2;
                    flip = 1;
                }
                double sh, ch;
                sincospi(double(m) / double(mod), &sh, &ch);  // angle -t/2
                const double a = sh / ch;                       // -tan(t/2)
                float af = float(a);
                if ((__float_as_uint(af) & 1u) != flip) af = nextafterf(af, double(af) < a ? HUGE_VALF : -HUGE_VALF);
                out[2 * (off + k)] = af;
                out[2 * (off + k) + 1] = T(-sinpi(2.0 * double(m) / double(mod)));  // sin(t)
            }
        }
        off += count;
    }
}

__global__ void noalloc_tables_kernel(unsigned char *scratch, int log_n, int log_n1, int log_n2, int dbl) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (dbl) {
        block_tables(reinterpret_cast<double *>(scratch + OFF_TWROW), log_n2, idx, stride);
        if (log_n1 > 0) block_tables(reinterpret_cast<double *>(scratch + OFF_TWCOL), log_n1, idx, stride);
    } else {
        block_tables(reinterpret_cast<float *>(scratch + OFF_TWROW), log_n2, idx, stride);
        if (log_n1 > 0) block_tables(reinterpret_cast<float *>(scratch + OFF_TWCOL), log_n1, idx, stride);
    }
    if (log_n1 > 0) {  // four-step tables (FP64): lo[a] = W_N^a, hi[b] = W_N^(b 2^h)
        const int h = (log_n + 1) / 2;
        const double n = double(int64_t(1) << log_n);
        double *lo = reinterpret_cast<double *>(scratch + OFF_TW4LO);
        double *hi = reinterpret_cast<double *>(scratch + OFF_TW4HI);
        for (int a = idx; a < (1 << h); a += stride) sincospi(-2.0 * a / n, &lo[2 * a + 1], &lo[2 * a]);
        for (int b = idx; b < (1 << (log_n - h)); b += stride)
            sincospi(-2.0 * double(int64_t(b) << h) / n, &hi[2 * b + 1], &hi[2 * b]);
    }
}

struct DeviceState {
    void *ptr = nullptr;  // device address of g_noalloc_scratch
    int key = -1;         // log_n * 2 + dtype of the tables currently in the array
};
constexpr int MAX_DEVICES = 64;
DeviceState g_state[MAX_DEVICES];
std::mutex g_mutex;

rsw_status fail_na(rsw_status st, const char *msg) {
    char buf[256];
    snprintf(buf, sizeof buf, "rsw_fft_forward_noalloc: %s", msg);
    return set_error(st, buf);
}

}  // namespace

extern "C" rsw_status rsw_fft_forward_noalloc(const void *d_in, void *d_out, int64_t n, int dtype, void *stream) {
    if (!d_in || !d_out) return fail_na(RSW_ERR_INVALID, "NULL argument");
    if (dtype != RSW_C128 && dtype != RSW_C64) return fail_na(RSW_ERR_INVALID, "unknown dtype");
    if (n < 16 || (n & (n - 1)) != 0) return fail_na(RSW_ERR_INVALID, "n must be a power of two >= 16");
    if (n > MAX_N) return fail_na(RSW_ERR_INVALID, "n exceeds the no-allocation limit of 65536 samples");
    int log_n = 0;
    while ((int64_t(1) << log_n) < n) ++log_n;
    // the same level split as the plans: one level up to 2^13 (c128) / 2^14 (c64)
    const bool dbl = dtype == RSW_C128;
    const int row_max = dbl ? 13 : 14;
    int log_n1 = 0, log_n2 = log_n;
    if (log_n > row_max) {
        log_n1 = log_n / 2;
        log_n2 = log_n - log_n1;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail_na(RSW_ERR_CUDA, "no current device");
    unsigned char *scratch;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceState &st = g_state[dev];
        if (!st.ptr) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
            st.ptr = p;
        }
        scratch = static_cast<unsigned char *>(st.ptr);
        const int key = log_n * 2 + dtype;
        if (st.key != key) {
            noalloc_tables_kernel<<<16, 256, 0, s>>>(scratch, log_n, log_n1, log_n2, dbl ? 1 : 0);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
            st.key = key;
        }
    }
    PassArgs a{};
    a.n = n;
    a.log_n1 = log_n1;
    a.log_n2 = log_n2;
    a.tw_row = scratch + OFF_TWROW;
    a.tw_col = scratch + OFF_TWCOL;
    a.tw4_lo = scratch + OFF_TW4LO;
    a.tw4_hi = scratch + OFF_TW4HI;
    a.tw4_shift = (log_n + 1) / 2;
    a.tw_log = log_n;
    a.rb_n1 = 4;
    a.rb_nb = 4;
    a.tw_scale = 1.0 / double(n);
    a.pr.fac = 1.0 / double(n);
    void *spec = scratch;
    cudaError_t e;
    if (log_n1 > 0) {
        a.in = d_in;
        a.out = spec;
        a.flags = PF_FWD | PF_TW;
        if ((e = launch_col_pass(a, dbl, 16, s)) != cudaSuccess) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
        a.in = spec;
    } else {
        a.in = d_in;
    }
    a.out = spec;
    a.flags = PF_FWD;
    if ((e = launch_row_pass(a, dbl, 16, s)) != cudaSuccess) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
    if ((e = launch_spec_to_natural(spec, d_out, n, SpecLevels{log_n1, 0, log_n2, 4, 4, 4}, dbl, s)) != cudaSuccess)
        return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
    return RSW_OK;
}
