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
// intermediate spectrum of up to RSW_NOALLOC_MAX_N samples, then one slot of
// twiddle tables for every length (2^4 .. 2^16) and dtype, 258 KiB in all.
// Every GPU that loads the library holds the array until the process exits.
// Host code never dereferences the symbol: on the first call on each device
// (with that device current) the device address is taken with
// cudaGetSymbolAddress and passed to the kernels; it is taken again when the
// device's context changes (after a cudaDeviceReset).
//
// The first call for a length and dtype on a device builds that slot's tables
// with a small kernel on the caller's stream; later calls reuse the slot, which
// is never rebuilt, so a call for another length cannot change the tables of
// this one. A first call made while `stream` is capturing a graph is refused
// (RSW_ERR_INVALID), since its table build would only run at a replay. All
// calls share the spectrum and it keeps the last call's contents; every
// spectrum sample a call reads was written earlier in the same call, so
// nothing needs clearing. Calls whose work overlaps on the GPU (different
// streams without ordering, or several host threads) race on the array and
// must be serialised by the caller, including a call that overlaps the first
// call for its length and dtype.
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
constexpr int LOG_MIN = 4, LOG_MAX = 16;
constexpr int KEYS = 2 * (LOG_MAX - LOG_MIN + 1);     // (length, dtype) pairs
constexpr size_t ARRAY_BYTES = 1536 * 1024;
constexpr size_t SPEC_BYTES = size_t(MAX_N) * 16;  // intermediate spectrum, complex128 worst case

// The level split of the plans: one level up to 2^13 (c128) / 2^14 (c64),
// then two levels.
constexpr int split_n1(int log_n, bool dbl) { return log_n > (dbl ? 13 : 14) ? log_n / 2 : 0; }
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
// bytes of the block twiddles of a length-2^log_l block (16 samples per
// thread, radix-16 stages; 16-byte entries for complex128, 8 for complex64)
constexpr size_t block_tw_bytes(int log_l, bool dbl) {
    const int eb = dbl ? 16 : 8;
    const int max_ls = direct_max_ls(eb, log_l);
    int64_t n = 0;
    for (int s = 0; s < stage_count(log_l) - 1; ++s) n += stage_tw_entries(log_l, s, max_ls);
    return size_t(n > 0 ? n : 1) * size_t(eb);
}
// The table slot of one (length, dtype): block twiddles of the row and
// column levels, then the FP64 four-step tables lo[2^h], hi[2^(log_n - h)].
struct Slot {
    size_t tw_row, tw_col, tw4_lo, tw4_hi, end;
};
constexpr Slot slot_at(size_t base, int log_n, bool dbl) {
    const int l1 = split_n1(log_n, dbl), l2 = log_n - l1, h = (log_n + 1) / 2;
    Slot s{};
    s.tw_row = base;
    s.tw_col = align256(s.tw_row + block_tw_bytes(l2, dbl));
    s.tw4_lo = align256(s.tw_col + (l1 > 0 ? block_tw_bytes(l1, dbl) : 0));
    s.tw4_hi = align256(s.tw4_lo + (l1 > 0 ? (size_t(1) << h) * 16 : 0));
    s.end = align256(s.tw4_hi + (l1 > 0 ? (size_t(1) << (log_n - h)) * 16 : 0));
    return s;
}
constexpr int key_of(int log_n, int dtype) { return (log_n - LOG_MIN) * 2 + dtype; }
// slots in key order after the spectrum
constexpr Slot slot_of(int key) {
    size_t base = SPEC_BYTES;
    for (int k = 0;; ++k) {
        const Slot s = slot_at(base, LOG_MIN + k / 2, (k % 2) == RSW_C128);
        if (k == key) return s;
        base = s.end;
    }
}
static_assert(slot_of(KEYS - 1).end <= ARRAY_BYTES, "table slots exceed the array");

}  // namespace

// The scratch array of rsw_fft_forward_noalloc (see the file comment).
static __device__ __align__(256) unsigned char g_noalloc_scratch[ARRAY_BYTES];

namespace {

// Block twiddles of a block of length 2^log_l into `out` in the layout of
// the block FFT (rsw_stages.h): W_M^m = exp(-2 pi i m / M) as {cos, sin}
// (FP64) from sincospi of an exact argument, or for complex64 the packed
// lifting form {a, b} by the entry's tw_mode (the rule of the host-built
// tables): mode 1 takes out a quarter turn, mode 2 reduces m to
// (-M/2, M/2] and takes out a half turn beyond a quarter turn, then
// a = -tan(t/2), b = sin(t) of the remaining angle t = -2 pi m' / M; in mode
// 2 a is rounded to the nearest float whose lowest mantissa bit is the
// half-turn flag.
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
                const int mode = stage_tw_mode(log_l, s, max_ls, 4, k);
                m %= mod;
                unsigned flip = 0;
                if (mode == 1) {
                    m -= mod / 4;
                } else if (mode == 2) {
                    if (m > mod / 2) m -= mod;
                    if (4 * m > mod) {
                        m -= mod / 2;
                        flip = 1;
                    } else if (4 * m < -mod) {
                        m += mod / 2;
                        flip = 1;
                    }
                }
                double sh, ch;
                sincospi(double(m) / double(mod), &sh, &ch);  // angle -t/2
                const double a = sh / ch;                       // -tan(t/2)
                float af = float(a);
                if (mode == 2 && (__float_as_uint(af) & 1u) != flip)
                    af = nextafterf(af, double(af) < a ? HUGE_VALF : -HUGE_VALF);
                out[2 * (off + k)] = af;
                out[2 * (off + k) + 1] = T(-sinpi(2.0 * double(m) / double(mod)));  // sin(t)
            }
        }
        off += count;
    }
}

__global__ void noalloc_tables_kernel(unsigned char *scratch, Slot slot, int log_n, int log_n1, int log_n2, int dbl) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    if (dbl) {
        block_tables(reinterpret_cast<double *>(scratch + slot.tw_row), log_n2, idx, stride);
        if (log_n1 > 0) block_tables(reinterpret_cast<double *>(scratch + slot.tw_col), log_n1, idx, stride);
    } else {
        block_tables(reinterpret_cast<float *>(scratch + slot.tw_row), log_n2, idx, stride);
        if (log_n1 > 0) block_tables(reinterpret_cast<float *>(scratch + slot.tw_col), log_n1, idx, stride);
    }
    if (log_n1 > 0) {  // four-step tables (FP64): lo[a] = W_N^a, hi[b] = W_N^(b 2^h)
        const int h = (log_n + 1) / 2;
        const double n = double(int64_t(1) << log_n);
        double *lo = reinterpret_cast<double *>(scratch + slot.tw4_lo);
        double *hi = reinterpret_cast<double *>(scratch + slot.tw4_hi);
        for (int a = idx; a < (1 << h); a += stride) sincospi(-2.0 * a / n, &lo[2 * a + 1], &lo[2 * a]);
        for (int b = idx; b < (1 << (log_n - h)); b += stride)
            sincospi(-2.0 * double(int64_t(b) << h) / n, &hi[2 * b + 1], &hi[2 * b]);
    }
}

// Per device: the context the state belongs to (a device reset gives a new
// one), the array's device address in it, and the slots built there.
struct DeviceState {
    void *ctx = nullptr;
    unsigned char *ptr = nullptr;
    bool built[KEYS] = {};
};
constexpr int MAX_DEVICES = 64;
DeviceState g_state[MAX_DEVICES];
std::mutex g_mutex;

// the current context (driver cuCtxGetCurrent through the runtime's entry point)
void *current_context() {
    using Fn = int (*)(void **);
    static Fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<Fn>(p);
    }();
    void *ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

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
    const bool dbl = dtype == RSW_C128;
    const int log_n1 = split_n1(log_n, dbl), log_n2 = log_n - log_n1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail_na(RSW_ERR_CUDA, "no current device");
    // an error left by earlier work is not this call's to report or clear
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        char msg[160];
        snprintf(msg, sizeof msg, "a CUDA error from earlier work is pending: %s", cudaGetErrorString(pending));
        return fail_na(RSW_ERR_CUDA, msg);
    }
    const int key = key_of(log_n, dtype);
    const Slot slot = slot_of(key);
    unsigned char *scratch;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        DeviceState &st = g_state[dev];
        void *ctx = current_context();
        if (!st.ptr || ctx != st.ctx) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
            st = DeviceState{};
            st.ctx = ctx;
            st.ptr = static_cast<unsigned char *>(p);
        }
        scratch = st.ptr;
        if (!st.built[key]) {
            cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
            const cudaError_t ce = cudaStreamIsCapturing(s, &cap);
            if (ce != cudaSuccess) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(ce));
            if (cap != cudaStreamCaptureStatusNone)
                return fail_na(RSW_ERR_INVALID,
                               "the first call for this length and dtype on a device builds its tables and "
                               "cannot be made while the stream is capturing");
            noalloc_tables_kernel<<<16, 256, 0, s>>>(scratch, slot, log_n, log_n1, log_n2, dbl ? 1 : 0);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return fail_na(RSW_ERR_CUDA, cudaGetErrorString(e));
            st.built[key] = true;
        }
    }
    PassArgs a{};
    a.n = n;
    a.log_n1 = log_n1;
    a.log_n2 = log_n2;
    a.tw_row = scratch + slot.tw_row;
    a.tw_col = scratch + slot.tw_col;
    a.tw4_lo = scratch + slot.tw4_lo;
    a.tw4_hi = scratch + slot.tw4_hi;
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
