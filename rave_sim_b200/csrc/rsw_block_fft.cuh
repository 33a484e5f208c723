// Block FFT building blocks for the split-step passes (sm_100a).
//
// A "block" transforms C independent sequences of length L = 2^LOG_L held by
// one CTA. Each thread owns E = 16 elements in registers; stages are radix-16
// (the first stage takes the remaining radix 2/4/8/16). Forward stages are
// decimation in frequency: natural order in, digit-reversed order out.
// Inverse stages are the exact mirror (decimation in time): digit-reversed
// in, natural out, so a forward/inverse pair needs no reordering and the
// propagator is applied to the digit-reversed spectrum in registers.
//
// Stage s has radix R_s = 2^lr(s) and stride S_s = 2^ls(s). Butterfly beta
// (beta = tp + T*i) of stage s touches positions
//     (beta >> ls) * R*S + (beta & (S-1)) + q*S,   q = 0..R-1
// and is done by one thread, which reads and writes the same positions, so
// stages exchange data through shared memory with one barrier each.
// Shared memory holds the C sequences with one pad element per 16 (phys(p))
// and a per-sequence pitch chosen so that the accesses of one wavefront hit
// distinct banks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace rsw {

template <typename R> struct CxT;
template <> struct CxT<double> { using T = double2; };
template <> struct CxT<float> { using T = float2; };

__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) {
    return mk(a.x * s, a.y * s);
}

__host__ __device__ constexpr int brev_bits(int q, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((q >> b) & 1) << (bits - 1 - b);
    return r;
}

// x * W16^e with W16 = exp(DIR * 2 pi i / 16), e in [0, 8), e known after unrolling.
template <int DIR, typename C> __device__ __forceinline__ C tw16(C x, int e) {
    using R = decltype(x.x);
    const R c1 = R(0.92387953251128675613);  // cos(pi/8)
    const R s1 = R(0.38268343236508977173);  // sin(pi/8)
    const R h = R(0.70710678118654752440);   // cos(pi/4)
    const R d = R(DIR);
    switch (e) {
    case 0: return x;
    case 1: return cmul(x, mk(c1, d * s1));
    case 2: return mk(h * (x.x - d * x.y), h * (x.y + d * x.x));
    case 3: return cmul(x, mk(s1, d * c1));
    case 4: return mk(-d * x.y, d * x.x);
    case 5: return cmul(x, mk(-s1, d * c1));
    case 6: return mk(h * (-x.x - d * x.y), h * (d * x.x - x.y));
    default: return cmul(x, mk(-c1, d * s1));
    }
}

// In-register DFT of size R (2..16) on v[0..R-1], natural order in and out.
// DIR = -1: forward (exp(-2 pi i jk/R)); DIR = +1: inverse, unnormalised.
template <int R, int DIR, typename C> __device__ __forceinline__ void dft(C *v) {
#pragma unroll
    for (int span = R / 2; span >= 1; span >>= 1) {
#pragma unroll
        for (int start = 0; start < R; start += 2 * span) {
#pragma unroll
            for (int k = 0; k < span; ++k) {
                C a = v[start + k], b = v[start + k + span];
                v[start + k] = cadd(a, b);
                v[start + k + span] = tw16<DIR>(csub(a, b), k * (8 / span));
            }
        }
    }
    constexpr int bits = (R == 2) ? 1 : (R == 4) ? 2 : (R == 8) ? 3 : 4;
    C t[R];
#pragma unroll
    for (int q = 0; q < R; ++q) t[q] = v[brev_bits(q, bits)];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = t[q];
}

// Radix structure of a block of length 2^LOG_L.
template <int LOG_L> struct Radix {
    static_assert(LOG_L >= 4, "blocks hold at least 16 elements");
    static constexpr int L = 1 << LOG_L;
    static constexpr int E = 16;
    static constexpr int T = L / E;  // threads per sequence
    static constexpr int NS = (LOG_L + 3) / 4;
    static constexpr int LR0 = LOG_L - 4 * (NS - 1);
    __host__ __device__ static constexpr int lr(int s) { return s == 0 ? LR0 : 4; }
    __host__ __device__ static constexpr int ls(int s) { return LOG_L - LR0 - 4 * s; }
    // offset of stage s in the concatenated block twiddle table
    // (entries [(q-1)*S + j] = W_{R*S}^{j*q}, q = 1..R-1, j < S)
    __host__ __device__ static constexpr int64_t twoff(int s) {
        int64_t o = 0;
        for (int t = 0; t < s; ++t) o += int64_t((1 << lr(t)) - 1) << ls(t);
        return o;
    }
    static constexpr int64_t twsize = twoff(NS - 1);  // last stage has no twiddles
};

// Digit reversal of a block position for a block of length 2^log_l (runtime
// variant, used for row indices of the column level).
__host__ __device__ inline int64_t digitrev_rt(int64_t p, int log_l) {
    if (log_l <= 0) return 0;
    const int ns = (log_l + 3) / 4;
    const int lr0 = log_l - 4 * (ns - 1);
    int64_t f = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = s == 0 ? lr0 : 4;
        const int ls = log_l - lr0 - 4 * s;
        f |= ((p >> ls) & ((1 << lr) - 1)) << sh;
        sh += lr;
    }
    return f;
}
// Inverse of digitrev_rt: frequency index -> block position.
__host__ __device__ inline int64_t digitpos_rt(int64_t f, int log_l) {
    if (log_l <= 0) return 0;
    const int ns = (log_l + 3) / 4;
    const int lr0 = log_l - 4 * (ns - 1);
    int64_t p = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = s == 0 ? lr0 : 4;
        const int ls = log_l - lr0 - 4 * s;
        p |= ((f >> sh) & ((1 << lr) - 1)) << ls;
        sh += lr;
    }
    return p;
}

template <typename Real, int LOG_L, int C> struct Block : Radix<LOG_L> {
    using Rx = Radix<LOG_L>;
    using Cx = typename CxT<Real>::T;
    using Rx::E;
    using Rx::L;
    using Rx::NS;
    using Rx::T;
    static constexpr int NT = T * C;  // threads per CTA
    static constexpr int W = 32 / int(sizeof(Cx) / 4);  // elements per smem wavefront
    static constexpr int BASE = L + L / 16;
    static constexpr int WANT = (C >= W) ? 1 : W / C;
    static constexpr int PITCH = BASE + (((WANT - BASE) % W) + W) % W;
    static constexpr size_t SMEM = size_t(C) * PITCH * sizeof(Cx);

    __device__ static __forceinline__ int phys(int p) { return p + (p >> 4); }

    template <int s> __device__ static __forceinline__ int pos(int tp, int i, int q) {
        constexpr int LRS = Rx::lr(s), LSS = Rx::ls(s);
        const int beta = tp + T * i;
        const int j = beta & ((1 << LSS) - 1);
        const int b = beta >> LSS;
        return (b << (LRS + LSS)) + j + (q << LSS);
    }

    template <int s> __device__ static __forceinline__ void st(Cx *sm, int tp, const Cx *v) {
        constexpr int R = 1 << Rx::lr(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i)
#pragma unroll
            for (int q = 0; q < R; ++q) sm[phys(pos<s>(tp, i, q))] = v[i * R + q];
    }
    template <int s> __device__ static __forceinline__ void ld(const Cx *sm, int tp, Cx *v) {
        constexpr int R = 1 << Rx::lr(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i)
#pragma unroll
            for (int q = 0; q < R; ++q) v[i * R + q] = sm[phys(pos<s>(tp, i, q))];
    }

    // forward stage s: DFT_R then twiddle W_{RS}^{j q}
    template <int s> __device__ static __forceinline__ void dif(int tp, Cx *v, const Cx *__restrict__ tw) {
        constexpr int R = 1 << Rx::lr(s);
        constexpr int LSS = Rx::ls(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i) {
            dft<R, -1>(v + i * R);
            if constexpr (s < NS - 1) {
                const int j = (tp + T * i) & ((1 << LSS) - 1);
                const Cx *t = tw + Rx::twoff(s) + j;
#pragma unroll
                for (int q = 1; q < R; ++q) v[i * R + q] = cmul(v[i * R + q], __ldg(t + (int64_t(q - 1) << LSS)));
            }
        }
    }
    // inverse stage s: conjugate twiddle then inverse DFT_R
    template <int s> __device__ static __forceinline__ void dit(int tp, Cx *v, const Cx *__restrict__ tw) {
        constexpr int R = 1 << Rx::lr(s);
        constexpr int LSS = Rx::ls(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i) {
            if constexpr (s < NS - 1) {
                const int j = (tp + T * i) & ((1 << LSS) - 1);
                const Cx *t = tw + Rx::twoff(s) + j;
#pragma unroll
                for (int q = 1; q < R; ++q) v[i * R + q] = cmulc(v[i * R + q], __ldg(t + (int64_t(q - 1) << LSS)));
            }
            dft<R, +1>(v + i * R);
        }
    }

    // Full forward transform starting from stage-0 positions in registers;
    // ends with the values at last-stage positions in registers.
    template <int s = 0> __device__ static __forceinline__ void forward(Cx *sm, int tp, Cx *v, const Cx *tw) {
        dif<s>(tp, v, tw);
        if constexpr (s < NS - 1) {
            st<s>(sm, tp, v);
            __syncthreads();
            ld<s + 1>(sm, tp, v);
            forward<s + 1>(sm, tp, v, tw);
        }
    }
    // Full inverse transform from last-stage positions to stage-0 positions.
    template <int s = NS - 1> __device__ static __forceinline__ void inverse(Cx *sm, int tp, Cx *v, const Cx *tw) {
        dit<s>(tp, v, tw);
        if constexpr (s > 0) {
            st<s>(sm, tp, v);
            __syncthreads();
            ld<s - 1>(sm, tp, v);
            inverse<s - 1>(sm, tp, v, tw);
        }
    }

    // Position held by register (i, q) at the first / last stage.
    __device__ static __forceinline__ int first_pos(int tp, int r) {
        constexpr int R = 1 << Rx::lr(0);
        return pos<0>(tp, r / R, r % R);
    }
    __device__ static __forceinline__ int last_pos(int tp, int r) {
        constexpr int R = 1 << Rx::lr(NS - 1);
        return pos<NS - 1>(tp, r / R, r % R);
    }
};

}  // namespace rsw
