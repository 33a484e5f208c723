// Block FFT building blocks for the split-step passes (sm_100a).
//
// A "block" transforms C independent sequences of length L = 2^LOG_L held by
// one CTA. Each thread owns E = 8, 16 or 32 elements in registers; stages are
// radix-8 (E = 8) or radix-16, the last one takes the remaining radix
// (rsw_stages.h).
// Forward stages are decimation in frequency: natural order in,
// digit-reversed order out. Inverse stages are the exact mirror (decimation
// in time): digit-reversed in, natural out, so a forward/inverse pair needs
// no reordering and the propagator is applied to the digit-reversed spectrum
// in registers.
//
// Stage s has radix R_s = 2^lr(s) and stride S_s = 2^ls(s). Butterfly beta
// of stage s touches positions
//     (beta >> ls) * R*S + (beta & (S-1)) + q*S,   q = 0..R-1
// and is done by one thread, which reads and writes the same positions.
// Only the exchange between stages 0 and 1 spans the whole sequence; every
// later exchange stays inside a block of stage s, owned by a contiguous
// group of threads (Radix::beta), and is ordered by a barrier of that group
// alone: a warp or less for all but the longest blocks, so warps run through
// the inner stages without waiting for each other.
//
// Inside a butterfly the radix-R DFT is a radix-2 network in registers: the
// forward network takes natural order and leaves bit-reversed order (register
// brev(q) holds output q), the inverse network takes bit-reversed order and
// leaves natural order, so no register permutation is ever needed.
//
// Twiddles W_{RS}^{jq} of stage s live in shared memory, loaded once per CTA:
// a direct table [(q-1)*S + j] for strides S <= 128 (512 for complex64),
// otherwise two factors W^{(j mod 64) q} * W^{64 (j div 64) q} of 64 and S/64
// entries per q. FP64 butterflies may take only W^j from the tables and form
// the other powers as a running product (running()).
//
// Complex64 blocks rotate by lifting instead of complex multiplication: a
// rotation by theta is three shears xr += a xi; xi += b xr; xr += a xi with
// a = -tan(theta/2), b = sin(theta) (|theta| <= pi/2; a half turn s = -1 is
// taken out first). Three shears have determinant exactly 1 whatever the
// rounding of a and b, and the inverse rotation is the same shears with -a,
// -b in reverse order, so a forward/inverse pair undoes itself up to the
// rounding of the data. A complex product by the FP32-rounded (cos, sin)
// scales by |w|^2 = 1 + O(2^-24) instead, the same factor at every split
// step; over the hundreds of thin split steps of a sample that bias grows
// linearly and dominated the complex64 detector error (lifting: growth like
// the square root of the step count, measured 17x smaller after 200 steps in
// a float32 model of the forward/inverse pair). Table entries of complex64
// blocks are {a, b}. Angles beyond a quarter turn (tw_mode, rsw_stages.h)
// take a fixed quarter turn in the code where the output index q bounds the
// angle below a half turn, and otherwise a half-turn flag in the lowest
// mantissa bit of a (a is rounded to the nearest float of that parity: the
// rotation angle moves by at most one ulp of a, the same in the forward and
// the inverse pass, and the shears keep determinant 1); complex128 blocks
// keep {cos, sin}.
//
// Shared memory holds the C sequences with one pad element per E (phys(p):
// the last stage gives consecutive threads positions E apart, which the pad
// moves to neighbouring banks) and a per-sequence pitch chosen so that the
// accesses of one wavefront hit distinct banks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

#include "rsw_stages.h"

namespace rsw {

template <typename R> struct CxT;
template <> struct CxT<double> { using T = double2; };
template <> struct CxT<float> { using T = float2; };
// block twiddle table entry: {cos, sin} (FP64) or the lifting form {a, b}
// with the half turn in the low bit of a (FP32)
template <typename R> struct TwT;
template <> struct TwT<double> { using T = double2; };
template <> struct TwT<float> { using T = float2; };
// 16-byte entry of the per-row and per-tile factor tables and of the chirp
// table: {cos, sin} (FP64) or the lifting form {a, b, s, 0} (FP32)
template <typename R> struct LiftT;
template <> struct LiftT<double> { using T = double2; };
template <> struct LiftT<float> { using T = float4; };

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
// complex64: packed FP32x2 arithmetic (one instruction per complex add, sub
// or real scale); b * -1 + a rounds exactly like a - b
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }

// ------------------------------------------------------------ lifting
// x * exp(i theta) as three shears, a = -tan(theta/2), b = sin(theta)
__device__ __forceinline__ float2 lift(float2 x, float a, float b) {
    x.x = __fmaf_rn(a, x.y, x.x);
    x.y = __fmaf_rn(b, x.x, x.y);
    x.x = __fmaf_rn(a, x.y, x.x);
    return x;
}
// rotation by a 16-byte factor-table entry w = {a, b, s, -} (s: half turn,
// times an optional power-of-two scale, exact) and its inverse (same shears,
// -a and -b)
__device__ __forceinline__ float2 rot(float2 x, float4 w) { return lift(cscale(x, w.z), w.x, w.y); }
__device__ __forceinline__ float2 rot_inv(float2 x, float4 w) { return lift(cscale(x, w.z), -w.x, -w.y); }
// Lifting form of a unit complex number given in FP64: the half turn goes to
// s when Re w < 0 (then |theta| <= pi/2 and |a| <= 1); `scale` (a power of
// two) is folded into s. a = -Im w / (1 + Re w) with 1 + Re w in [1, 2]: the
// FP32 reciprocal refined by one Newton step in FP64 (relative error below
// 1e-14, then a single rounding to FP32), a few registers and no division.
__device__ __forceinline__ float4 lift_of(double2 w, double scale = 1.0) {
    double sg = scale;
    if (w.x < 0.0) {
        w.x = -w.x;
        w.y = -w.y;
        sg = -sg;
    }
    const double d = 1.0 + w.x;
    double r = double(__frcp_rn(float(d)));
    r = fma(r, fma(-d, r, 1.0), r);
    return make_float4(float(-w.y * r), float(w.y), float(sg), 0.f);
}
// +-1.0f from the half-turn bit of a packed block twiddle {a, b} (the low bit
// of a), and the product of the half turns of two entries
__device__ __forceinline__ float half_turn(float a) {
    return __uint_as_float((__float_as_uint(a) << 31) | 0x3f800000u);
}
__device__ __forceinline__ float half_turn2(float a, float b) {
    return __uint_as_float(((__float_as_uint(a) ^ __float_as_uint(b)) << 31) | 0x3f800000u);
}
__device__ __forceinline__ float2 rot(float2 x, float2 w) { return lift(cscale(x, half_turn(w.x)), w.x, w.y); }
__device__ __forceinline__ float2 rot_inv(float2 x, float2 w) { return lift(cscale(x, half_turn(w.x)), -w.x, -w.y); }
// multiply by i^q (q mod 4), exact
template <int Q> __device__ __forceinline__ float2 quarter(float2 x) {
    constexpr int q = ((Q % 4) + 4) % 4;
    if constexpr (q == 0) return x;
    else if constexpr (q == 1) return make_float2(-x.y, x.x);
    else if constexpr (q == 2) return make_float2(-x.x, -x.y);
    else return make_float2(x.y, -x.x);
}

__host__ __device__ constexpr int brev_bits(int q, int bits) {
    int r = 0;
    for (int b = 0; b < bits; ++b) r |= ((q >> b) & 1) << (bits - 1 - b);
    return r;
}
__host__ __device__ constexpr int ilog2(int r) { return r <= 1 ? 0 : 1 + ilog2(r >> 1); }

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

// Complex64: the same rotations by lifting. The forward rotation
// exp(-i pi e / 8) is i^q * exp(i t pi / 8) with |t| <= 2 (t = -e - 4q),
// applied as the shears of t, then the exact quarter turns; the inverse
// (DIR = +1) is its exact mirror: the quarter turns back, then the shears
// with negated coefficients.
template <int DIR, int EE> __device__ __forceinline__ float2 tw16_lift(float2 x) {
    constexpr int q = EE <= 2 ? 0 : EE <= 6 ? -1 : -2;
    constexpr int t = -EE - 4 * q;
    constexpr float A1 = 0.19891236737965800691f;  // tan(pi/16)
    constexpr float B1 = 0.38268343236508977173f;  // sin(pi/8)
    constexpr float A2 = 0.41421356237309504880f;  // tan(pi/8)
    constexpr float B2 = 0.70710678118654752440f;  // sin(pi/4)
    constexpr float a = t == -2 ? A2 : t == -1 ? A1 : t == 1 ? -A1 : 0.f;
    constexpr float b = t == -2 ? -B2 : t == -1 ? -B1 : t == 1 ? B1 : 0.f;
    if constexpr (DIR < 0) {
        if constexpr (t != 0) x = lift(x, a, b);
        return quarter<q>(x);
    } else {
        x = quarter<-q>(x);
        if constexpr (t != 0) x = lift(x, -a, -b);
        return x;
    }
}
template <int DIR> __device__ __forceinline__ float2 tw16(float2 x, int e) {
    switch (e) {
    case 0: return x;
    case 1: return tw16_lift<DIR, 1>(x);
    case 2: return tw16_lift<DIR, 2>(x);
    case 3: return tw16_lift<DIR, 3>(x);
    case 4: return tw16_lift<DIR, 4>(x);
    case 5: return tw16_lift<DIR, 5>(x);
    case 6: return tw16_lift<DIR, 6>(x);
    default: return tw16_lift<DIR, 7>(x);
    }
}

// Radix-2 decimation-in-frequency network: natural order in, bit-reversed out.
template <int R, int DIR, typename C> __device__ __forceinline__ void net_dif(C *v) {
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
}
// Radix-2 decimation-in-time network: bit-reversed order in, natural out.
template <int R, int DIR, typename C> __device__ __forceinline__ void net_dit(C *v) {
#pragma unroll
    for (int span = 1; span < R; span <<= 1) {
#pragma unroll
        for (int start = 0; start < R; start += 2 * span) {
#pragma unroll
            for (int k = 0; k < span; ++k) {
                C a = v[start + k], b = tw16<DIR>(v[start + k + span], k * (8 / span));
                v[start + k] = cadd(a, b);
                v[start + k + span] = csub(a, b);
            }
        }
    }
}

// Radix structure of a block of length 2^LOG_L with E_ elements per thread
// (the stage structure and twiddle layout do not depend on E_).
template <int LOG_L, int E_ = 16, int MAX_LS = 7> struct Radix {
    static_assert(LOG_L >= 4, "blocks hold at least 16 elements");
    static_assert(E_ == 8 || E_ == 16 || E_ == 32, "8, 16 or 32 elements per thread");
    static constexpr int L = 1 << LOG_L;
    static constexpr int E = E_;
    static constexpr int RB = digit_bits(E_);  // radix 2^RB stages
    static constexpr int T = L / E;  // threads per sequence
    static constexpr int NS = stage_count(LOG_L, RB);
    __host__ __device__ static constexpr int lr(int s) { return stage_lr(LOG_L, s, RB); }
    __host__ __device__ static constexpr int ls(int s) { return stage_ls(LOG_L, s, RB); }
    __host__ __device__ static constexpr bool direct(int s) { return stage_direct(LOG_L, s, MAX_LS, RB); }
    __host__ __device__ static constexpr int twoff(int s) { return stage_tw_offset(LOG_L, s, MAX_LS, RB); }
    static constexpr int TW = twoff(NS - 1) > 0 ? twoff(NS - 1) : 1;
    // butterflies per thread in stage s
    __host__ __device__ static constexpr int M(int s) { return E >> lr(s); }
    // Butterfly i of thread tp in stage s. Stage 0 strides by T (consecutive
    // threads touch consecutive positions: coalesced global access); later
    // stages give each thread M consecutive butterflies, so that every block
    // of stage s (R_s * S_s positions) belongs to a contiguous, aligned range
    // of R_s * S_s / E threads and the exchange after stage s stays inside it.
    __host__ __device__ static constexpr int beta(int s, int tp, int i) { return s == 0 ? tp + T * i : tp * M(s) + i; }
    // threads of one sequence that exchange data between stages s and s + 1
    __host__ __device__ static constexpr int group(int s) { return s == 0 ? T : (1 << (lr(s) + ls(s))) / E; }
};

template <typename Real, int LOG_L, int C, int E_ = 16>
struct Block : Radix<LOG_L, E_, direct_max_ls(2 * sizeof(Real), LOG_L)> {
    using Rx = Radix<LOG_L, E_, direct_max_ls(2 * sizeof(Real), LOG_L)>;
    using Cx = typename CxT<Real>::T;
    using Tw = typename TwT<Real>::T;  // twiddle table entry (16 bytes)
    static constexpr bool LIFT = sizeof(Real) == 4;  // complex64: rotations by lifting
    using Rx::E;
    using Rx::L;
    using Rx::NS;
    using Rx::T;
    static constexpr int NT = T * C;  // threads per CTA
    static constexpr int W = 32 / int(sizeof(Cx) / 4);  // elements per smem wavefront
    static constexpr int LOG_E = ilog2(E_);
    static constexpr int BASE = L + (L >> LOG_E);
    static constexpr int WANT = (C >= W) ? 1 : W / C;
    static constexpr int PITCH = BASE + (((WANT - BASE) % W) + W) % W;
    static constexpr size_t DATA = size_t(C) * PITCH * sizeof(Cx);
    static constexpr size_t SMEM = DATA + size_t(Rx::TW) * sizeof(Tw);
    static constexpr int RL = 1 << Rx::lr(NS - 1);  // radix of the last stage

    __device__ static __forceinline__ int phys(int p) { return p + (p >> LOG_E); }

    template <int s> __device__ static __forceinline__ int pos(int tp, int i, int q) {
        constexpr int LRS = Rx::lr(s), LSS = Rx::ls(s);
        const int beta = Rx::beta(s, tp, i);
        const int j = beta & ((1 << LSS) - 1);
        const int b = beta >> LSS;
        return (b << (LRS + LSS)) + j + (q << LSS);
    }
    // register holding position q of butterfly i: natural or bit-reversed layout
    template <int s, bool BR> __device__ static constexpr int reg(int i, int q) {
        constexpr int R = 1 << Rx::lr(s);
        return i * R + (BR ? brev_bits(q, Rx::lr(s)) : q);
    }

    template <int s, bool BR> __device__ static __forceinline__ void st(Cx *sm, int tp, const Cx *v) {
        constexpr int R = 1 << Rx::lr(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i)
#pragma unroll
            for (int q = 0; q < R; ++q) sm[phys(pos<s>(tp, i, q))] = v[reg<s, BR>(i, q)];
    }
    template <int s, bool BR> __device__ static __forceinline__ void ld(const Cx *sm, int tp, Cx *v) {
        constexpr int R = 1 << Rx::lr(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i)
#pragma unroll
            for (int q = 0; q < R; ++q) v[reg<s, BR>(i, q)] = sm[phys(pos<s>(tp, i, q))];
    }

    // twiddle W_{RS}^{j q} of stage s from the shared-memory tables (complex128)
    template <int s> __device__ static __forceinline__ Cx twid(const Tw *tw, int j, int q) {
        constexpr int LSS = Rx::ls(s);
        const Cx *t = tw + Rx::twoff(s);
        if constexpr (Rx::direct(s)) {
            return t[((q - 1) << LSS) + j];
        } else {
            constexpr int R = 1 << Rx::lr(s);
            const Cx a = t[(q - 1) * 64 + (j & 63)];
            const Cx b = t[(R - 1) * 64 + (q - 1) * (1 << (LSS - 6)) + (j >> 6)];
            return cmul(a, b);
        }
    }
    // complex64: x * W_{RS}^{j q} (INV: x * conj(W)) by lifting, with the
    // entry's tw_mode (q is a constant after unrolling): mode 1 adds the fixed
    // quarter turn, mode 2 the half turn of the entry's flag. A factored
    // twiddle is two rotations (the low factor is mode 0), undone in reverse
    // order by the inverse.
    template <bool INV> __device__ static __forceinline__ Cx rot_mode(Cx x, Tw w, int mode) {
        if (mode == 2) x = cscale(x, half_turn(w.x));
        if (INV) {
            if (mode == 1) x = quarter<1>(x);
            return lift(x, -w.x, -w.y);
        }
        x = lift(x, w.x, w.y);
        return mode == 1 ? quarter<-1>(x) : x;
    }
    template <int s, bool INV> __device__ static __forceinline__ Cx twlift(const Tw *tw, int j, int q, Cx x) {
        constexpr int LSS = Rx::ls(s);
        constexpr int R = 1 << Rx::lr(s);
        const Tw *t = tw + Rx::twoff(s);
        const int mode = tw_mode(q, R);
        if constexpr (Rx::direct(s)) {
            return rot_mode<INV>(x, t[((q - 1) << LSS) + j], mode);
        } else {
            static_assert(LSS >= 8, "factored stages have strides >= 256 (low factors below a quarter turn)");
            const Tw a = t[(q - 1) * 64 + (j & 63)];
            const Tw b = t[(R - 1) * 64 + (q - 1) * (1 << (LSS - 6)) + (j >> 6)];
            if constexpr (INV) return lift(rot_mode<true>(x, b, mode), -a.x, -a.y);
            else return rot_mode<false>(lift(x, a.x, a.y), b, mode);
        }
    }

    // FP64 twiddles as the running product W^(jq) = W^(j(q-1)) W^j (error
    // below R ulp): one table lookup per butterfly instead of R - 1. For
    // factored stages this takes as many complex products as the two-factor
    // lookups. Radix-8 blocks of 2^10 and more (the 1024-thread complex128
    // column kernels, held back by shared-memory instruction issue) also
    // trade the direct lookups for R - 2 products: 7 % faster at 2^11.
    // complex64 keeps the lookups.
    template <int s> static constexpr bool running() {
        return sizeof(Real) == 8 && (!Rx::direct(s) || (E == 8 && LOG_L >= 10));
    }

    // forward stage s: natural in -> radix-R DFT -> bit-reversed out, twiddled
    template <int s> __device__ static __forceinline__ void dif(int tp, Cx *v, const Tw *tw) {
        constexpr int R = 1 << Rx::lr(s);
        constexpr int LSS = Rx::ls(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i) {
            net_dif<R, -1>(v + i * R);
            if constexpr (s < NS - 1) {
                const int j = Rx::beta(s, tp, i) & ((1 << LSS) - 1);
                if constexpr (running<s>()) {
                    const Cx w1 = twid<s>(tw, j, 1);
                    Cx w = w1;
#pragma unroll
                    for (int q = 1; q < R; ++q) {
                        Cx &x = v[reg<s, true>(i, q)];
                        x = cmul(x, w);
                        if (q < R - 1) w = cmul(w, w1);
                    }
                } else {
#pragma unroll
                    for (int q = 1; q < R; ++q) {
                        Cx &x = v[reg<s, true>(i, q)];
                        if constexpr (LIFT) x = twlift<s, false>(tw, j, q, x);
                        else x = cmul(x, twid<s>(tw, j, q));
                    }
                }
            }
        }
    }
    // inverse stage s: bit-reversed in -> conjugate twiddle -> inverse DFT -> natural out
    template <int s> __device__ static __forceinline__ void dit(int tp, Cx *v, const Tw *tw) {
        constexpr int R = 1 << Rx::lr(s);
        constexpr int LSS = Rx::ls(s);
#pragma unroll
        for (int i = 0; i < E / R; ++i) {
            if constexpr (s < NS - 1) {
                const int j = Rx::beta(s, tp, i) & ((1 << LSS) - 1);
                if constexpr (running<s>()) {
                    const Cx w1 = twid<s>(tw, j, 1);
                    Cx w = w1;
#pragma unroll
                    for (int q = 1; q < R; ++q) {
                        Cx &x = v[reg<s, true>(i, q)];
                        x = cmulc(x, w);
                        if (q < R - 1) w = cmul(w, w1);
                    }
                } else {
#pragma unroll
                    for (int q = 1; q < R; ++q) {
                        Cx &x = v[reg<s, true>(i, q)];
                        if constexpr (LIFT) x = twlift<s, true>(tw, j, q, x);
                        else x = cmulc(x, twid<s>(tw, j, q));
                    }
                }
            }
            net_dit<R, +1>(v + i * R);
        }
    }

    // Barrier of the exchange between stages s and s + 1 (either direction).
    // The exchanging threads form aligned groups of Rx::group(s) * C
    // consecutive threads (threads are numbered tp * C + c): one warp or less
    // synchronises with __syncwarp, larger groups with a named barrier of
    // their own, the whole CTA with __syncthreads. Each position is written
    // in a stage only by the thread that read it in that stage, so one
    // barrier per exchange orders every access. With more than 15 groups
    // (named barriers 1..15) aligned pairs, quadruples, ... of groups share
    // one barrier.
    static constexpr int sync_lanes(int g) { return g >= NT || g <= 32 || NT / g <= 15 ? g : sync_lanes(2 * g); }
    template <int s> __device__ static __forceinline__ void exchange_sync() {
        constexpr int G = sync_lanes(Rx::group(s) * C);
        if constexpr (G >= NT) {
            __syncthreads();
        } else if constexpr (G <= 32) {
            __syncwarp();
        } else {
            static_assert(NT / G <= 15, "named barriers 1..15");
            asm volatile("bar.sync %0, %1;" ::"r"(1 + int(threadIdx.x) / G), "r"(G) : "memory");
        }
    }

    // Full forward transform from stage-0 positions (natural layout) to
    // last-stage positions (bit-reversed layout) in registers.
    template <int s = 0> __device__ static __forceinline__ void forward(Cx *sm, int tp, Cx *v, const Tw *tw) {
        dif<s>(tp, v, tw);
        if constexpr (s < NS - 1) {
            st<s, true>(sm, tp, v);
            exchange_sync<s>();
            ld<s + 1, false>(sm, tp, v);
            forward<s + 1>(sm, tp, v, tw);
        }
    }
    // Full inverse transform from last-stage positions (bit-reversed layout)
    // to stage-0 positions (natural layout).
    template <int s = NS - 1> __device__ static __forceinline__ void inverse(Cx *sm, int tp, Cx *v, const Tw *tw) {
        dit<s>(tp, v, tw);
        if constexpr (s > 0) {
            st<s, false>(sm, tp, v);
            exchange_sync<s - 1>();
            ld<s - 1, true>(sm, tp, v);
            inverse<s - 1>(sm, tp, v, tw);
        }
    }

    // position held by register r in the natural layout of stage 0 and in the
    // bit-reversed layout of the last stage
    __device__ static __forceinline__ int first_pos(int tp, int r) {
        constexpr int R = 1 << Rx::lr(0);
        return pos<0>(tp, r / R, r % R);
    }
    __device__ static __forceinline__ int last_pos(int tp, int r) {
        constexpr int LRL = Rx::lr(NS - 1);
        return pos<NS - 1>(tp, r / RL, brev_bits(r % RL, LRL));
    }
    // Frequency index of last_pos(tp, r). The last stage gives thread tp the
    // E consecutive positions tp*E + last_off(r), so the frequency splits into
    // a per-thread part and a compile-time part with disjoint bits:
    // last_freq(tp, r) == freq_base(tp) | freq_off(r).
    static constexpr int last_off(int r) { return (r / RL) * RL + brev_bits(r % RL, Rx::lr(NS - 1)); }
    static constexpr int freq_off(int r) { return digitrev_c(last_off(r), LOG_L, Rx::RB); }
    __device__ static __forceinline__ int freq_base(int tp) { return digitrev_c(tp * E, LOG_L, Rx::RB); }
    __device__ static __forceinline__ int last_freq(int tp, int r) { return freq_base(tp) | freq_off(r); }

    // copy the block's twiddle tables (global, host-built layout) into shared memory
    __device__ static __forceinline__ void load_twiddles(Tw *tw_sm, const Tw *__restrict__ tw_g) {
        for (int k = threadIdx.x; k < Rx::TW; k += NT) tw_sm[k] = tw_g[k];
    }
};

}  // namespace rsw
