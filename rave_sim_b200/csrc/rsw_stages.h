// Stage structure of the block FFT, shared by the device kernels, the host
// twiddle-table builder and the device table builder of the no-allocation
// entry point, so that all three agree on one layout.
//
// A block of length L = 2^log_l is transformed in NS = ceil(log_l / rb)
// stages of digit width rb (radix 2^rb: 16 for kernels with 16 or 32 samples
// per thread, 8 for 8 samples per thread), the remainder radix last. Stage s
// has radix R_s = 2^lr(s) and stride S_s = 2^ls(s), with
// ls(s) = log_l - (lr(0) + ... + lr(s)); the last stage has stride 1.
// Forward stages are decimation in frequency (large strides first), so the
// spectrum ends up in digit-reversed order: position p holds frequency
//     f = sum_s digit_s(p) * R_0 * ... * R_{s-1},   digit_s(p) = (p >> ls(s)) mod R_s.
//
// Twiddles W_{R S}^{j q} (q = 1..R-1, j < S) of every stage but the last are
// stored per stage: direct [(q-1) S + j] for S <= 2^max_ls, otherwise
// factored into W^{(j & 63) q} at [(q-1) 64 + (j & 63)] and
// W^{64 (j >> 6) q} at [(R-1) 64 + (q-1) (S/64) + (j >> 6)]. max_ls depends
// on the element size (direct_max_ls): complex64 tables stay direct up to
// strides of 512 (61 KB), complex128 ones up to 128 (30 KB).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define RSW_HD __host__ __device__
#else
#define RSW_HD
#endif

namespace rsw {

// Complex64 blocks of 2^13 (the two-level rows) use the factored form above
// 2^7 too: their smaller tables let two 512-thread CTAs share an SM.
RSW_HD constexpr int direct_max_ls(int elem_bytes, int log_l = 0) {
    return elem_bytes <= 8 && log_l != 13 ? 9 : 7;
}

// digit width of the kernels with e samples per thread
RSW_HD constexpr int digit_bits(int e) { return e == 8 ? 3 : 4; }

RSW_HD constexpr int stage_count(int log_l, int rb = 4) { return log_l <= 0 ? 0 : (log_l + rb - 1) / rb; }
RSW_HD constexpr int stage_lr(int log_l, int s, int rb = 4) {
    return s < stage_count(log_l, rb) - 1 ? rb : log_l - rb * (stage_count(log_l, rb) - 1);
}
RSW_HD constexpr int stage_ls(int log_l, int s, int rb = 4) {
    return s < stage_count(log_l, rb) - 1 ? log_l - rb * (s + 1) : 0;
}
RSW_HD constexpr bool stage_direct(int log_l, int s, int max_ls, int rb = 4) { return stage_ls(log_l, s, rb) <= max_ls; }
// twiddle entries of stage s (none for the last stage)
RSW_HD constexpr int stage_tw_entries(int log_l, int s, int max_ls, int rb = 4) {
    return s >= stage_count(log_l, rb) - 1 ? 0
           : stage_direct(log_l, s, max_ls, rb)
               ? ((1 << stage_lr(log_l, s, rb)) - 1) << stage_ls(log_l, s, rb)
               : ((1 << stage_lr(log_l, s, rb)) - 1) * (64 + (1 << (stage_ls(log_l, s, rb) - 6)));
}
RSW_HD constexpr int stage_tw_offset(int log_l, int s, int max_ls, int rb = 4) {
    int o = 0;
    for (int t = 0; t < s; ++t) o += stage_tw_entries(log_l, t, max_ls, rb);
    return o;
}

// exponent m and modulus R*S of table entry k of stage s: the entry is W_{RS}^m
RSW_HD inline void stage_tw_entry(int log_l, int s, int max_ls, int rb, int64_t k, int64_t *m, int64_t *mod) {
    const int64_t R = int64_t(1) << stage_lr(log_l, s, rb), S = int64_t(1) << stage_ls(log_l, s, rb);
    *mod = R * S;
    if (stage_direct(log_l, s, max_ls, rb)) {
        *m = (k / S + 1) * (k % S);
    } else if (k < (R - 1) * 64) {
        *m = (k / 64 + 1) * (k % 64);
    } else {
        const int64_t kk = k - (R - 1) * 64;
        *m = (kk / (S / 64) + 1) * 64 * (kk % (S / 64));
    }
}

// How a complex64 lifting entry (rsw_block_fft.cuh) covers angles beyond a
// quarter turn. Twiddle q of a radix-R stage, W_{RS}^{jq} with j < S, has an
// angle in (-2 pi q / R, 0]:
//   mode 0 (4q <= R):  within (-pi/2, 0]: the entry is the rotation itself;
//   mode 1 (2q <= R):  within (-pi, 0]: the entry rotates by the angle + pi/2
//                      and the kernel follows it with a fixed quarter turn -i;
//   mode 2 (q > R/2):  the entry carries a half-turn flag in the low bit of a.
// The low factors W^{(j mod 64) q} of factored stages (S >= 256) stay below
// a quarter turn: mode 0.
RSW_HD constexpr int tw_mode(int q, int r) { return 4 * q <= r ? 0 : 2 * q <= r ? 1 : 2; }
RSW_HD inline int stage_tw_mode(int log_l, int s, int max_ls, int rb, int64_t k) {
    const int64_t R = int64_t(1) << stage_lr(log_l, s, rb), S = int64_t(1) << stage_ls(log_l, s, rb);
    if (stage_direct(log_l, s, max_ls, rb)) return tw_mode(int(k / S + 1), int(R));
    if (k < (R - 1) * 64) return 0;
    return tw_mode(int((k - (R - 1) * 64) / (S / 64) + 1), int(R));
}

// Frequency index held at block position p after the forward stages. The map
// is a permutation of the bits of p, so positions with disjoint bits map to
// frequencies with disjoint bits: digitrev(a | b) == digitrev(a) | digitrev(b).
RSW_HD constexpr int digitrev_c(int p, int log_l, int rb = 4) {
    int f = 0, sh = 0;
    for (int s = 0; s < stage_count(log_l, rb); ++s) {
        const int lr = stage_lr(log_l, s, rb);
        f |= ((p >> stage_ls(log_l, s, rb)) & ((1 << lr) - 1)) << sh;
        sh += lr;
    }
    return f;
}
RSW_HD inline int64_t digitrev_rt(int64_t p, int log_l, int rb = 4) {
    const int ns = stage_count(log_l, rb);
    int64_t f = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = stage_lr(log_l, s, rb);
        f |= ((p >> stage_ls(log_l, s, rb)) & ((int64_t(1) << lr) - 1)) << sh;
        sh += lr;
    }
    return f;
}
// Inverse of digitrev_rt: frequency index -> block position.
RSW_HD inline int64_t digitpos_rt(int64_t f, int log_l, int rb = 4) {
    const int ns = stage_count(log_l, rb);
    int64_t p = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = stage_lr(log_l, s, rb);
        p |= ((f >> sh) & ((int64_t(1) << lr) - 1)) << stage_ls(log_l, s, rb);
        sh += lr;
    }
    return p;
}

}  // namespace rsw
