// Stage structure of the block FFT, shared by the device kernels, the host
// twiddle-table builder and the device table builder of the no-allocation
// entry point, so that all three agree on one layout.
//
// A block of length L = 2^log_l is transformed in NS = ceil(log_l / 4)
// stages: radix-16 stages first, the remaining radix 2/4/8/16 last. Stage s
// has radix R_s = 2^lr(s) and stride S_s = 2^ls(s), with
// ls(s) = log_l - (lr(0) + ... + lr(s)); the last stage has stride 1.
// Forward stages are decimation in frequency (large strides first), so the
// spectrum ends up in digit-reversed order: position p holds frequency
//     f = sum_s digit_s(p) * R_0 * ... * R_{s-1},   digit_s(p) = (p >> ls(s)) mod R_s.
//
// Twiddles W_{R S}^{j q} (q = 1..R-1, j < S) of every stage but the last are
// stored per stage: direct [(q-1) S + j] for S <= 2^RSW_DIRECT_MAX_LS,
// otherwise factored into W^{(j & 63) q} at [(q-1) 64 + (j & 63)] and
// W^{64 (j >> 6) q} at [(R-1) 64 + (q-1) (S/64) + (j >> 6)].
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define RSW_HD __host__ __device__
#else
#define RSW_HD
#endif

namespace rsw {

constexpr int RSW_DIRECT_MAX_LS = 7;

RSW_HD constexpr int stage_count(int log_l) { return log_l <= 0 ? 0 : (log_l + 3) / 4; }
RSW_HD constexpr int stage_lr(int log_l, int s) {
    return s < stage_count(log_l) - 1 ? 4 : log_l - 4 * (stage_count(log_l) - 1);
}
RSW_HD constexpr int stage_ls(int log_l, int s) { return s < stage_count(log_l) - 1 ? log_l - 4 * (s + 1) : 0; }
RSW_HD constexpr bool stage_direct(int log_l, int s) { return stage_ls(log_l, s) <= RSW_DIRECT_MAX_LS; }
// twiddle entries of stage s (none for the last stage)
RSW_HD constexpr int stage_tw_entries(int log_l, int s) {
    return s >= stage_count(log_l) - 1 ? 0
           : stage_direct(log_l, s)
               ? ((1 << stage_lr(log_l, s)) - 1) << stage_ls(log_l, s)
               : ((1 << stage_lr(log_l, s)) - 1) * (64 + (1 << (stage_ls(log_l, s) - 6)));
}
RSW_HD constexpr int stage_tw_offset(int log_l, int s) {
    int o = 0;
    for (int t = 0; t < s; ++t) o += stage_tw_entries(log_l, t);
    return o;
}

// exponent m and modulus R*S of table entry k of stage s: the entry is W_{RS}^m
RSW_HD inline void stage_tw_entry(int log_l, int s, int64_t k, int64_t *m, int64_t *mod) {
    const int64_t R = int64_t(1) << stage_lr(log_l, s), S = int64_t(1) << stage_ls(log_l, s);
    *mod = R * S;
    if (stage_direct(log_l, s)) {
        *m = (k / S + 1) * (k % S);
    } else if (k < (R - 1) * 64) {
        *m = (k / 64 + 1) * (k % 64);
    } else {
        const int64_t kk = k - (R - 1) * 64;
        *m = (kk / (S / 64) + 1) * 64 * (kk % (S / 64));
    }
}

// Frequency index held at block position p after the forward stages. The map
// is a permutation of the bits of p, so positions with disjoint bits map to
// frequencies with disjoint bits: digitrev(a | b) == digitrev(a) | digitrev(b).
RSW_HD constexpr int digitrev_c(int p, int log_l) {
    int f = 0, sh = 0;
    for (int s = 0; s < stage_count(log_l); ++s) {
        const int lr = stage_lr(log_l, s);
        f |= ((p >> stage_ls(log_l, s)) & ((1 << lr) - 1)) << sh;
        sh += lr;
    }
    return f;
}
RSW_HD inline int64_t digitrev_rt(int64_t p, int log_l) {
    const int ns = stage_count(log_l);
    int64_t f = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = stage_lr(log_l, s);
        f |= ((p >> stage_ls(log_l, s)) & ((int64_t(1) << lr) - 1)) << sh;
        sh += lr;
    }
    return f;
}
// Inverse of digitrev_rt: frequency index -> block position.
RSW_HD inline int64_t digitpos_rt(int64_t f, int log_l) {
    const int ns = stage_count(log_l);
    int64_t p = 0;
    int sh = 0;
    for (int s = 0; s < ns; ++s) {
        const int lr = stage_lr(log_l, s);
        p |= ((f >> sh) & ((int64_t(1) << lr) - 1)) << stage_ls(log_l, s);
        sh += lr;
    }
    return p;
}

}  // namespace rsw
