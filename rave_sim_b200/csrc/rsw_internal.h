// Internal structures shared by the host library (rsw_host.cpp) and the CUDA
// kernels (rsw_kernels.cu). Not part of the public ABI.
#pragma once

#include <stdint.h>
#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

namespace rsw {

enum TransKind : int {
    TR_NONE = 0,
    TR_SCALAR = 1,   // u *= fa
    TR_GRATING = 2,  // u *= mask ? fa : fb, mask = mod(x/p + dc/2, 1) < dc
    TR_DBA = 3,      // mask = (mod(x/p0 + dc0/2,1) < dc0) & (mod(x/p1,1) < dc1)
    TR_SAMPLE = 4,   // u *= exp(i y * interp(x, row_x, row_db, 0, 0))
};

// Transmission through one grating sub-step, a substrate, or one sample row.
struct TransArgs {
    int kind;
    double2 fa, fb;  // material factors
    // grating coordinates: per-chunk np.linspace (start, step)
    double pitch0, pitch1, half_dc0, dc0, dc1;
    double inv_pitch0, inv_pitch1;       // 1/pitch (correctly rounded), for the corrected quotient
    int64_t chunk_size;  // >= N: single chunk
    double xstart0, step0;               // single-chunk values
    const double *chunk_xstart;          // per-chunk tables (device) when several chunks
    const double *chunk_step;
    int64_t half_n_floor;                // N // 2 (integer)
    // sample row
    double dx;                           // field sampling
    double half_n;                       // N / 2 (float)
    double psx, sample_xpos, sample_hw;  // row_x[j] = (j*psx + xpos) - hw
    double sample_inv_psx;
    int64_t x_len;
    const int8_t *row_grid;              // grid row (device)
    const double2 *mat_db;               // deltabeta per material index (device), [0] = vacuum
    const double2 *mat_factor;           // exp(i y db) per material index (device)
    double sample_y;                     // 2 pi dz / wl
};

// Fresnel propagator of one split step (applied in the row pass).
struct PropArgs {
    int has_h;          // multiply by the transfer function
    int has_cut;        // zero the cutoff range
    double c;           // fl(fl(pi*wl)*dz)
    double2 A;          // exp(-i 2 pi dz / wl)
    double fac;         // 1.0 / N
    double dx;
    double rdx;         // 1.0 / dx
    int64_t cut_lo, cut_hi;  // zero natural frequency indices k in [cut_lo, cut_hi)
    // Chirp form of the transfer function (two-level plans): phase in turns
    // G * ks^2, G = c / (2 pi N^2 dx^2) as a double-double, ks = kbase + M k2s;
    // h3 = exp(2 pi i G M^2 k2s^2) in the row kernel's register order, M = N1 Nb.
    int chirp;
    double g_hi, g_lo;
    const void *h3;
    // Exact angular-spectrum kernel (opt-in; not in the reference): H = A
    // exp(i phi), phi = z2pi fx^2 / (inv_wl + sqrt(inv_wl2 - fx^2)), evaluated
    // per sample (no chirp form); evanescent fx^2 >= inv_wl2 is zeroed.
    int exact;
    double inv_wl, inv_wl2, z2pi;
};

enum PassFlags : int {
    PF_FWD = 1,       // run the forward transform of this level
    PF_INV = 2,       // run the inverse transform of this level
    PF_TW = 4,        // four-step twiddle: column, after fwd: W_M^(n2 k1); row, after inv:
                      // conj(W_M^(n2 tw_k)) (hi factors times tw_scale)
    PF_TRANS = 8,     // apply transmission (column: between inv and fwd; single-level row: before fwd)
    PF_SCALE = 16,    // single-level row: multiply by 1/N after the inverse
    PF_ONES = 32,     // input is the plane wave u = 1 (input buffer not read)
    PF_SPEC_IN = 64,  // row: input is a spectrum (digit-reversed layout), start with the inverse
    PF_TWI = 128,     // column: before the inverse, conj(W_M^(n2 k1)) * tw_scale
    PF_TWF = 256,     // row: before the forward, W_M^(n2 tw_k) (the conjugate of PF_TW's factor)
    PF_NOSTORE = 512, // column detection pass: bin the field only, do not write it
};

// Per-instance values of a batched pass: several sources with the same
// field length and element geometry (the energies of one field length) run
// in lockstep, each transform of the batch one instance. Only the values that
// depend on the wavelength differ between instances.
// Column pass: the transmission factors of the split step's element.
struct BatchTrans {
    double2 fa, fb;                         // grating / DBA / scalar factors
    const double2 *mat_db, *mat_factor;     // sample: per-material tables of the instance
    double sample_y;                        // sample: 2 pi dz / wl
};
// Row pass: the transfer function of the split step (chirp form).
struct BatchProp {
    double2 A;
    double g_hi, g_lo;
    const void *h3;
    int64_t cut_lo, cut_hi;                 // used where PropArgs::has_cut
};

// Detector binning fused into the last inverse column pass of a phase step
// (square_and_downsample, big-wave/propagation.py:279-320). Pixel j holds the
// samples [bounds[j], bounds[j+1]) (np.histogram bins, built on the host);
// the pass adds |u|^2 of its samples into sum[j] (FP64, zero between passes),
// and the CTA that finishes last adds weight * (((sum cos_j) dx) psy) / r_j
// into acc/comp (Kahan) and zeroes sum and count again.
struct DetectArgs {
    const int64_t *bounds;   // n_pix + 1
    const double *cosv, *rv; // per pixel
    int64_t n_pix;
    int64_t lo, hi;          // bounds[0], bounds[n_pix]: the detector's sample range
    double inv_w;            // n_pix / (hi - lo): first guess of a sample's pixel
    double dx, psy, weight;
    double *sum;             // n_pix raw sums
    unsigned *count;         // CTAs done
    double *acc, *comp;      // the phase step's accumulator row
    // batched passes: instance b bins into sum + b * sum_stride and adds with
    // weight bweight[b]; the instances are added in order (n_inst of them)
    const double *bweight;
    int64_t sum_stride;
    int n_inst;
    // optional: the pixel values of each instance (unweighted) also written
    // to inst_out + b * inst_stride
    double *inst_out;
    int64_t inst_stride;
};

// Arguments of one pass. N = N1 * N2 samples; three-level plans split the
// row level further, N2 = Nb * Nr, with a middle pass of the column kernel.
//   row kernel:    rows of 2^log_n2 samples; row index = p1 * Nb + pb, spectrum
//                  index k = k1 + N1 * (kb + Nb * k2) with k1 = digitrev(p1),
//                  kb = digitrev(pb); log_nb = 0 for two-level plans
//   column kernel: columns of 2^log_n1 samples at stride 2^log_n2, in
//                  n >> (log_n1 + log_n2) consecutive batches
struct PassArgs {
    const void *in;
    void *out;
    int64_t n;
    int log_n1;
    int log_n2;
    int log_nb;     // row kernel: middle level (0: none)
    int rb_n1, rb_nb;  // row kernel: digit widths of the column and middle levels (digitrev of the row)
    int flags;
    const void *tw_row;   // block twiddles of the row level
    const void *tw_col;   // block twiddles of the column level
    const void *tw4_lo;   // four-step twiddles (FP64): W_M^m = lo[m & mask] * hi[m >> shift], M = 2^tw_log
    const void *tw4_hi;
    int tw4_shift;
    int tw_log;
    double tw_scale;      // factor of the conjugate twiddles (1/N at the last inverse level)
    TransArgs tr;
    PropArgs pr;
    DetectArgs det;
    // batched passes (NULL: one set of values for every transform):
    // column pass, per instance of the batch; row pass, likewise
    const BatchTrans *btr;
    const BatchProp *bpr;
    // column pass: when set, the launch functions store the kernel's resident
    // CTAs on the current device here and launch nothing
    int64_t *resident;
    // column pass, filled in by its launch function: a 2-D TMA map over the
    // input (rows of 2^log_n2 samples as 8-byte words; boxes of one tile's
    // columns by up to 256 rows), through which each CTA prefetches its next
    // tile into L2; in_map_ok 0: no prefetch
    int in_map_ok;
    CUtensorMap in_map;
};

// Level structure of the internal spectrum layout (log2 lengths and digit
// widths of the column, middle and row levels).
struct SpecLevels {
    int log_n1, log_nb, log_nr;
    int rb_n1, rb_nb, rb_nr;
};

// Phase-step signal retrieval: the 3 x K pseudo-inverse of [sin phi_k,
// cos phi_k, 1] (rows a, b, c at stride RSW_RETRIEVAL_MAX) and the design
// matrix columns for the residuals.
constexpr int RSW_RETRIEVAL_MAX = 64;
struct RetrievalArgs {
    int k;
    double p[3 * RSW_RETRIEVAL_MAX];
    double sn[RSW_RETRIEVAL_MAX], cs[RSW_RETRIEVAL_MAX];
};

}  // namespace rsw
