// Radix-16 stage study (not part of the propagation path): one radix-16 DFT
// stage of complex64 data done three ways, each followed by a shared-memory
// exchange like the one between FFT stages, repeated `reps` times on data
// held on chip so that the arithmetic, not HBM, is timed:
//   kind 0: the engine's register network (rsw::net_dif / net_dit: FFMA2
//           additions, lifting rotations), one 16-point vector per thread;
//   kind 1: Y = F X on the tensor cores, F the 32 x 32 real form of the
//           16-point DFT (scaled by 1/4, unitary), X eight vectors as a
//           32 x 8 matrix, mma.sync m16n8k8 with TF32 operands;
//   kind 2: kind 1 with both operands split into TF32 high and low parts and
//           three products (hi*lo + lo*hi + hi*hi), FP32-level accuracy.
// With reps = 1 and no exchange the output is the DFT (kind 0: unscaled,
// bit-reversed within each vector; kinds 1 and 2: scaled by 1/4, natural
// order), for the error check.
#include <cuda_runtime.h>
#include <stdint.h>

#include "rsw_block_fft.cuh"

namespace {

constexpr int NT = 256;  // threads per CTA

// kind 0: thread v owns vector v; forward network then inverse network
// (the pair returns 16 x the input; the exact power-of-two scale 1/16 keeps
// the values bounded), an exchange through shared memory after each stage
__global__ void __launch_bounds__(NT) stage_network(const float2 *__restrict__ in, float2 *__restrict__ out,
                                                    int64_t nvec, int reps) {
    __shared__ float2 sm[16][NT + 1];
    const int64_t v = int64_t(blockIdx.x) * NT + threadIdx.x;  // nvec is a multiple of NT (host check)
    float2 x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = in[v * 16 + k];
    const int lane = threadIdx.x & 31, wbase = threadIdx.x & ~31;
    for (int r = 0; r < reps; ++r) {
        if ((r & 1) == 0) {
            rsw::net_dif<16, -1>(x);
        } else {
            rsw::net_dit<16, +1>(x);
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = rsw::cscale(x[k], 0.0625f);
        }
        if (r + 1 < reps) {  // exchange: every value moves to another lane of the warp
#pragma unroll
            for (int k = 0; k < 16; ++k) sm[k][threadIdx.x] = x[k];
            __syncwarp();
#pragma unroll
            for (int k = 0; k < 16; ++k) x[k] = sm[k][wbase + (lane ^ (k + 1))];
            __syncwarp();
        }
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) out[v * 16 + k] = x[k];
}

__device__ __forceinline__ uint32_t tf32(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return r;
}

__device__ __forceinline__ void mma_tf32(float *d, const uint32_t *a, const uint32_t *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// kinds 1 and 2: warp w of the CTA owns vectors 8 w' .. 8 w' + 7 of its batch
// (w' the global warp index). X[r][n] = Re x_r (r < 16) or Im x_{r-16} of
// vector n; fragments of m16n8k8 (g = lane / 4, t = lane % 4):
//   A (rows of F):  {F[g][t], F[g+8][t], F[g][t+4], F[g+8][t+4]} of each 16 x 8 tile
//   B (X):          {X[t][g], X[t+4][g]} of each 8 x 8 tile
//   D (Y):          {Y[g][2t], Y[g][2t+1], Y[g+8][2t], Y[g+8][2t+1]} of each 16 x 8 tile
template <bool SPLIT>
__global__ void __launch_bounds__(NT) stage_mma(const float *__restrict__ F, const float *__restrict__ in,
                                                float *__restrict__ out, int64_t nvec, int reps) {
    __shared__ float ys[NT / 32][32][9];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int64_t batch = int64_t(blockIdx.x) * (NT / 32) + w;  // 8 vectors; nvec / 8 batches (host check)
    uint32_t ahi[2][4][4], alo[2][4][4];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            const int r0 = rt * 16 + g, c0 = kc * 8 + t;
            const float f[4] = {F[r0 * 32 + c0], F[(r0 + 8) * 32 + c0], F[r0 * 32 + c0 + 4], F[(r0 + 8) * 32 + c0 + 4]};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ahi[rt][kc][i] = tf32(f[i]);
                alo[rt][kc][i] = tf32(f[i] - __uint_as_float(ahi[rt][kc][i]));
            }
        }
    // X of this warp's batch
    float xv[4][2];
    auto xidx = [&](int r) { return ((batch * 8 + g) * 16 + (r & 15)) * 2 + (r >> 4); };
#pragma unroll
    for (int kc = 0; kc < 4; ++kc) {
        xv[kc][0] = in[xidx(kc * 8 + t)];
        xv[kc][1] = in[xidx(kc * 8 + t + 4)];
    }
    float d[2][4];
    for (int r = 0; r < reps; ++r) {
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int i = 0; i < 4; ++i) d[rt][i] = 0.f;
#pragma unroll
        for (int kc = 0; kc < 4; ++kc) {
            uint32_t bh[2] = {tf32(xv[kc][0]), tf32(xv[kc][1])};
            if constexpr (SPLIT) {
                uint32_t bl[2] = {tf32(xv[kc][0] - __uint_as_float(bh[0])), tf32(xv[kc][1] - __uint_as_float(bh[1]))};
#pragma unroll
                for (int rt = 0; rt < 2; ++rt) {
                    mma_tf32(d[rt], alo[rt][kc], bh);
                    mma_tf32(d[rt], ahi[rt][kc], bl);
                }
            }
#pragma unroll
            for (int rt = 0; rt < 2; ++rt) mma_tf32(d[rt], ahi[rt][kc], bh);
        }
        if (r + 1 < reps) {  // exchange: the D layout back into the B layout through shared memory
#pragma unroll
            for (int rt = 0; rt < 2; ++rt) {
                ys[w][rt * 16 + g][2 * t] = d[rt][0];
                ys[w][rt * 16 + g][2 * t + 1] = d[rt][1];
                ys[w][rt * 16 + g + 8][2 * t] = d[rt][2];
                ys[w][rt * 16 + g + 8][2 * t + 1] = d[rt][3];
            }
            __syncwarp();
#pragma unroll
            for (int kc = 0; kc < 4; ++kc) {
                xv[kc][0] = ys[w][kc * 8 + t][g];
                xv[kc][1] = ys[w][kc * 8 + t + 4][g];
            }
            __syncwarp();
        }
    }
    // Y[j][n] -> out vector n, sample j (real part rows 0..15, imaginary 16..31)
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) {
        const int64_t v0 = batch * 8 + 2 * t, v1 = v0 + 1;
        out[(v0 * 16 + g) * 2 + rt] = d[rt][0];
        out[(v1 * 16 + g) * 2 + rt] = d[rt][1];
        out[(v0 * 16 + g + 8) * 2 + rt] = d[rt][2];
        out[(v1 * 16 + g + 8) * 2 + rt] = d[rt][3];
    }
}

}  // namespace

extern "C" {

// One timed launch of kind 0/1/2 over n complex64 samples (n a multiple of
// 4096) from in to out (device buffers; F the 32 x 32 row-major real DFT
// matrix for kinds 1 and 2); *ms receives the CUDA-event time of the launch.
// Returns a cudaError_t value (0 = success, 1 = bad arguments).
int rsw_study_radix16(int kind, const void *F, const void *in, void *out, int64_t n, int reps, float *ms) {
    if (n <= 0 || n % 4096 != 0 || reps < 1 || kind < 0 || kind > 2 || !in || !out || (kind > 0 && !F)) return 1;
    const int64_t nvec = n / 16;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    if (kind == 0) {
        stage_network<<<unsigned(nvec / NT), NT>>>((const float2 *)in, (float2 *)out, nvec, reps);
    } else {
        const unsigned grid = unsigned(nvec / 8 / (NT / 32));
        if (kind == 1) stage_mma<false><<<grid, NT>>>((const float *)F, (const float *)in, (float *)out, nvec, reps);
        else stage_mma<true><<<grid, NT>>>((const float *)F, (const float *)in, (float *)out, nvec, reps);
    }
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return int(err);
}

}  // extern "C"
