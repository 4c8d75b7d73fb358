// cnn_gemm.cuh — the closure network's training convolutions on the 5th-gen tensor cores.
//
// Every 3x3 periodic convolution of training is one skinny GEMM with N = 32 (padded) on tcgen05,
// BF16 operands and FP32 accumulators in tensor memory, fed by an explicit im2col expansion:
//   forward          D[pixel][co] = sum_k A[pixel][k] B[k][co],  A = im2col(x), k = tap * Ci + ci,
//                    B = w[co][ci][tap]; epilogue z = D + bias, a = GELU(z)            (ROWS mode)
//   data gradient    D[pixel][ci] = sum_k A[pixel][k] B[k][ci],  A = im2col(dz), k = tap * Co + co,
//                    B = w[co][ci][8 - tap]; epilogue dx = D * GELU'(z_prev)           (ROWS mode)
//   weight gradient  D[m][co] = sum_pixel A[m][pixel] B[pixel][co], A = im2col(x) transposed,
//                    m = tap * Ci + ci, B = dz, and a row of ones (m = 9 Ci) whose product is
//                    db; K split over the CTAs, each writes its partial D, and a fixed-order
//                    FP64 sum forms dw and db                                          (SPLITK mode)
// The activations and gradients stay FP32 [B][C][H][W] like the SIMT path (cnn.cuh), so loss,
// GELU and Adam are unchanged; only the convolutions round their operands to bf16.
//
// Operands in global memory are blocks in the MMA's canonical K-major no-swizzle layout:
//   A block = 128 rows x 16 k (4 KB): element (r, k) at (k / 8) * 1024 + (r / 8) * 64 + (r % 8) * 8
//             + k % 8 (two K core-matrix columns 2048 bytes apart, 8-row core matrices 128 apart);
//   B block = 32 columns x 16 k (1 KB): element (n, k) at (k / 8) * 256 + (n / 8) * 64 + (n % 8) * 8
//             + k % 8.
// ROWS mode stores A tile-major ([M tile][K step] blocks: one bulk copy per tile) and all of B
// once per CTA; SPLITK mode stores A step-major ([K step][M tile]) and B per K step, so a chunk of
// K steps is one contiguous run of each.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dns2d {
namespace cnngemm {

constexpr int BM = 128, BK = 16, BN = 32;
constexpr int A_BLOCK = BM * BK;  // bf16 elements of an A block (4 KB)
constexpr int B_BLOCK = BN * BK;  // bf16 elements of a B block (1 KB)
constexpr int KC = 4;             // SPLITK: K steps per chunk (one pipeline stage)
constexpr int MAX_KS = 18;        // ROWS: K steps per tile (9 taps x 32 channels = 288)
constexpr int MAX_MT = 3;         // SPLITK: M tiles (9 taps x 32 channels = 288 rows)

__host__ __device__ __forceinline__ int a_elem(int r, int k) { return (k >> 3) * 1024 + (r >> 3) * 64 + (r & 7) * 8 + (k & 7); }
__host__ __device__ __forceinline__ int b_elem(int n, int k) { return (k >> 3) * 256 + (n >> 3) * 64 + (n & 7) * 8 + (k & 7); }

// K steps of an im2col with C channels (9 C padded to a multiple of 16)
__host__ __device__ __forceinline__ int ksteps_of(int C) { return (9 * C + BK - 1) / BK; }

enum Epi { EPI_FWD = 0, EPI_DGRAD = 1, EPI_PART = 2 };

// work buffers of the training GEMMs (grown on demand by the host wrappers)
struct Work {
    __nv_bfloat16 *A = nullptr, *Bm = nullptr;
    size_t A_cap = 0, B_cap = 0;  // elements
    float *part = nullptr;
    size_t part_cap = 0;          // floats
    int *err = nullptr;           // 1: an mbarrier wait ran out
};

// z = conv(x) + bias and, when a is set, a = GELU(z); x [B][Ci][H][W], z / a [B][Co][H][W]
cudaError_t conv_fwd(const float *x, int Ci, const float *w, const float *bias, int Co, float *z, float *a, int B,
                     int H, int W, Work &wk, cudaStream_t st);
// dx = conv(dz, flipped w) * GELU'(zprev); dz [B][Co][H][W], zprev / dx [B][Ci][H][W]
cudaError_t conv_dgrad(const float *dz, int Co, const float *w, int Ci, const float *zprev, float *dx, int B, int H,
                       int W, Work &wk, cudaStream_t st);
// dw[co][ci][tap] = sum dz[b][co][p] x[b][ci][p + tap], db[co] = sum dz[b][co][p]
cudaError_t conv_wgrad(const float *x, int Ci, const float *dz, int Co, float *dw, float *db, int B, int H, int W,
                       Work &wk, cudaStream_t st);
void work_free(Work &wk);

}  // namespace cnngemm
}  // namespace dns2d
