// cnn_gemm.cu — training convolutions of the closure network as tcgen05 GEMMs (cnn_gemm.cuh):
// im2col expansions, operand packing, the GEMM kernel and its epilogues, the split-K reduction.
#include "cnn_gemm.cuh"
#include "cnn_tc.cuh"

#include <algorithm>

namespace dns2d {
namespace cnngemm {
namespace {

using cnntc::bulk_g2s;
using cnntc::idesc_bf16;
using cnntc::mbar_arrive;
using cnntc::mbar_expect_tx;
using cnntc::mbar_init;
using cnntc::mbar_wait;
using cnntc::mma_bf16;
using cnntc::mma_commit;
using cnntc::saddr;
using cnntc::smem_desc;

// the same GELU and derivative as the FP32 path (erf form)
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint4 pack8(const float (&v)[8])
{
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    return u;
}

// ROWS-mode A: row m = pixel (b, y, x) of B images, k = tap * C + c (tap = 3 ky + kx), value
// x[b][c][(y + ky - 1) % H][(x + kx - 1) % W]; rows >= M and k >= 9 C are zero.  One thread per
// row (pixel), walking k with running (tap, c) counters and the tap's source offset recomputed
// only when the tap changes; a warp's 32 consecutive pixels load 128 contiguous bytes per (tap,
// c) and store 512 contiguous bytes per 8 k.
__global__ void k_im2col_rows(const float *__restrict__ x, int C, int H, int W, int M, int MT, int KS,
                              __nv_bfloat16 *__restrict__ A)
{
    const int HW = H * W;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < MT * BM; m += gridDim.x * blockDim.x) {
        const bool valid = m < M;
        const int b = valid ? m / HW : 0, p = m - b * HW, y = p / W, xx = p - y * W;
        const float *xb = x + (size_t)b * C * HW;
        __nv_bfloat16 *Am = A + (size_t)(m / BM) * KS * A_BLOCK;
        const int r = m % BM;
        if ((C & 7) == 0) {
            // C a multiple of 8: each 8-k chunk is 8 channels of one tap, one source offset per tap
            int k8 = 0;
            for (int tap = 0; tap < 9; ++tap) {
                const int sy = (y + tap / 3 - 1 + H) % H, sx = (xx + tap % 3 - 1 + W) % W;
                const float *src = xb + (size_t)sy * W + sx;
                for (int c0 = 0; c0 < C; c0 += 8, ++k8) {
                    float v[8];
#pragma unroll
                    for (int i = 0; i < 8; ++i) v[i] = valid ? __ldg(src + (size_t)(c0 + i) * HW) : 0.0f;
                    *reinterpret_cast<uint4 *>(Am + (size_t)(k8 >> 1) * A_BLOCK + a_elem(r, (k8 & 1) * 8)) = pack8(v);
                }
            }
            const uint4 z = make_uint4(0u, 0u, 0u, 0u);
            for (; k8 < KS * 2; ++k8)
                *reinterpret_cast<uint4 *>(Am + (size_t)(k8 >> 1) * A_BLOCK + a_elem(r, (k8 & 1) * 8)) = z;
            continue;
        }
        int tap = 0, c = 0, off = 0;
        bool newtap = true;
        for (int k8 = 0; k8 < KS * 2; ++k8) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float val = 0.0f;
                if (tap < 9) {
                    if (newtap) {
                        const int sy = (y + tap / 3 - 1 + H) % H, sx = (xx + tap % 3 - 1 + W) % W;
                        off = sy * W + sx;
                        newtap = false;
                    }
                    if (valid) val = __ldg(xb + (size_t)c * HW + off);
                    if (++c == C) {
                        c = 0;
                        ++tap;
                        newtap = true;
                    }
                }
                v[i] = val;
            }
            *reinterpret_cast<uint4 *>(Am + (size_t)(k8 >> 1) * A_BLOCK + a_elem(r, (k8 & 1) * 8)) = pack8(v);
        }
    }
}

// SPLITK-mode A: row m = tap * C + c, k = pixel (b, y, x) of B images (the count a multiple of
// 16), value x[b][c][(y + ky - 1) % H][(x + kx - 1) % W]; row 9 C is all ones (its product row
// is the bias gradient sum_p dz), the rows after it zero (9 C is never a multiple of 128 for
// C <= 32, so row 9 C always exists).  One thread per (8 consecutive pixels, tap), pixels
// fastest: the 8 source offsets are computed once, then every channel is 8 loads (a warp reads
// 32 contiguous groups) and one 16-byte store; "tap" 9 writes the ones row and the zero rows.
// Blocks [K step][M tile].
__global__ void k_im2col_cols(const float *__restrict__ x, int C, int H, int W, int K, int MT,
                              __nv_bfloat16 *__restrict__ A)
{
    const int HW = H * W, K8 = K / 8, R = MT * BM;
    const long long total = (long long)K8 * 10;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const int tap = (int)(e / K8), k8 = (int)(e - (long long)tap * K8);
        __nv_bfloat16 *Ak = A + (size_t)(k8 >> 1) * MT * A_BLOCK;
        const int kk = (k8 & 1) * 8;
        if (tap == 9) {
            float one[8], zero[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                one[i] = 1.0f;
                zero[i] = 0.0f;
            }
            for (int m = 9 * C; m < R; ++m)
                *reinterpret_cast<uint4 *>(Ak + (size_t)(m / BM) * A_BLOCK + a_elem(m % BM, kk)) =
                    pack8(m == 9 * C ? one : zero);
            continue;
        }
        const int dx = tap % 3;
        {
            // W a multiple of 8: the 8 pixels are one row segment x0 .. x0 + 7 (x0 a multiple of
            // 8); away from the periodic wrap their taps are one aligned 12-float window read as
            // float4s: dx = 0 needs x0 - 1 .. x0 + 6, dx = 1 x0 .. x0 + 7, dx = 2 x0 + 1 .. x0 + 8
            const int k0 = k8 * 8, b = k0 / HW, p = k0 - b * HW, y = p / W, x0 = p - y * W;
            if ((W & 7) == 0 && !(dx == 0 && x0 == 0) && !(dx == 2 && x0 + 8 == W)) {
                const int sy = (y + tap / 3 - 1 + H) % H;
                const float *row = x + (size_t)b * C * HW + (size_t)sy * W;
                for (int c = 0; c < C; ++c) {
                    const float *rp = row + (size_t)c * HW;
                    float v[8];
                    if (dx == 1) {
                        const float4 a = __ldg(reinterpret_cast<const float4 *>(rp + x0));
                        const float4 d = __ldg(reinterpret_cast<const float4 *>(rp + x0 + 4));
                        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
                        v[4] = d.x; v[5] = d.y; v[6] = d.z; v[7] = d.w;
                    } else {
                        const int w0 = dx == 0 ? x0 - 4 : x0;
                        const float4 a = __ldg(reinterpret_cast<const float4 *>(rp + w0));
                        const float4 d = __ldg(reinterpret_cast<const float4 *>(rp + w0 + 4));
                        const float4 f = __ldg(reinterpret_cast<const float4 *>(rp + w0 + 8));
                        if (dx == 0) {
                            v[0] = a.w; v[1] = d.x; v[2] = d.y; v[3] = d.z;
                            v[4] = d.w; v[5] = f.x; v[6] = f.y; v[7] = f.z;
                        } else {
                            v[0] = a.y; v[1] = a.z; v[2] = a.w; v[3] = d.x;
                            v[4] = d.y; v[5] = d.z; v[6] = d.w; v[7] = f.x;
                        }
                    }
                    const int m = tap * C + c;
                    *reinterpret_cast<uint4 *>(Ak + (size_t)(m / BM) * A_BLOCK + a_elem(m % BM, kk)) = pack8(v);
                }
                continue;
            }
        }
        size_t src[8];
        {
            const int k0 = k8 * 8;
            int b = k0 / HW, p = k0 - b * HW, y = p / W, xx = p - y * W;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int sy = (y + tap / 3 - 1 + H) % H, sx = (xx + tap % 3 - 1 + W) % W;
                src[i] = (size_t)b * C * HW + (size_t)sy * W + sx;
                if (++xx == W) {
                    xx = 0;
                    if (++y == H) {
                        y = 0;
                        ++b;
                    }
                }
            }
        }
        for (int c = 0; c < C; ++c) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = __ldg(x + src[i] + (size_t)c * HW);
            const int m = tap * C + c;
            *reinterpret_cast<uint4 *>(Ak + (size_t)(m / BM) * A_BLOCK + a_elem(m % BM, kk)) = pack8(v);
        }
    }
}

// ROWS-mode B from the weights w[co][ci][tap]: forward (flip 0) B[k = tap * Ci + ci][n = co];
// data gradient (flip 1) B[k = tap * Co + co][n = ci] = w[co][ci][8 - tap]; columns >= the
// output channels and k beyond 9 x the input channels are zero.  KS blocks.
__global__ void k_pack_weights_gemm(const float *__restrict__ w, int Ci, int Co, int flip, int KS,
                                    __nv_bfloat16 *__restrict__ Bm)
{
    const int Kin = flip ? Co : Ci, Nout = flip ? Ci : Co;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < KS * BK * BN; e += gridDim.x * blockDim.x) {
        const int k = e / BN, n = e - k * BN, tap = k / Kin, c = k - tap * Kin;
        float val = 0.0f;
        if (n < Nout && tap < 9)
            val = flip ? w[((size_t)c * Ci + n) * 9 + (8 - tap)] : w[((size_t)n * Ci + c) * 9 + tap];
        Bm[(size_t)(k / BK) * B_BLOCK + b_elem(n, k % BK)] = __float2bfloat16_rn(val);
    }
}

// SPLITK-mode B from dz[b][co][pixel]: B[k = pixel][n = co] (columns >= Co zero), one block per
// K step; one thread per (column, 8 consecutive pixels)
__global__ void k_pack_dz(const float *__restrict__ dz, int Co, int HW, int K, __nv_bfloat16 *__restrict__ Bm)
{
    const int K8 = K / 8;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < BN * K8; e += gridDim.x * blockDim.x) {
        const int k8 = e / BN, n = e - k8 * BN;
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int k = k8 * 8 + i, b = k / HW, p = k - b * HW;
            v[i] = n < Co ? dz[((size_t)b * Co + n) * HW + p] : 0.0f;
        }
        *reinterpret_cast<uint4 *>(Bm + (size_t)(k8 >> 1) * B_BLOCK + b_elem(n, (k8 & 1) * 8)) = pack8(v);
    }
}

// dw[co][ci][tap] = sum over the G partials (fixed order, FP64) of part[g][tap * Ci + ci][co], and
// db[co] from row 9 Ci (the ones row)
__global__ void k_reduce_wgrad(const float *__restrict__ part, int G, int MT, int Ci, int Co, float *__restrict__ dw,
                               float *__restrict__ db)
{
    const int R = MT * BM, nw = Co * Ci * 9;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nw + Co; e += gridDim.x * blockDim.x) {
        int m, co;
        if (e < nw) {
            co = e / (Ci * 9);
            const int r = e - co * Ci * 9, ci = r / 9, tap = r - ci * 9;
            m = tap * Ci + ci;
        } else {
            co = e - nw;
            m = 9 * Ci;
        }
        double s = 0.0;
        for (int g = 0; g < G; ++g) s += (double)part[((size_t)g * R + m) * BN + co];
        if (e < nw)
            dw[e] = (float)s;
        else
            db[co] = (float)s;
    }
}

struct GemmArgs {
    const __nv_bfloat16 *A = nullptr, *Bm = nullptr;
    int epi = EPI_FWD;
    int MT = 0;   // ROWS: pixel tiles; SPLITK: row tiles (<= MAX_MT)
    int KS = 0;   // ROWS: K steps per tile; SPLITK: K steps in all
    int M = 0, Nv = 0, HW = 1;
    const float *bias = nullptr;
    float *z = nullptr, *a = nullptr;  // forward outputs [B][Nv][HW]
    const float *zprev = nullptr;      // data gradient: GELU'(zprev) factor, [B][Nv][HW]
    float *dx = nullptr;               // data gradient output [B][Nv][HW]
    float *part = nullptr;             // SPLITK: [gridDim.x][MT * 128][32]
    int *err = nullptr;
};

constexpr int kGemmThreads = 192;  // SPLITK: warps 0-3 epilogue (TMEM lanes), 4 producer, 5 MMA issuer
constexpr int kRowThreads = 320;   // ROWS: warps 0-7 epilogue (16 columns each), 8 producer, 9 MMA issuer
constexpr int kRowStages = 2, kSplitStages = 3;

__device__ __forceinline__ unsigned char *aligned_base(unsigned char *sm)
{
    return sm + ((1024u - (saddr(sm) & 1023u)) & 1023u);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *holder, int cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(holder)), "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// ROWS mode: CTA c takes pixel tiles c, c + G, ...; per tile one bulk copy of its KS A blocks
// into one of two stages, KS MMAs (128 x 32 x 16) into one of two TMEM accumulators, and the
// forward or data-gradient epilogue (8 warps, 16 channels each).  B (all KS blocks) is loaded once.  Every wait is bounded
// (2 s): one that runs out sets *err and the roles stop after their copies and MMAs in flight.
__global__ void __launch_bounds__(kRowThreads, 1) k_gemm_rows(const __grid_constant__ GemmArgs q)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t full[kRowStages], empty[kRowStages], tfull[2], tempty[2], wbar;
    __shared__ int info[kRowStages], tinfo[2];
    __shared__ uint32_t tmem_holder;
    __shared__ float sbias[BN];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KS = q.KS;
    unsigned char *sB = aligned_base(sm);
    unsigned char *sA = sB + ((KS * 1024 + 1023) / 1024) * 1024;
    const int stageB = KS * A_BLOCK * 2;  // bytes of one stage
    if (tid < BN) sbias[tid] = (q.epi == EPI_FWD && tid < q.Nv) ? q.bias[tid] : 0.0f;
    if (warp == 0) tmem_alloc(&tmem_holder, 64);
    if (tid == 0) {
        for (int s = 0; s < kRowStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 2);
            mbar_init(&tempty[b], 8);
        }
        mbar_init(&wbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_holder;

    if (warp == 8) {
        if (lane == 0) {
            mbar_expect_tx(&wbar, (uint32_t)(KS * B_BLOCK * 2));
            bulk_g2s(sB, q.Bm, (uint32_t)(KS * B_BLOCK * 2), &wbar);
            int k = 0;
            for (;; ++k) {
                const int s = k % kRowStages;
                int item = (int)blockIdx.x + k * (int)gridDim.x;
                if (item >= q.MT) item = -1;
                bool free = true;
                if (k >= kRowStages && !mbar_wait(&empty[s], (uint32_t)((k / kRowStages - 1) & 1))) {
                    atomicExch(q.err, 1);
                    item = -1;
                    free = false;
                }
                info[s] = item;
                if (item < 0) {
                    if (free) mbar_arrive(&full[s]);
                    break;
                }
                mbar_expect_tx(&full[s], (uint32_t)stageB);
                bulk_g2s(sA + (size_t)s * stageB, q.A + (size_t)item * KS * A_BLOCK, (uint32_t)stageB, &full[s]);
            }
            for (int kk = (k - kRowStages + 1 > 0 ? k - kRowStages + 1 : 0); kk < k; ++kk)
                mbar_wait(&full[kk % kRowStages], (uint32_t)((kk / kRowStages) & 1));
            mbar_wait(&wbar, 0);
        }
        __syncwarp();
    } else if (warp == 9) {
        if (lane == 0) {
            bool ok = mbar_wait(&wbar, 0);
            if (!ok) atomicExch(q.err, 1);
            const uint64_t db0 = smem_desc(saddr(sB), 512, 128);
            constexpr uint32_t idesc = idesc_bf16(BN);
            int k = 0, last_k = -1;
            for (;; ++k) {
                const int s = k % kRowStages, bb = k & 1;
                int item = -1;
                if (ok) {
                    if (mbar_wait(&full[s], (uint32_t)((k / kRowStages) & 1))) {
                        item = info[s];
                    } else {
                        atomicExch(q.err, 1);
                        ok = false;
                    }
                }
                if (k >= 2 && !mbar_wait(&tempty[bb], (uint32_t)((k / 2 - 1) & 1))) {
                    atomicExch(q.err, 1);
                    break;
                }
                tinfo[bb] = item;
                if (item < 0) {
                    mbar_arrive(&tfull[bb], 2);  // end marker
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint64_t da0 = smem_desc(saddr(sA) + (uint32_t)(s * stageB), 2048, 128);
                for (int ks = 0; ks < KS; ++ks)
                    mma_bf16(tmem + (uint32_t)(bb * BN), da0 + (uint64_t)((ks * A_BLOCK * 2) >> 4),
                             db0 + (uint64_t)((ks * B_BLOCK * 2) >> 4), idesc, ks > 0 ? 1u : 0u);
                mma_commit(&empty[s]);
                mma_commit(&tfull[bb]);
                mbar_arrive(&tfull[bb]);
                last_k = k;
            }
            if (last_k >= 0) mbar_wait(&empty[last_k % kRowStages], (uint32_t)((last_k / kRowStages) & 1));
        }
        __syncwarp();
    } else {
        // warp w: TMEM lanes 32 (w % 4) .. (pixels), columns 16 (w / 4) .. + 15 (channels)
        const int qd = warp & 3, c0 = 16 * (warp >> 2);
        for (int k = 0;; ++k) {
            const int bb = k & 1;
            const bool got = mbar_wait(&tfull[bb], (uint32_t)((k / 2) & 1));
            if (!__all_sync(0xffffffffu, got)) {
                if (lane == 0) atomicExch(q.err, 1);
                break;
            }
            const int item = tinfo[bb];
            if (item < 0) break;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            uint32_t r[16];
            tmem_ld16(tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(bb * BN + c0), r);
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[bb]);
            const int m = item * BM + qd * 32 + lane;
            if (m < q.M && c0 < q.Nv) {
                const int b = m / q.HW, p = m - b * q.HW;
                const size_t o0 = (size_t)b * q.Nv * q.HW + p + (size_t)c0 * q.HW;
                if (q.epi == EPI_FWD) {
                    float zv[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) zv[j] = __uint_as_float(r[j]) + sbias[c0 + j];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (c0 + j < q.Nv) q.z[o0 + (size_t)j * q.HW] = zv[j];
                    if (q.a) {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (c0 + j < q.Nv) q.a[o0 + (size_t)j * q.HW] = gelu(zv[j]);
                    }
                } else {
                    float zp[16];  // every load before any store (dx and zprev are different tensors)
#pragma unroll
                    for (int j = 0; j < 16; ++j) zp[j] = c0 + j < q.Nv ? __ldg(q.zprev + o0 + (size_t)j * q.HW) : 0.0f;
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (c0 + j < q.Nv) q.dx[o0 + (size_t)j * q.HW] = __uint_as_float(r[j]) * gelu_grad(zp[j]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(64));
}

// SPLITK mode: CTA c takes chunks c, c + G, ... of KC K steps; per chunk one bulk copy of its
// KC x MT A blocks and one of its KC B blocks into one of three stages, and KC x MT MMAs that
// accumulate into MT TMEM accumulators (32 columns each) over all of the CTA's chunks; at the end
// the epilogue writes the CTA's partial D[MT * 128][32] to part[c] (zeros for a CTA without a
// chunk).  Bounded waits as in ROWS mode.
__global__ void __launch_bounds__(kGemmThreads, 1) k_gemm_splitk(const __grid_constant__ GemmArgs q)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t full[kSplitStages], empty[kSplitStages], tfull;
    __shared__ int info[kSplitStages], done_chunks;
    __shared__ uint32_t tmem_holder;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int MT = q.MT, KS = q.KS, nchunks = (KS + KC - 1) / KC;
    const int aBytes = KC * MT * A_BLOCK * 2, stageBytes = aBytes + KC * B_BLOCK * 2;
    unsigned char *sS = aligned_base(sm);
    if (warp == 0) tmem_alloc(&tmem_holder, 128);
    if (tid == 0) {
        for (int s = 0; s < kSplitStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&tfull, 2);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_holder;

    if (warp == 4) {
        if (lane == 0) {
            int k = 0;
            for (;; ++k) {
                const int s = k % kSplitStages;
                int item = (int)blockIdx.x + k * (int)gridDim.x;
                if (item >= nchunks) item = -1;
                bool free = true;
                if (k >= kSplitStages && !mbar_wait(&empty[s], (uint32_t)((k / kSplitStages - 1) & 1))) {
                    atomicExch(q.err, 1);
                    item = -1;
                    free = false;
                }
                info[s] = item;
                if (item < 0) {
                    if (free) mbar_arrive(&full[s]);
                    break;
                }
                const int kc = KS - item * KC < KC ? KS - item * KC : KC;
                unsigned char *st = sS + (size_t)s * stageBytes;
                mbar_expect_tx(&full[s], (uint32_t)(kc * (MT * A_BLOCK + B_BLOCK) * 2));
                bulk_g2s(st, q.A + (size_t)item * KC * MT * A_BLOCK, (uint32_t)(kc * MT * A_BLOCK * 2), &full[s]);
                bulk_g2s(st + aBytes, q.Bm + (size_t)item * KC * B_BLOCK, (uint32_t)(kc * B_BLOCK * 2), &full[s]);
            }
            for (int kk = (k - kSplitStages + 1 > 0 ? k - kSplitStages + 1 : 0); kk < k; ++kk)
                mbar_wait(&full[kk % kSplitStages], (uint32_t)((kk / kSplitStages) & 1));
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(BN);
            int k = 0, done = 0, last_k = -1;
            for (;; ++k) {
                const int s = k % kSplitStages;
                if (!mbar_wait(&full[s], (uint32_t)((k / kSplitStages) & 1))) {
                    atomicExch(q.err, 1);
                    break;
                }
                const int item = info[s];
                if (item < 0) break;
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const int kc = KS - item * KC < KC ? KS - item * KC : KC;
                const uint32_t st = saddr(sS) + (uint32_t)(s * stageBytes);
                const uint64_t da0 = smem_desc(st, 2048, 128), db0 = smem_desc(st + (uint32_t)aBytes, 512, 128);
                for (int ks = 0; ks < kc; ++ks)
                    for (int mt = 0; mt < MT; ++mt)
                        mma_bf16(tmem + (uint32_t)(mt * BN), da0 + (uint64_t)(((ks * MT + mt) * A_BLOCK * 2) >> 4),
                                 db0 + (uint64_t)((ks * B_BLOCK * 2) >> 4), idesc, (done > 0 || ks > 0) ? 1u : 0u);
                mma_commit(&empty[s]);
                ++done;
                last_k = k;
            }
            done_chunks = done;
            mma_commit(&tfull);  // the accumulators are complete once every MMA issued is done
            mbar_arrive(&tfull);
            if (last_k >= 0) mbar_wait(&empty[last_k % kSplitStages], (uint32_t)((last_k / kSplitStages) & 1));
        }
        __syncwarp();
    } else {
        const bool got = mbar_wait(&tfull, 0u);
        if (!__all_sync(0xffffffffu, got)) {
            if (lane == 0) atomicExch(q.err, 1);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const int done = done_chunks;
            for (int mt = 0; mt < MT; ++mt) {
                uint32_t r[32];
                if (done > 0) {
                    tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * BN), r);
                } else {
#pragma unroll
                    for (int n = 0; n < 32; ++n) r[n] = 0u;
                }
                float4 *dst = reinterpret_cast<float4 *>(
                    q.part + (((size_t)blockIdx.x * MT + mt) * BM + warp * 32 + lane) * BN);
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    dst[i] = make_float4(__uint_as_float(r[4 * i]), __uint_as_float(r[4 * i + 1]),
                                         __uint_as_float(r[4 * i + 2]), __uint_as_float(r[4 * i + 3]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(128));
}

}  // namespace
}  // namespace cnngemm
}  // namespace dns2d

namespace dns2d {
namespace cnngemm {
namespace {

cudaError_t grow(void **p, size_t *cap, size_t need, size_t elem)
{
    if (need <= *cap) return cudaSuccess;
    cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, need * elem);
    if (e == cudaSuccess) *cap = need;
    return e;
}

cudaError_t ensure(Work &wk, size_t a_el, size_t b_el, size_t part_f, cudaStream_t st)
{
    cudaError_t e;
    if (!wk.err) {
        if ((e = cudaMalloc((void **)&wk.err, 4)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(wk.err, 0, 4, st)) != cudaSuccess) return e;
    }
    if (a_el > wk.A_cap || b_el > wk.B_cap || part_f > wk.part_cap)
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;  // the old buffers may be in use
    if ((e = grow((void **)&wk.A, &wk.A_cap, a_el, 2)) != cudaSuccess) return e;
    if ((e = grow((void **)&wk.Bm, &wk.B_cap, b_el, 2)) != cudaSuccess) return e;
    return grow((void **)&wk.part, &wk.part_cap, part_f, 4);
}

int sm_count()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1) sms = 1;
    }
    return sms;
}

int blocks_for(long long items) { return (int)std::max<long long>(1, std::min<long long>(4096, (items + 255) / 256)); }

// ROWS-mode GEMM on the expanded A (already in wk.A) and packed B (in wk.Bm)
cudaError_t run_rows(GemmArgs g, Work &wk, cudaStream_t st)
{
    g.A = wk.A;
    g.Bm = wk.Bm;
    g.err = wk.err;
    const size_t smem = 1024 + (size_t)(g.KS * B_BLOCK * 2 + 1023) / 1024 * 1024 + (size_t)kRowStages * g.KS * A_BLOCK * 2;
    cudaError_t e = cudaFuncSetAttribute(k_gemm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_gemm_rows<<<std::min(g.MT, sm_count()), kRowThreads, smem, st>>>(g);
    return cudaGetLastError();
}

}  // namespace

cudaError_t conv_fwd(const float *x, int Ci, const float *w, const float *bias, int Co, float *z, float *a, int B,
                     int H, int W, Work &wk, cudaStream_t st)
{
    if (Ci < 1 || Ci > BN || Co < 1 || Co > BN) return cudaErrorInvalidValue;
    const int M = B * H * W, MT = (M + BM - 1) / BM, KS = ksteps_of(Ci);
    if (KS > MAX_KS) return cudaErrorInvalidValue;  // the shared-memory stages are sized for it
    cudaError_t e = ensure(wk, (size_t)MT * KS * A_BLOCK, (size_t)KS * B_BLOCK, 0, st);
    if (e != cudaSuccess) return e;
    k_im2col_rows<<<blocks_for((long long)MT * BM), 256, 0, st>>>(x, Ci, H, W, M, MT, KS, wk.A);
    k_pack_weights_gemm<<<blocks_for((long long)KS * BK * BN), 256, 0, st>>>(w, Ci, Co, 0, KS, wk.Bm);
    GemmArgs g;
    g.epi = EPI_FWD;
    g.MT = MT;
    g.KS = KS;
    g.M = M;
    g.Nv = Co;
    g.HW = H * W;
    g.bias = bias;
    g.z = z;
    g.a = a;
    return run_rows(g, wk, st);
}

cudaError_t conv_dgrad(const float *dz, int Co, const float *w, int Ci, const float *zprev, float *dx, int B, int H,
                       int W, Work &wk, cudaStream_t st)
{
    if (Ci < 1 || Ci > BN || Co < 1 || Co > BN) return cudaErrorInvalidValue;
    const int M = B * H * W, MT = (M + BM - 1) / BM, KS = ksteps_of(Co);
    if (KS > MAX_KS) return cudaErrorInvalidValue;
    cudaError_t e = ensure(wk, (size_t)MT * KS * A_BLOCK, (size_t)KS * B_BLOCK, 0, st);
    if (e != cudaSuccess) return e;
    k_im2col_rows<<<blocks_for((long long)MT * BM), 256, 0, st>>>(dz, Co, H, W, M, MT, KS, wk.A);
    k_pack_weights_gemm<<<blocks_for((long long)KS * BK * BN), 256, 0, st>>>(w, Ci, Co, 1, KS, wk.Bm);
    GemmArgs g;
    g.epi = EPI_DGRAD;
    g.MT = MT;
    g.KS = KS;
    g.M = M;
    g.Nv = Ci;
    g.HW = H * W;
    g.zprev = zprev;
    g.dx = dx;
    return run_rows(g, wk, st);
}

cudaError_t conv_wgrad(const float *x, int Ci, const float *dz, int Co, float *dw, float *db, int B, int H, int W,
                       Work &wk, cudaStream_t st)
{
    const int K = B * H * W, HW = H * W;
    if (Ci < 1 || Ci > BN || Co < 1 || Co > BN || K % BK != 0) return cudaErrorInvalidValue;
    const int MT = 9 * Ci / BM + 1, KS = K / BK, nchunks = (KS + KC - 1) / KC;  // rows 0 .. 9 Ci
    if (MT > MAX_MT) return cudaErrorInvalidValue;  // the shared-memory stages are sized for it
    const int G = std::min(nchunks, sm_count());
    cudaError_t e = ensure(wk, (size_t)KS * MT * A_BLOCK, (size_t)KS * B_BLOCK, (size_t)G * MT * BM * BN, st);
    if (e != cudaSuccess) return e;
    k_im2col_cols<<<blocks_for((long long)(K / 8) * 10), 256, 0, st>>>(x, Ci, H, W, K, MT, wk.A);
    k_pack_dz<<<blocks_for((long long)BN * (K / 8)), 256, 0, st>>>(dz, Co, HW, K, wk.Bm);
    GemmArgs g;
    g.A = wk.A;
    g.Bm = wk.Bm;
    g.epi = EPI_PART;
    g.MT = MT;
    g.KS = KS;
    g.part = wk.part;
    g.err = wk.err;
    const size_t smem = 1024 + (size_t)kSplitStages * KC * (MT * A_BLOCK + B_BLOCK) * 2;
    if ((e = cudaFuncSetAttribute(k_gemm_splitk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    k_gemm_splitk<<<G, kGemmThreads, smem, st>>>(g);
    k_reduce_wgrad<<<blocks_for((long long)Co * Ci * 9 + Co), 256, 0, st>>>(wk.part, G, MT, Ci, Co, dw, db);
    return cudaGetLastError();
}

void work_free(Work &wk)
{
    cudaFree(wk.A);
    cudaFree(wk.Bm);
    cudaFree(wk.part);
    cudaFree(wk.err);
    wk = Work{};
}

}  // namespace cnngemm
}  // namespace dns2d
