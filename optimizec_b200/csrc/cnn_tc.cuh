// cnn_tc.cuh — BF16 tensor-core (tcgen05) inference path of the closure network.
//
// The hidden 3x3 convolutions (32 -> 32 channels, periodic) run as implicit GEMMs on the 5th-gen
// tensor cores: D[128 pixels][32 co] += A[128 pixels][16 ci] B[16 ci][32 co], 18 MMAs per tile
// (9 taps x 2 halves of the 32 input channels), FP32 accumulation in tensor memory.
//
// Activations are bf16 in chunk planes (plane c holds channels 8c..8c+7 of a pixel, 16 bytes)
// and in strips: each 128-pixel strip of the image is stored with its two neighbouring pixels
// and one periodic frame row above and below, row by row, each row as its 4 chunk planes of 130
// pixels (act_bytes, store_px).  The producing layer's epilogue writes every halo copy.  A CTA
// owns 128 consecutive pixels of TR = 2 image rows; its 4-row, 130-pixel halo is then one
// contiguous run, copied unchanged into shared memory as [row][plane][pixel].  In that layout the
// A operand of tap (dy, dx) is the same K-major "no swizzle" canonical tile (8-pixel core
// matrices 128 bytes apart, the two K chunks one plane, 2080 bytes, apart) started at another
// 16-byte address, so the 9 taps need no data movement.  The weights are staged as
// [tap][chunk][co][8 ci] bf16.  One thread issues the MMAs and commits them to an mbarrier; the
// warps then read their 32 TMEM lanes (pixels) x 32 columns (output channels), add the bias,
// apply GELU and store bf16.  The last layer (32 -> 1) is the same MMA with N = 16 (15 zero weight columns) writing channel 0
// in FP32 times the output scale.  The first layer (3 -> 32) builds its A operand as an im2col
// tile in shared memory (K = 3 channels x 9 taps = 27, padded to 32) straight from the three FP32
// input planes times their input scales: 2 MMAs per tile.
//
// Every wait on the mbarrier is bounded: past the limit the kernel sets an error flag, skips the
// accumulator read and still frees its tensor memory.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dns2d {
namespace cnntc {

constexpr int C = 32;        // hidden channels (input and output of the tensor-core layers)
constexpr int TM = 128;      // pixels per tile (MMA M)
constexpr int TR = 2;        // image rows per CTA (one tile each, sharing the halo)
constexpr int HW = TM + 2;   // halo width (a strip of 128 pixels and its two neighbours)
constexpr int PLANEB = HW * 16;                  // 2 080: one chunk plane of one halo row
constexpr int ROWB = 4 * PLANEB;                 // 8 320: one halo row, its 4 chunk planes
constexpr int A_BYTES = (TR + 2) * ROWB;         // 33 280: a tile's halo, [row][plane][pixel][16 bytes]
constexpr int NT = 128;                          // 4 warps = 128 TMEM lanes
// instruction descriptor: D f32, A/B bf16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

// per output width NO (32 hidden channels, or 16 for the 32 -> 1 layer: 1 channel + 15 zero
// weight columns, the smallest MMA N): weights [dx][chunk][2 - dy][NO][8] bf16, so that for one
// (dx, chunk) the kernel rows of consecutive dy (reversed) are consecutive MMA N rows
template <int NO>
struct TcShape {
    static constexpr int B_BYTES = 9 * 4 * NO * 16;
    static constexpr int SMEM_BYTES = A_BYTES + B_BYTES;
    static constexpr int TMEM_COLS = NO * TR <= 32 ? 32 : NO * TR;  // allocation: power of 2 >= 32
    static constexpr uint32_t IDESC = idesc_bf16(NO);
};
constexpr unsigned long long kWaitNs = 2000000000ull;  // an mbarrier wait gives up after 2 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// UMMA shared-memory descriptor, K-major, no swizzle (version 1 = sm_100 format)
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}


// GELU of the bf16 path: the tanh form of Hendrycks and Gimpel,
//   0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with the hardware tanh approximation; its deviation from z Phi(z) stays below the bf16
// rounding of the stored activations (tests compare against the exact erf form).
__device__ __forceinline__ float gelu_f(float z)
{
    const float u = 0.7978845608028654f * fmaf(0.044715f * z, z * z, z);
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
    return 0.5f * z * (1.0f + t);
}

// periodic index in [0, n) of i in [-n, 2n)
__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// Activations in strips: image b, strip xs (128 pixels), padded row py (0 .. H + 1), chunk plane
// c, strip pixel lp (0 .. 129) -> 16 bytes at ((((b S + xs) (H + 2) + py) 4 + c) 130 + lp), S =
// W / 128.  Strip pixel lp is image column 128 xs + lp - 1 and padded row py is image row py - 1,
// both periodic, so a tile's halo (rows py = y0 .. y0 + TR + 1 of one strip) is one contiguous
// run of A_BYTES.
__host__ __device__ __forceinline__ size_t act_bytes(int B, int H, int W)
{
    return (size_t)B * (W / TM) * (H + 2) * ROWB;
}

// the 4 chunks of image pixel (y, x) of image b, at its place in its strip and at every halo
// position (the neighbouring strips' edge pixels, the frame rows) that repeats it (H >= 2)
__device__ __forceinline__ void store_px(__nv_bfloat16 *act, int b, int H, int W, int y, int x, const uint4 (&v)[4])
{
    const int S = W / TM, xs = x / TM, lp = x - xs * TM + 1;
    const int py1 = y == 0 ? H + 1 : (y == H - 1 ? 0 : -1);
    // the left neighbour's pixel 129 repeats lp = 1; the right neighbour's pixel 0 repeats lp = 128
    const int xs1 = lp == 1 ? (xs + S - 1) % S : (lp == TM ? (xs + 1) % S : -1);
    const int lp1 = lp == 1 ? TM + 1 : 0;
    uint4 *img = reinterpret_cast<uint4 *>(act) + (size_t)b * S * (H + 2) * (ROWB / 16);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int py = i == 0 ? y + 1 : py1;
        if (py < 0) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int s = j == 0 ? xs : xs1;
            if (s < 0) continue;
            uint4 *d = img + ((size_t)s * (H + 2) + py) * (ROWB / 16) + (j == 0 ? lp : lp1);
#pragma unroll
            for (int c = 0; c < 4; ++c) d[c * HW] = v[c];
        }
    }
}

// weights of a 32 -> Co layer, w[co][ci][3][3] f32 -> wtc[tap][chunk][NO][8] bf16 (co >= Co zero)
template <int NO>
__global__ void k_pack_weights(const float *__restrict__ w, int Co, __nv_bfloat16 *__restrict__ wtc)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 9 * 4 * NO * 8; e += gridDim.x * blockDim.x) {
        const int dx = e / (4 * 3 * NO * 8), r = e % (4 * 3 * NO * 8);
        const int ch = r / (3 * NO * 8), r2 = r % (3 * NO * 8);
        const int j = r2 / (NO * 8), r3 = r2 % (NO * 8), co = r3 / 8, k = r3 % 8;
        const int ci = ch * 8 + k, dy = 2 - j;
        wtc[e] = __float2bfloat16_rn(co < Co ? w[((size_t)co * C + ci) * 9 + dy * 3 + dx] : 0.0f);
    }
}

// ------------------------------------------------------------------------------------------
// tcgen05 / mbarrier steps shared by the kernels (one CTA of 128 threads)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr(dst)), "l"(src) : "memory");
}

// warp 0 allocates the tensor memory, thread 0 initialises the mbarrier; then every thread makes
// its own shared-memory writes visible to the tensor-core proxy and the CTA synchronises
template <int COLS>
__device__ __forceinline__ uint32_t tc_setup(uint32_t *holder, uint64_t *mbar)
{
    const int tid = threadIdx.x;
    if ((tid >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(holder)),
                     "r"(COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(mbar)), "r"(1));
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    return *holder;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(mbar))
                 : "memory");
}

// wait (at most kWaitNs) for the phase of the given parity to complete; false when it ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity)
{
    uint32_t done = 0;
    const unsigned long long t0 = global_ns();
    for (;;) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(saddr(mbar)), "r"(parity)
            : "memory");
        if (done || global_ns() - t0 > kWaitNs) break;
    }
    return done != 0;
}

__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *m, uint32_t count = 1)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(saddr(m)), "r"(count)
                 : "memory");
}

// one arrival that also announces the bytes the stage's bulk copies will deliver
__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(saddr(m)),
                 "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16) completing on m
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *m)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"(bytes), "r"(saddr(m))
                 : "memory");
}

// orders this thread's generic-proxy view of global memory with its async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

// bounded wait for phase 0 of the mbarrier; false when the limit ran out
__device__ __forceinline__ bool mma_wait(uint64_t *mbar)
{
    const bool done = mbar_wait(mbar, 0u);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    return done;
}

template <int COLS>
__device__ __forceinline__ void tc_teardown(uint32_t tmem_d)
{
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem_d), "r"(COLS));
}

// The MMAs of one tile (TR = 2 output rows, accumulators NO columns apart from d0): halo row h
// feeds output row h - dy for every dy with 0 <= h - dy < TR, and those rows share the A
// operand, so one MMA per (h, dx, K half) covers them all with N = NO x (number of such dy): the
// weight rows of consecutive dy (reversed) are consecutive in the packed layout, and so are the
// accumulators of the output rows.  Halo rows 0 and TR + 1 (one output row each) go first and
// start their accumulator; rows 1 .. TR then accumulate: 6 (TR + 2) = 24 MMAs instead of 36.
// A from [row][plane][pixel] at a0 (planes PLANEB, rows ROWB bytes apart), B from the layer's
// packed weights at b0; descriptors built once (their 14-bit start-address field cannot carry:
// shared memory < 256 KB).
template <int NO>
__device__ __forceinline__ void issue_conv_tile(uint32_t d0, uint32_t a0, uint32_t b0)
{
    static_assert(TR == 2, "halo-row order written for two output rows");
    const uint64_t da = smem_desc(a0, PLANEB, 128), db = smem_desc(b0, 3 * NO * 16, 128);
    constexpr int order[TR + 2] = {0, TR + 1, 1, 2};
#pragma unroll
    for (int i = 0; i < TR + 2; ++i) {
        const int h = order[i];
        const int dy_lo = h - (TR - 1) > 0 ? h - (TR - 1) : 0, dy_hi = h < 2 ? h : 2;  // valid dy range
        const int nj = dy_hi - dy_lo + 1, j0 = 2 - dy_hi, r0 = h - dy_hi;             // first output row
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
#pragma unroll
            for (int kh = 0; kh < 2; ++kh)
                mma_bf16(d0 + (uint32_t)(NO * r0), da + (uint64_t)((h * ROWB + 2 * kh * PLANEB + dx * 16) >> 4),
                         db + (uint64_t)((((dx * 4 + 2 * kh) * 3 + j0) * NO * 16) >> 4), idesc_bf16(NO * nj),
                         (i >= 2 || dx > 0 || kh > 0) ? 1u : 0u);
    }
}

// 32 accumulator columns (already loaded) -> bias, GELU, bf16: the pixel's 4 chunks
__device__ __forceinline__ void gelu_chunks(const uint32_t (&r)[32], const float *bias, uint4 (&v)[4])
{
    __align__(16) __nv_bfloat162 o[C / 2];
#pragma unroll
    for (int co = 0; co < C; co += 2)
        o[co / 2] = __floats2bfloat162_rn(gelu_f(__uint_as_float(r[co]) + bias[co]),
                                          gelu_f(__uint_as_float(r[co + 1]) + bias[co + 1]));
    const uint4 *src = reinterpret_cast<const uint4 *>(o);
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = src[q];
}

// 32 consecutive accumulator columns of this warp's 32 lanes
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

// this warp's 32 lanes x 32 columns -> bias, GELU, bf16 pixel (y, x) of image b in the padded layout
__device__ __forceinline__ void epilogue32(uint32_t taddr, const float *__restrict__ bias, __nv_bfloat16 *act, int b,
                                           int H, int W, int y, int x)
{
    uint32_t r[32];
    tmem_ld32(taddr, r);
    uint4 v[4];
    gelu_chunks(r, bias, v);
    store_px(act, b, H, W, y, x, v);
}

// ------------------------------------------------------------------------------------------
// 32 -> NO layer.  Grid (W/128 * H/TR, B), 128 threads; W % 128 == 0, H % TR == 0.
// Input x and output y in the padded chunk-planar layout.  NO = 32: GELU, bf16 output y.  NO = 16:
// channel 0 times out_scale, f32 output yf ([B][H][W], no activation).
// ------------------------------------------------------------------------------------------
template <int NO>
__global__ void __launch_bounds__(NT) k_conv_tc(const __nv_bfloat16 *__restrict__ x,
                                                const __nv_bfloat16 *__restrict__ wtc,
                                                const float *__restrict__ bias, __nv_bfloat16 *__restrict__ y,
                                                float *__restrict__ yf, float out_scale, int H, int W,
                                                int *__restrict__ err)
{
    using S = TcShape<NO>;
    constexpr int B_BYTES = S::B_BYTES, TMEM_COLS = S::TMEM_COLS;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    unsigned char *sA = sm;
    unsigned char *sB = sm + A_BYTES;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = W / TM;
    const int y0 = (blockIdx.x / tiles_x) * TR;
    const int x0 = (blockIdx.x % tiles_x) * TM;
    const size_t img = (size_t)blockIdx.y * H * W;

    // halo: padded rows y0 .. y0 + TR + 1 of the strip, one contiguous run
    const uint4 *xin = reinterpret_cast<const uint4 *>(x) +
                       (((size_t)blockIdx.y * tiles_x + blockIdx.x % tiles_x) * (H + 2) + y0) * (ROWB / 16);
    for (int e = tid; e < A_BYTES / 16; e += NT) cp16(sA + e * 16, xin + e);
    for (int e = tid; e < B_BYTES / 16; e += NT) cp16(sB + e * 16, wtc + (size_t)e * 8);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const uint32_t tmem_d = tc_setup<TMEM_COLS>(&tmem_base, &mbar);

    if (tid == 0) {
        issue_conv_tile<NO>(tmem_d, saddr(sA), saddr(sB));  // output row y0 + rr in columns [NO rr, NO rr + NO)
        mma_commit(&mbar);
    }
    if (mma_wait(&mbar)) {
        const int m = warp * 32 + lane;  // TMEM lane = pixel of the tile
#pragma unroll 1
        for (int rr = 0; rr < TR; ++rr) {
            const uint32_t taddr = tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)(NO * rr);
            const size_t pix = img + (size_t)(y0 + rr) * W + x0 + m;
            if constexpr (NO == 32) {
                epilogue32(taddr, bias, y, blockIdx.y, H, W, y0 + rr, x0 + m);
            } else {
                uint32_t r0;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n" : "=r"(r0) : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                yf[pix] = (__uint_as_float(r0) + bias[0]) * out_scale;
            }
        }
    } else if (lane == 0) {
        atomicExch(err, 1);
    }
    tc_teardown<TMEM_COLS>(tmem_d);
}

// ------------------------------------------------------------------------------------------
// 3 -> 32 layer on the tensor cores: K = 27 (channel ci, tap ky, kx at k = 9 ci + 3 ky + kx),
// padded to 32.  The inputs are three f32 planes p[c] (image b at p[c] + b * pstride) times
// s[c]; the im2col tile of TR rows x 128 pixels is built in shared memory as 4 chunk planes of
// [pixel][8 k] bf16.  Weights [chunk][32 co][8 k] bf16 (k >= 27 zero).  GELU, bf16 output in the
// padded chunk-planar layout.
// ------------------------------------------------------------------------------------------
struct FirstIn {
    const float *p[3];
    float s[3];
    size_t pstride;
};
constexpr int PLANE_F = TR * TM * 16;        // bytes of one chunk plane of the im2col tile
constexpr int B_FIRST = 4 * C * 16;          // 2 KB of weights
constexpr int SMEM_FIRST = 4 * PLANE_F + B_FIRST;
constexpr int NT_FIRST = TR * TM;            // 256: one im2col pixel each; warps 4 rr + q read row rr

// w0[co][ci][3][3] f32 -> [chunk][co][8] bf16
static __global__ void k_pack_first(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wtc)
{
    for (int e = threadIdx.x; e < 4 * C * 8; e += blockDim.x) {
        const int ch = e / (C * 8), r = e % (C * 8), co = r / 8, k = ch * 8 + r % 8;
        wtc[e] = __float2bfloat16_rn(k < 27 ? w[co * 27 + k] : 0.0f);
    }
}

static __global__ void __launch_bounds__(NT_FIRST) k_conv_tc_first(FirstIn in, const __nv_bfloat16 *__restrict__ wtc,
                                                      const float *__restrict__ bias, __nv_bfloat16 *__restrict__ y,
                                                      int H, int W, int *__restrict__ err)
{
    constexpr int COLS = C * TR;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    unsigned char *sA = sm;
    unsigned char *sB = sm + 4 * PLANE_F;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles_x = W / TM;
    const int y0 = (blockIdx.x / tiles_x) * TR;
    const int x0 = (blockIdx.x % tiles_x) * TM;
    const int b = blockIdx.y;
    for (int e = tid; e < B_FIRST / 16; e += NT_FIRST) cp16(sB + e * 16, wtc + (size_t)e * 8);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    // im2col: one pixel of the TR x 128 tile per thread
    {
        const int pi = tid;  // = rr * 128 + m
        const int rr = pi / TM, m = pi - rr * TM;
        const int yy = y0 + rr, xx = x0 + m;
        const int xm = wrap(xx - 1, W), xp = wrap(xx + 1, W);
        __align__(16) __nv_bfloat16 v[32];
#pragma unroll
        for (int ci = 0; ci < 3; ++ci) {
            const float *pl = in.p[ci] + (size_t)b * in.pstride;
#pragma unroll
            for (int ky = 0; ky < 3; ++ky) {
                const float *row = pl + (size_t)wrap(yy + ky - 1, H) * W;
                v[ci * 9 + ky * 3 + 0] = __float2bfloat16_rn(row[xm] * in.s[ci]);
                v[ci * 9 + ky * 3 + 1] = __float2bfloat16_rn(row[xx] * in.s[ci]);
                v[ci * 9 + ky * 3 + 2] = __float2bfloat16_rn(row[xp] * in.s[ci]);
            }
        }
#pragma unroll
        for (int k = 27; k < 32; ++k) v[k] = __float2bfloat16_rn(0.0f);
        const uint4 *src = reinterpret_cast<const uint4 *>(v);
#pragma unroll
        for (int c = 0; c < 4; ++c) *reinterpret_cast<uint4 *>(sA + c * PLANE_F + pi * 16) = src[c];
    }
    const uint32_t tmem_d = tc_setup<COLS>(&tmem_base, &mbar);
    if (tid == 0) {
        const uint32_t a0 = saddr(sA), b0 = saddr(sB);
        constexpr uint32_t idesc = TcShape<32>::IDESC;
#pragma unroll
        for (int rr = 0; rr < TR; ++rr)
#pragma unroll
            for (int h = 0; h < 2; ++h)
                mma_bf16(tmem_d + (uint32_t)(C * rr), smem_desc(a0 + (2 * h) * PLANE_F + rr * TM * 16, PLANE_F, 128),
                         smem_desc(b0 + (2 * h) * C * 16, C * 16, 128), idesc, h ? 1u : 0u);
        mma_commit(&mbar);
    }
    if (mma_wait(&mbar)) {
        // warp w: TMEM lanes 32 (w % 4) .. (pixels) of output row w / 4
        const int qd = warp & 3, rr = warp >> 2;
        const uint32_t taddr = tmem_d + ((uint32_t)(qd * 32) << 16) + (uint32_t)(C * rr);
        epilogue32(taddr, bias, y, b, H, W, y0 + rr, x0 + qd * 32 + lane);
    } else if (lane == 0) {
        atomicExch(err, 1);
    }
    tc_teardown<COLS>(tmem_d);
}

}  // namespace cnntc
}  // namespace dns2d
