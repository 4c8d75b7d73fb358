// cluster.cuh — large-grid path: every row / column transform of length L = 4 M is spread over a
// cluster of 4 CTAs (thread-block cluster, distributed shared memory).
//
// At N = 29400 a row of the padded grid holds L = 44100 complex values (353 KB), more than one
// CTA's shared memory (at N = 16384, 24576 values: 197 KB, too large for the two-array column
// CTA), so each transform is split as L = 4 x M:
//   forward (decimation in frequency, cluster radix first):
//     X[4 k2 + c] = sum_m W_M^{m k2} [ W_L^{m c} sum_s x[m + M s] W_4^{s c} ]
//     -> for every m one radix-4 butterfly over x[m + M s], twiddled by W_L^{m c}, whose output
//        c is written into CTA c's shared memory at position m (DSMEM store); then every CTA
//        runs an M-point Stockham FFT on its array and holds X[4 k2 + c] at position k2.
//   inverse (decimation in time, cluster radix last):
//     x[m + M s] = sum_c W_4^{-s c} [ W_L^{-m c} P_c[m] ],  P_c = M-point inverse FFT of
//     X[4 k2 + c] over k2
//     -> every CTA transforms its own array, then for every m one radix-4 butterfly reads
//        P_c[m] from the 4 CTAs (DSMEM loads) and yields the 4 physical values x[m + M s].
// The inverse's butterfly for m produces exactly the 4 values the forward's butterfly for m
// consumes, so the row pass goes C2R -> products -> R2C with the products in registers, as in
// the single-CTA kernels.  Each m is owned by one thread of one CTA, which reads position m in
// all 4 CTAs and writes the same positions back: no two threads touch one position between
// cluster barriers.
//
// The HBM traffic stays at the two-pass minimum of the single-CTA design: the row pass reads
// U, W and writes D, E once; the column pass reads D, E and om2, fnm1 and writes om2, fnm1, U, W
// once.  The twiddles W_L^{c m} (c = 1..3, m < M) are the catalog stage (R = 4, Ns = M), built in
// FP64 and rounded once like the per-stage tables.
#pragma once
#include <cooperative_groups.h>

#include "dns2d_kernels.cuh"

namespace dns2d {
namespace cg = cooperative_groups;

template <int N_>
struct CfgC {
    static constexpr bool enabled = false;
};

#define DNS2D_CFGC(N_, NT_, MINBR_, MINBC_, PS_, ...)                                          \
    template <>                                                                                \
    struct CfgC<N_> {                                                                          \
        static constexpr bool enabled = true;                                                  \
        static constexpr int N = N_, H = N_ / 2, L = 3 * N_ / 2, M = L / 4, PS = PS_;          \
        static constexpr int MP = SmemLen<M, PS_>::value, NT = NT_, MINB_R = MINBR_, MINB_C = MINBC_; \
        static constexpr int MQ = (M + 3) / 4; /* butterflies of the cluster radix per CTA */ \
        using Plan = Radices<__VA_ARGS__>;                                                     \
        static_assert(L % 4 == 0 && radix_product(Plan{}) == M, "plan");                       \
    };
// NT threads per CTA (at least M / R for every radix R of the plan); CTAs per SM asked of the
// register allocator for the row kernels (MINB_R) and the column kernels (MINB_C, two arrays of
// shared memory and more live values), each the faster of the candidates measured on B200;
// shared-memory padding PS (one float2 every 2^PS) from the half-warp bank-conflict model of the
// local plan's stages: every 16 makes the power-of-two-rich plans conflict-free (1.17x -> 1.0x
// the ideal wavefronts at M = 3072 and 6144, 1.21x -> 1.08x at 3456), every 256 suits the odd
// radices of M = 11025 (1.55x -> 1.32x)
//           N      NT  MINB_R MINB_C PS  local radix plan (product = 3N/8)
DNS2D_CFGC(840,    63,  1, 1,  5,  7, 5, 9)     // L = 1260 = 4 x 315 (test size of the cluster path)
DNS2D_CFGC(8192,  256,  4, 3,  4,  16, 16, 12)  // L = 12288 = 4 x 3072
DNS2D_CFGC(9216,  288,  4, 3,  4,  16, 12, 18)  // L = 13824 = 4 x 3456 = 2^9 3^3
DNS2D_CFGC(16384, 384,  3, 2,  4,  16, 16, 24)  // L = 24576 = 4 x 6144 (the reference's N=16384 runs)
DNS2D_CFGC(29400, 525,  1, 1,  8,  21, 21, 25)  // L = 44100 = 4 x 11025 = 2^2 3^2 5^2 7^2
#undef DNS2D_CFGC

template <int N>
constexpr TwCatalog make_catalog_c()
{
    TwCatalog c;
    c.add(typename CfgC<N>::Plan{});
    const int cross[] = {CfgC<N>::M, 4};  // adds the stage (4, Ns = M): W_L^{r m}, r = 1..3
    c.add_plan(cross, 2);
    return c;
}

template <int N>
struct TwCatC {
    static constexpr TwCatalog cat = make_catalog_c<N>();
    static constexpr int off(int R, int NS) { return cat.find(R, NS); }
};

// W_L^{r m} (forward sign) from the cross stage table, r = 1..3
template <int N>
__device__ __forceinline__ float2 cross_tw(const float2 *__restrict__ tw, int r, int m)
{
    constexpr int OFF = TwCatC<N>::off(4, CfgC<N>::M);
    static_assert(OFF >= 0, "cross stage missing from the catalog");
    return __ldg(tw + OFF + (size_t)(r - 1) * CfgC<N>::M + m);
}

// Cluster barrier without release / acquire ordering.  Used where the barrier only has to hold
// every CTA of the cluster (all started before distributed shared memory is written; none gone
// while a peer still reads its shared memory), and nothing written before it is read across the
// cluster after it.  A full cl.sync() there would also wait for this thread's outstanding global
// stores.  Remote values read before it are already consumed (they feed the stores issued before
// the barrier), so those reads are complete.
__device__ __forceinline__ void cluster_sync_relaxed()
{
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
    asm volatile("barrier.cluster.wait.aligned;\n" ::: "memory");
}

// the 4 CTAs' copies of a shared-memory array
struct Peers {
    float2 *p[4];
    __device__ __forceinline__ Peers(cg::cluster_group &cl, float2 *s)
    {
#pragma unroll
        for (int r = 0; r < 4; ++r) p[r] = cl.map_shared_rank(s, r);
    }
};

// forward cluster butterfly for position m: x[s] = x[m + M s] in, output c to CTA c
template <int N>
__device__ __forceinline__ void cross_fwd(float2 (&x)[4], const Peers &dst, int m, const float2 *tw)
{
    DFT<4, false>::run(x);
#pragma unroll
    for (int r = 1; r < 4; ++r) x[r] = cmul(x[r], cross_tw<N>(tw, r, m));
#pragma unroll
    for (int r = 0; r < 4; ++r) dst.p[r][sidx<CfgC<N>::PS>(m)] = x[r];
}

// inverse cluster butterfly for position m: P_c[m] from the 4 CTAs in, x[m + M s] out
template <int N>
__device__ __forceinline__ void cross_inv(float2 (&x)[4], const Peers &src, int m, const float2 *tw)
{
#pragma unroll
    for (int r = 0; r < 4; ++r) x[r] = src.p[r][sidx<CfgC<N>::PS>(m)];
#pragma unroll
    for (int r = 1; r < 4; ++r) x[r] = cmul(x[r], cconj(cross_tw<N>(tw, r, m)));
    DFT<4, true>::run(x);
}

// Hermitian packing of U + iW (row z) at mode k (C2R semantics: Re only on kx = 0)
template <int L, int H>
__device__ __forceinline__ float2 packed_uw(const float2 *__restrict__ U, const float2 *__restrict__ W, int k)
{
    const bool lo = k < H, hi = k > L - H;
    if (!lo && !hi) return make_float2(0.f, 0.f);
    const int kk = lo ? k : L - k;
    const float2 a = U[(size_t)kk << 2], b = W[(size_t)kk << 2];
    if (k == 0) return make_float2(a.x, b.x);
    if (lo) return make_float2(a.x - b.y, a.y + b.x);
    return make_float2(a.x + b.y, b.x - a.y);
}

// ------------------------------------------------------------------------------------------
// Row pass: U, W row z -> C2R -> (u + iw)^2 -> R2C -> D, E row z.  Grid (4 L, members).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_R) k_rows_step_c(Pointers p0)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int z = blockIdx.x >> 2;
    const Peers pe(cl, s);
    const float2 *__restrict__ U = p.work + widx<L, H>(0, z, 0);
    const float2 *__restrict__ W = p.work + widx<L, H>(1, z, 0);
    // Q[k] of the Hermitian packing belongs to CTA k % 4 at position k / 4.  Each CTA reads a
    // contiguous quarter of U, W (k < H) once and stores Q[k] and Q[L-k] into the owners' shared
    // memory; the zero band [H, L-H] is cleared locally.  The first barrier makes sure every CTA
    // of the cluster runs before shared memory is written across it.
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) {
        const int k = 4 * k2 + c;
        if (k >= H && k <= L - H) s[sidx<CfgC<N>::PS>(k2)] = make_float2(0.f, 0.f);
    }
    cluster_sync_relaxed();
    {
        constexpr int HQ = (H + 3) / 4;
        const int k0 = c * HQ, k1 = min(H, k0 + HQ);
        for (int k = k0 + (int)threadIdx.x; k < k1; k += NT) {
            const float2 a = U[(size_t)k << 2], b = W[(size_t)k << 2];
            if (k == 0) {
                pe.p[0][sidx<CfgC<N>::PS>(0)] = make_float2(a.x, b.x);
            } else {
                pe.p[k & 3][sidx<CfgC<N>::PS>(k >> 2)] = make_float2(a.x - b.y, a.y + b.x);
                const int km = L - k;
                pe.p[km & 3][sidx<CfgC<N>::PS>(km >> 2)] = make_float2(a.x + b.y, b.x - a.y);
            }
        }
    }
    cl.sync();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    const int m1 = min(M, (c + 1) * MQ);
    for (int m = c * MQ + threadIdx.x; m < m1; m += NT) {
        float2 x[4];
        cross_inv<N>(x, pe, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = make_float2(x[q].x * x[q].x - x[q].y * x[q].y, 2.0f * x[q].x * x[q].y);
        cross_fwd<N>(x, pe, m, p.tw);
    }
    cl.sync();
    fft_run<Cat, M, MP, false, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    // unpack D = (Q[k] + conj Q[L-k]) / 2, E = -i (Q[k] - conj Q[L-k]) / 4 for k < H; Q[k] sits in
    // CTA k % 4 at position k / 4.  Each CTA writes a contiguous quarter of the k range.
    float2 *__restrict__ Do = p.work + widx<L, H>(0, z, 0);
    float2 *__restrict__ Eo = p.work + widx<L, H>(1, z, 0);
    {
        constexpr int HQ = (H + 3) / 4;
        const int k0 = c * HQ, k1 = min(H, k0 + HQ);
        for (int k = k0 + (int)threadIdx.x; k < k1; k += NT) {
            const int kp = (k == 0) ? 0 : L - k;
            const float2 q = pe.p[k & 3][sidx<CfgC<N>::PS>(k >> 2)];
            const float2 m = pe.p[kp & 3][sidx<CfgC<N>::PS>(kp >> 2)];
            Do[(size_t)k << 2] = make_float2(0.5f * (q.x + m.x), 0.5f * (q.y - m.y));
            Eo[(size_t)k << 2] = make_float2(0.25f * (q.y + m.y), -0.25f * (q.x - m.x));
        }
    }
    cluster_sync_relaxed();
}

// kz index kzi = 4 k2 + c of this CTA -> compact iz (-1: the 3/2 padding band)
template <int N>
__device__ __forceinline__ int iz_of_kzi(int kzi, int &kz)
{
    constexpr int H = N / 2, L = 3 * N / 2;
    if (kzi < H) {
        kz = kzi;
        return kzi;
    }
    if (kzi >= L - H) {
        kz = kzi - L;
        return kz + N;
    }
    kz = 0;
    return -1;
}

// cluster-wide FP64 (E, Z) partial of column kx -> part[kx]; the last column's rank-0 CTA sums
// the partials in column order into hist[slot] (deterministic)
template <int NT>
__device__ __forceinline__ void cluster_energy(cg::cluster_group &cl, const Pointers &p, int kx, int ncols,
                                               double2 *cpart, double2 *red, bool *am_last, int hist_slot)
{
    if (cl.block_rank() == 0) {
        if (threadIdx.x == 0) {
            double2 acc = make_double2(0.0, 0.0);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double2 q = *cl.map_shared_rank(cpart, r);
                acc.x += q.x;
                acc.y += q.y;
            }
            p.part[kx] = acc;
            __threadfence();
            const unsigned int n = atomicAdd(p.counter, 1u);
            *am_last = (n == (unsigned)ncols - 1);
        }
        __syncthreads();
        if (*am_last) {
            double2 acc = make_double2(0.0, 0.0);
            for (int i = threadIdx.x; i < ncols; i += NT) {
                const double2 q = __ldcg(&p.part[i]);
                acc.x += q.x;
                acc.y += q.y;
            }
            acc = block_sum2<NT>(acc, red);
            if (threadIdx.x == 0) {
                p.hist[hist_slot] = acc;
                *p.counter = 0u;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// Column pass: D, E column kx -> z-forward -> FN, CN/AB2 update, FNM1 <- FN, velocity recovery,
// 3/2 padding -> z-inverse -> U, W column kx.  Grid (4 H, members).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_C)
    k_cols_step_c(Pointers p0, int first, int hist_slot)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    __shared__ double2 red[32];
    __shared__ double2 cpart;
    __shared__ bool am_last;
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int kx = blockIdx.x >> 2;
    float2 *sD = s, *sE = s + MP;
    const Peers pD(cl, sD), pE(cl, sE);
    const int m0 = c * MQ, m1 = min(M, (c + 1) * MQ);
    cluster_sync_relaxed();  // every CTA of the cluster running before its shared memory is written
    for (int m = m0 + threadIdx.x; m < m1; m += NT) {
        float2 d[4], e[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            d[q] = p.work[widx<L, H>(0, m + q * M, kx)];
            e[q] = p.work[widx<L, H>(1, m + q * M, kx)];
        }
        cross_fwd<N>(d, pD, m, p.tw);
        cross_fwd<N>(e, pE, m, p.tw);
    }
    cl.sync();
    fft_run<Cat, M, MP, false, 1, NT, CfgC<N>::PS>(sD, p.tw, typename C::Plan{});
    fft_run<Cat, M, MP, false, 1, NT, CfgC<N>::PS>(sE, p.tw, typename C::Plan{});

    const StepParams prm = *p.prm;
    const float dt = prm.dt;
    const float cnm1 = first ? prm.cnm1_first : prm.cn;
    const double hvdt = 0.5 * (double)prm.visc * (double)dt;
    const double c2n = 0.5 * (double)dt * (2.0 + (double)cnm1);
    const double c3n = -0.5 * (double)dt * (double)cnm1;
    const float divxz = (float)(1.0 / ((double)L * (double)L));
    double2 ez = make_double2(0.0, 0.0);
    const double wgt = (kx == 0) ? 0.5 : 1.0;
    float2 *om2c = p.om2 + (size_t)kx * N;
    float2 *fnc = p.fnm1 + (size_t)kx * N;
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) {
        int kz;
        const int iz = iz_of_kzi<N>(4 * k2 + c, kz);
        if (iz < 0) {
            sD[sidx<CfgC<N>::PS>(k2)] = make_float2(0.f, 0.f);
            sE[sidx<CfgC<N>::PS>(k2)] = make_float2(0.f, 0.f);
            continue;
        }
        const float2 d = sD[sidx<CfgC<N>::PS>(k2)];
        const float2 e = sE[sidx<CfgC<N>::PS>(k2)];
        float2 fn = make_float2(0.f, 0.f);
        if (kz != -H) {
            const float ga = (float)kz * (float)kx;
            const float g2a2 = (float)kz * (float)kz - (float)kx * (float)kx;
            fn.x = (ga * d.x + g2a2 * e.x) * divxz;
            fn.y = (ga * d.y + g2a2 * e.y) * divxz;
            if (p.force) fn = add_forcing(fn, p, kx, iz, N);
        }
        const double K2 = (double)kx * kx + (double)kz * kz;
        const float2 on = cn_update(om2c[iz], fn, fnc[iz], K2, hvdt, c2n, c3n);
        om2c[iz] = on;
        fnc[iz] = fn;
        float2 u, w;
        double invK2;
        recover_velocity(kx, kz, on, u, w, invK2);
        sD[sidx<CfgC<N>::PS>(k2)] = u;
        sE[sidx<CfgC<N>::PS>(k2)] = w;
        const double pw = (double)on.x * on.x + (double)on.y * on.y;
        ez.x += wgt * pw * invK2;
        ez.y += wgt * pw;
    }
    ez = block_sum2<NT>(ez, red);
    if (threadIdx.x == 0) cpart = ez;
    __syncthreads();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(sD, p.tw, typename C::Plan{});
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(sE, p.tw, typename C::Plan{});
    cl.sync();
    cluster_energy<NT>(cl, p, kx, gridDim.x >> 2, &cpart, red, &am_last, hist_slot);
    for (int m = m0 + threadIdx.x; m < m1; m += NT) {
        float2 x[4];
        cross_inv<N>(x, pD, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) p.work[widx<L, H>(0, m + q * M, kx)] = x[q];
        cross_inv<N>(x, pE, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) p.work[widx<L, H>(1, m + q * M, kx)] = x[q];
    }
    cluster_sync_relaxed();
}

// ------------------------------------------------------------------------------------------
// Column set-up (k_cols_init semantics): mode 0 from the compact velocity spectrum uw (om2 =
// i (kz u - kx w), fnm1 = 0), mode 1 velocity recovery from om2.  -> U, W columns.
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_C)
    k_cols_init_c(Pointers p0, const float2 *__restrict__ uw, int mode)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int kx = blockIdx.x >> 2;
    float2 *sU = s, *sW = s + MP;
    const Peers pU(cl, sU), pW(cl, sW);
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) {
        int kz;
        const int iz = iz_of_kzi<N>(4 * k2 + c, kz);
        float2 u = make_float2(0.f, 0.f), w = u;
        if (iz >= 0) {
            if (mode == 0) {
                const size_t b = 2 * ((size_t)iz * H + kx);
                u = uw[b];
                w = uw[b + 1];
                const float gz = (float)kz, ax = (float)kx;
                const float dx_ = gz * u.x - ax * w.x, dy_ = gz * u.y - ax * w.y;
                p.om2[(size_t)kx * N + iz] = make_float2(-dy_, dx_);
                p.fnm1[(size_t)kx * N + iz] = make_float2(0.f, 0.f);
            } else {
                double invK2;
                recover_velocity(kx, kz, p.om2[(size_t)kx * N + iz], u, w, invK2);
            }
        }
        sU[sidx<CfgC<N>::PS>(k2)] = u;
        sW[sidx<CfgC<N>::PS>(k2)] = w;
    }
    __syncthreads();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(sU, p.tw, typename C::Plan{});
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(sW, p.tw, typename C::Plan{});
    cl.sync();
    for (int m = c * MQ + threadIdx.x; m < min(M, (c + 1) * MQ); m += NT) {
        float2 x[4];
        cross_inv<N>(x, pU, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) p.work[widx<L, H>(0, m + q * M, kx)] = x[q];
        cross_inv<N>(x, pW, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) p.work[widx<L, H>(1, m + q * M, kx)] = x[q];
    }
    cl.sync();
}

// ------------------------------------------------------------------------------------------
// Velocity rows (k_rows_velocity semantics): U, W row -> u, w physical; optional phys planes
// and CFL maximum.
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_R)
    k_rows_velocity_c(Pointers p0, float *phys, float *cflm, float dx)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    __shared__ float red[32];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int z = blockIdx.x >> 2;
    const Peers pe(cl, s);
    const float2 *__restrict__ U = p.work + widx<L, H>(0, z, 0);
    const float2 *__restrict__ W = p.work + widx<L, H>(1, z, 0);
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) s[sidx<CfgC<N>::PS>(k2)] = packed_uw<L, H>(U, W, 4 * k2 + c);
    __syncthreads();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    float mx = 0.0f;
    for (int m = c * MQ + threadIdx.x; m < min(M, (c + 1) * MQ); m += NT) {
        float2 x[4];
        cross_inv<N>(x, pe, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (phys) {
                const size_t o = (size_t)z * L + m + q * M;
                phys[o] = x[q].x;
                phys[(size_t)L * L + o] = x[q].y;
            }
            mx = fmaxf(mx, cfl_term(x[q].x, x[q].y, dx));
        }
    }
    cl.sync();
    if (cflm) {
        mx = block_max<NT>(mx, red);
        if (threadIdx.x == 0) atomic_max_nonneg(cflm + blockIdx.y, mx);
    }
}

// ------------------------------------------------------------------------------------------
// Physical rows -> U, W rows (k_rows_from_phys semantics, x-forward of u + iw scaled by 1/L).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_R)
    k_rows_from_phys_c(Pointers p, const float *phys)
{
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int z = blockIdx.x >> 2;
    const Peers pe(cl, s);
    cluster_sync_relaxed();  // every CTA of the cluster running before its shared memory is written
    for (int m = c * MQ + threadIdx.x; m < min(M, (c + 1) * MQ); m += NT) {
        float2 x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const size_t o = (size_t)z * L + m + q * M;
            x[q] = make_float2(phys[o], phys[(size_t)L * L + o]);
        }
        cross_fwd<N>(x, pe, m, p.tw);
    }
    cl.sync();
    fft_run<Cat, M, MP, false, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    const float sc = 1.0f / (float)L;
    float2 *__restrict__ Uo = p.work + widx<L, H>(0, z, 0);
    float2 *__restrict__ Wo = p.work + widx<L, H>(1, z, 0);
    for (int k2 = threadIdx.x; 4 * k2 + c < H; k2 += NT) {
        const int k = 4 * k2 + c;
        const int kp = (k == 0) ? 0 : L - k;
        const float2 q = s[sidx<CfgC<N>::PS>(k2)];
        const float2 m = pe.p[kp & 3][sidx<CfgC<N>::PS>(kp >> 2)];
        Uo[(size_t)k << 2] = make_float2(0.5f * sc * (q.x + m.x), 0.5f * sc * (q.y - m.y));
        Wo[(size_t)k << 2] = make_float2(0.5f * sc * (q.y + m.y), -0.5f * sc * (q.x - m.x));
    }
    cl.sync();
}

// ------------------------------------------------------------------------------------------
// Scalar field to physical space (k_cols_scalar / k_rows_scalar semantics).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_C)
    k_cols_scalar_c(Pointers p, float2 *scratch, int kind)
{
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int kx = blockIdx.x >> 2;
    const Peers pe(cl, s);
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) {
        int kz;
        const int iz = iz_of_kzi<N>(4 * k2 + c, kz);
        float2 v = make_float2(0.f, 0.f);
        if (iz >= 0) {
            v = p.om2[(size_t)kx * N + iz];
            if (kind == 1) {
                const float k2f = (float)kx * (float)kx + (float)kz * (float)kz + 1.0e-30f;
                v = make_float2(v.x / k2f, v.y / k2f);
                if (kx == 0 && iz == 0) v = make_float2(0.f, 0.f);
            }
        }
        s[sidx<CfgC<N>::PS>(k2)] = v;
    }
    __syncthreads();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    for (int m = c * MQ + threadIdx.x; m < min(M, (c + 1) * MQ); m += NT) {
        float2 x[4];
        cross_inv<N>(x, pe, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) scratch[widx<L, H>(0, m + q * M, kx)] = x[q];
    }
    cl.sync();
}

template <int N>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(CfgC<N>::NT, CfgC<N>::MINB_R)
    k_rows_scalar_c(Pointers p, const float2 *scratch, float *out, float2 *minmax)
{
    using C = CfgC<N>;
    using Cat = TwCatC<N>;
    constexpr int L = C::L, H = C::H, M = C::M, MP = C::MP, NT = C::NT, MQ = C::MQ;
    extern __shared__ float2 s[];
    __shared__ float red[32];
    __shared__ float s_nmn;
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int z = blockIdx.x >> 2;
    const Peers pe(cl, s);
    const float2 *__restrict__ A = scratch + widx<L, H>(0, z, 0);
    for (int k2 = threadIdx.x; k2 < M; k2 += NT) {
        const int k = 4 * k2 + c;
        float2 v = make_float2(0.f, 0.f);
        if (k == 0) {
            v = make_float2(A[0].x, 0.f);
        } else if (k < H) {
            v = A[(size_t)k << 2];
        } else if (k > L - H) {
            const float2 a = A[(size_t)(L - k) << 2];
            v = make_float2(a.x, -a.y);
        }
        s[sidx<CfgC<N>::PS>(k2)] = v;
    }
    __syncthreads();
    fft_run<Cat, M, MP, true, 1, NT, CfgC<N>::PS>(s, p.tw, typename C::Plan{});
    cl.sync();
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (int m = c * MQ + threadIdx.x; m < min(M, (c + 1) * MQ); m += NT) {
        float2 x[4];
        cross_inv<N>(x, pe, m, p.tw);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            out[(size_t)z * L + m + q * M] = x[q].x;
            mn = fminf(mn, x[q].x);
            mx = fmaxf(mx, x[q].x);
        }
    }
    cl.sync();
    const float nmn = block_max<NT>(-mn, red);
    if (threadIdx.x == 0) s_nmn = nmn;
    const float bmx = block_max<NT>(mx, red);
    if (threadIdx.x == 0) minmax[blockIdx.x] = make_float2(-s_nmn, bmx);
}

}  // namespace dns2d
