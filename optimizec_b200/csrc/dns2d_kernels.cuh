// dns2d_kernels.cuh — device kernels of the fused 2D vorticity step.
//
// Data layout in HBM (N base modes, L = 3N/2 padded grid, H = N/2 retained kx):
//   om2, fnm1 : [kx][kz] complex64, kz in compact order iz (kz = iz < N/2 ? iz : iz - N).
//               The reference keeps [iz][ix] (cuda/cuda_dns.h:62-63); the column pass reads
//               whole kx columns, so the state is stored transposed here and converted at the
//               API boundary.
//   work      : [2][L/4][H][4] complex64.  Component c, physical row z, mode kx sits at
//               ((z/4)*H + kx)*4 + z%4.  Between the column pass and the row pass it holds the
//               velocity after the z-inverse transform, U(z,kx) and W(z,kx); between the row
//               pass and the column pass it holds the x-forward transforms of the products,
//               D(z,kx) = F_x[u^2 - w^2] and E(z,kx) = F_x[u w].  Groups of 4 rows are
//               contiguous per kx, so the row pass reads/writes whole 4-row tiles and the column
//               pass moves full 32-byte sectors.
//
// One time step of the reference (cuda/mem_cuda.cu:1848-1857: STEP2B -> STEP3 -> STEP2A)
// becomes two kernels:
//   row pass    (k_rows_step):  U,W rows -> C2R -> u,w -> (u+iw)^2 -> R2C -> D,E rows
//               = STEP2A's x-inverse + STEP2B's products and x-forward
//   column pass (k_cols_step):  D,E columns -> z-forward (kz in [-N/2,N/2)) -> FN ->
//               Crank-Nicolson/AB2 update of om2, fnm1 <- FN -> velocity recovery ->
//               3/2 zero-padding -> z-inverse -> U,W columns
//               = STEP2B's z-forward + zero row N, STEP3, STEP2A's dealias/reshuffle/z-inverse
#pragma once
#include "fft.cuh"


namespace dns2d {

// ------------------------------------------------------------------------------------------
// per-size configuration
// ------------------------------------------------------------------------------------------
template <int N_>
struct Cfg;

// per-stage twiddle catalog of size N (defined below, after the large-grid plans)
template <int N>
struct TwCat;

#define DNS2D_CFG(N_, ROWS_, NTB_, NTA_, PS_, EX_, ...)                                      \
    template <>                                                                                \
    struct Cfg<N_> {                                                                           \
        static constexpr int N = N_;                                                           \
        static constexpr int H = N_ / 2;                                                       \
        static constexpr int L = 3 * N_ / 2;                                                   \
        static constexpr int PS = PS_; /* shared-memory padding: one float2 every 2^PS */      \
        static constexpr int LP = SmemLen<L, PS_, EX_>::value;                                 \
        static constexpr int ROWS = ROWS_;                                                     \
        static constexpr int NTB = NTB_;                                                       \
        static constexpr int NTA = NTA_;                                                       \
        using Plan = Radices<__VA_ARGS__>;                                                     \
    };

// Padding (PS) and array stride (EX, the float2 added to the 16-rounded padded length) of the
// small sizes, chosen with a model of the half-warp bank conflicts of every stage of their three
// radix plans, rows (4 or 8 arrays per CTA) and columns (2 arrays); e.g. N = 128, plan (16, 12):
// 2.0x / 1.71x the conflict-free wavefronts with one float2 every 32 and arrays 4 apart, 1.12x /
// 1.07x with one every 16 and arrays 12 apart; N = 512, plan (16, 16, 3): 1.17x -> 1.0x.
//          N     ROWS  NTB  NTA  PS EX  radix plan (product = 3N/2)
DNS2D_CFG(16,    4,   64,  32,  5, 4,  4, 6)
DNS2D_CFG(32,    4,   64,  32,  5, 4,  8, 6)
DNS2D_CFG(64,    4,  128,  64,  4, 8,  8, 12)
DNS2D_CFG(128,   4,  192,  64,  4, 12, 16, 12)
DNS2D_CFG(256,   4,  256, 128,  4, 9,  16, 24)
DNS2D_CFG(512,   4,  384, 192,  4, 0,  16, 16, 3)
DNS2D_CFG(1024,  4,  512, 256,  5, 4,  16, 8, 12)
DNS2D_CFG(2048,  4,  768, 384,  5, 4,  16, 16, 12)
DNS2D_CFG(4096,  2,  768, 768,  5, 4,  16, 16, 24)
#undef DNS2D_CFG

// Alternative radix plans of the small-grid row and column passes (k_rows_step, k_cols_step),
// chosen per device by the autotuner; plan 0 is Cfg<N>::Plan.  The plans factor L differently or
// in another order, so they round differently (each within the FP32 tolerance of the oracle
// tests); the large sizes run plan-specialised kernels and have one plan.
template <int N>
struct AltPlans {
    static constexpr int count = 1;
    using P1 = typename Cfg<N>::Plan;
    using P2 = typename Cfg<N>::Plan;
};
template <>
struct AltPlans<64> {
    static constexpr int count = 3;
    using P1 = Radices<12, 8>;
    using P2 = Radices<4, 24>;
};
template <>
struct AltPlans<128> {
    static constexpr int count = 3;
    using P1 = Radices<12, 16>;
    using P2 = Radices<8, 24>;
};
template <>
struct AltPlans<256> {
    static constexpr int count = 3;
    using P1 = Radices<24, 16>;
    using P2 = Radices<8, 6, 8>;
};
template <>
struct AltPlans<512> {
    static constexpr int count = 3;
    using P1 = Radices<3, 16, 16>;
    using P2 = Radices<8, 8, 12>;
};

// work-buffer index (float2 units) of component c, physical row z, mode kx
template <int L, int H>
__device__ __forceinline__ size_t widx(int c, int z, int kx)
{
    return (size_t)c * ((size_t)L * H) + (((size_t)(z >> 2) * H + kx) << 2) + (z & 3);
}

// parameters that change between segments of the run (read from device memory so a captured
// CUDA graph can be replayed with new values)
struct StepParams {
    float dt;          // time step of this segment
    float cnm1_first;  // CNM1 seen by the first step of the segment (host value before it)
    float cn;          // CN; after the first step the reference has CNM1 == CN
    float visc;        // viscosity
};

struct Pointers {
    float2 *om2;
    float2 *fnm1;
    float2 *work;
    const float2 *tw;       // per-stage twiddle tables of the size's catalog (TwCat<N>)
    const StepParams *prm;
    double2 *part;          // per-column (E, Z) partial sums, [H]
    unsigned int *counter;  // arrival counter for the last-block reduction
    double2 *hist;          // per-step (E, Z) history
    const float2 *force;    // optional spectral forcing added to FN, [kx][kz] like om2 (closure)
    const float *gate;      // optional 0/1 factor on the forcing, decided on the device per step
    // batched ensembles: member m (blockIdx.y) uses its own state, work, parameter block,
    // partials, counter and history at these strides (all 0 for a single run)
    size_t s_state, s_work;
    int s_part, s_hist;
    // kernel configuration (the autotuner's choice; every choice gives the same arithmetic):
    // rows per CTA of the small-grid row pass (0: the size's default), thread groups per column
    // CTA of the large-grid column pass (0: default), L2 prefetch distances in CTAs (0: off)
    int rows_tile = 0, cols_groups = 0;
    int pf_rows = 296, pf_cols = 74;
    // radix plan of the small-grid row / column pass (0: Cfg<N>::Plan, 1, 2: AltPlans<N>); unlike
    // the knobs above a plan changes the FP32 rounding
    int plan_rows = 0, plan_cols = 0;
    // closure forcing limiter: |forcing| <= force_clamp |FN| per mode (0: off)
    float force_clamp = 0.0f;

    __device__ __forceinline__ Pointers member(int m) const
    {
        Pointers q = *this;
        q.om2 = om2 + (size_t)m * s_state;
        q.fnm1 = fnm1 + (size_t)m * s_state;
        q.work = work + (size_t)m * s_work;
        q.prm = prm + (s_state ? m : 0);
        q.part = part + (size_t)m * s_part;
        q.counter = counter + (s_state ? m : 0);
        q.hist = hist + (size_t)m * s_hist;
        q.force = force ? force + (size_t)m * s_state : nullptr;
        q.gate = gate;
        return q;
    }
};

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------

// FN of mode (kx, iz) plus the closure forcing: times the energy gate (0/1), and with a clamp
// alpha > 0 limited in magnitude to alpha |FN| of the same mode (where the resolved transfer
// vanishes, e.g. shells the cascade has not reached, the closure adds nothing)
__device__ __forceinline__ float2 add_forcing(float2 fn, const Pointers &p, int kx, int iz, int N)
{
    const float g = p.gate ? *p.gate : 1.0f;
    const float2 f = p.force[(size_t)kx * N + iz];
    if (p.force_clamp <= 0.0f) return make_float2(fmaf(g, f.x, fn.x), fmaf(g, f.y, fn.y));
    float fx = g * f.x, fy = g * f.y;
    const float af = sqrtf(fx * fx + fy * fy), an = p.force_clamp * sqrtf(fn.x * fn.x + fn.y * fn.y);
    if (af > an) {
        const float sc = an / af;
        fx *= sc;
        fy *= sc;
    }
    return make_float2(fn.x + fx, fn.y + fy);
}

// CFL contribution |u|/DX + |w|/DZ with IEEE division/addition (cuda/dns_cuda.cu:497-502)
__device__ __forceinline__ float cfl_term(float u, float w, float dx)
{
    return __fadd_rn(__fdiv_rn(fabsf(u), dx), __fdiv_rn(fabsf(w), dx));
}

// ordered max of non-negative floats through their bit patterns
__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v)
{
    atomicMax(reinterpret_cast<unsigned int *>(addr), __float_as_uint(v));
}

template <int NT>
__device__ __forceinline__ float block_max(float v, float *red)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (NT + 31) / 32) ? red[l] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ double2 block_sum2(double2 v, double2 *red)
{
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (NT + 31) / 32) ? red[l] : make_double2(0.0, 0.0);
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
    }
    return v;  // valid in thread 0
}

// Hermitian packing of two real rows' half spectra a = F[u], b = F[w] (kx < H) into the full
// complex spectrum of u + i w.  Like a C2R transform, only Re of the kx = 0 entries is used.
template <int L, int H, int ROWS, int NT, int LP, int PS = 5>
__device__ __forceinline__ void rows_load_pack(float2 *s, const float2 *__restrict__ work, int z0)
{
    for (int e = threadIdx.x; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 a = work[widx<L, H>(0, z0 + r, k)];
        const float2 b = work[widx<L, H>(1, z0 + r, k)];
        float2 *x = s + r * LP;
        if (k == 0) {
            x[sidx<PS>(0)] = make_float2(a.x, b.x);
        } else {
            x[sidx<PS>(k)] = make_float2(a.x - b.y, a.y + b.x);
            x[sidx<PS>(L - k)] = make_float2(a.x + b.y, b.x - a.y);
        }
    }
    constexpr int NZ = L - 2 * H + 1;  // zero band kx in [H, L-H]
    for (int e = threadIdx.x; e < ROWS * NZ; e += NT) {
        const int r = e / NZ, k = H + (e - r * NZ);
        s[r * LP + sidx<PS>(k)] = make_float2(0.f, 0.f);
    }
}

// ------------------------------------------------------------------------------------------
// Row pass of one step.
// ------------------------------------------------------------------------------------------
template <int N, int ROWS = Cfg<N>::ROWS, class Plan = typename Cfg<N>::Plan>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_step(Pointers p0)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NTB;
    extern __shared__ float2 smem[];
    const int z0 = blockIdx.x * ROWS;
    rows_load_pack<L, H, ROWS, NT, LP, PS>(smem, p.work, z0);
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, ROWS, NT, PS>(smem, p.tw, Plan{});
    // products: (u + i w)^2 = (u^2 - w^2) + i (2 u w)
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        float2 *a = smem + r * LP + sidx<PS>(x);
        const float2 z = *a;
        *a = make_float2(z.x * z.x - z.y * z.y, 2.0f * z.x * z.y);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, ROWS, NT, PS>(smem, p.tw, Plan{});
    // unpack: D = F[u^2 - w^2] = (Q[k] + conj Q[L-k]) / 2, E = F[u w] = -i (Q[k] - conj Q[L-k]) / 4
    for (int e = threadIdx.x; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 *x = smem + r * LP;
        const float2 q = x[sidx<PS>(k)];
        const float2 m = x[sidx<PS>(k == 0 ? 0 : L - k)];
        p.work[widx<L, H>(0, z0 + r, k)] = make_float2(0.5f * (q.x + m.x), 0.5f * (q.y - m.y));
        p.work[widx<L, H>(1, z0 + r, k)] = make_float2(0.25f * (q.y + m.y), -0.25f * (q.x - m.x));
    }
}

// ------------------------------------------------------------------------------------------
// Crank-Nicolson / Adams-Bashforth update of one mode (cuda/step3_cuda.cu:82-100):
//   om' = ((1 - a) om + c2n FN + c3n FNM1) / (1 + a),  a = hvdt K^2,
// with the factors formed in FP64 and each rounded once to float.  The viscous part is carried
// as the decrement d1 = (1 - a)/(1 + a) - 1 = -2a/(1 + a), and om' = om + (d1 om + c2 FN + c3 FNM1)
// is rounded once: rounding the multiplier (1 - a)/(1 + a) itself to float would quantise the
// decay of the energy-bearing low-k modes, where 2a (~1e-7 K^2 at Re = 1e4) is comparable to the
// float spacing just below 1, into a systematic energy drift of ~1e-8 per step.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cn_update(float2 om, float2 fn, float2 fo, double K2, double hvdt, double c2n,
                                            double c3n)
{
    const double arg = hvdt * K2;
    const double inv = 1.0 / (1.0 + arg);
    const float d1 = (float)(-2.0 * arg * inv);
    const float c2 = (float)(c2n * inv);
    const float c3 = (float)(c3n * inv);
    const float ix = fmaf(d1, om.x, fmaf(c2, fn.x, c3 * fo.x));
    const float iy = fmaf(d1, om.y, fmaf(c2, fn.y, c3 * fo.y));
    return make_float2(om.x + ix, om.y + iy);
}

// ------------------------------------------------------------------------------------------
// Velocity recovery of one mode (cuda/step3_cuda.cu:103-138): u = -i kz om / K^2,
// w = i kx om / K^2; on kx = 0: u = -i om / kz (0 at kz = 0), w = 0.  The factors kz/K^2 and
// kx/K^2 are formed in FP64 and rounded once.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void recover_velocity(int kx, int kz, float2 om, float2 &u, float2 &w,
                                                 double &invK2)
{
    const double K2 = (double)kx * kx + (double)kz * kz;
    invK2 = (K2 > 0.0) ? 1.0 / K2 : 0.0;
    float gu, gw;
    if (kx >= 1) {
        gu = (float)((double)kz * invK2);
        gw = (float)((double)kx * invK2);
    } else {
        gu = (kz != 0) ? (float)(1.0 / (double)kz) : 0.0f;
        gw = 0.0f;
    }
    // -i * gu * om = (gu*om.y, -gu*om.x); +i * gw * om = (-gw*om.y, gw*om.x)
    u = make_float2(gu * om.y, -gu * om.x);
    w = make_float2(-gw * om.y, gw * om.x);
}

// ------------------------------------------------------------------------------------------
// Column pass of one step.
// ------------------------------------------------------------------------------------------
template <int N, class Plan = typename Cfg<N>::Plan>
__global__ void __launch_bounds__(Cfg<N>::NTA) k_cols_step(Pointers p0, int first, int hist_slot)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NTA;
    extern __shared__ float2 smem[];
    __shared__ double2 red[32];
    __shared__ bool am_last;
    const int kx = blockIdx.x;
    float2 *sD = smem, *sE = smem + LP;
    for (int z = threadIdx.x; z < L; z += NT) {
        sD[sidx<PS>(z)] = p.work[widx<L, H>(0, z, kx)];
        sE[sidx<PS>(z)] = p.work[widx<L, H>(1, z, kx)];
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, 2, NT, PS>(smem, p.tw, Plan{});

    const StepParams prm = *p.prm;
    const float dt = prm.dt;
    const float cnm1 = first ? prm.cnm1_first : prm.cn;
    // Crank-Nicolson factors in FP64: om' = ((1-a) om + dt/2 (2+cnm1) FN - dt/2 cnm1 FNM1)/(1+a)
    const double hvdt = 0.5 * (double)prm.visc * (double)dt;
    const double c2n = 0.5 * (double)dt * (2.0 + (double)cnm1);
    const double c3n = -0.5 * (double)dt * (double)cnm1;
    const float divxz = (float)(1.0 / ((double)L * (double)L));
    double2 ez = make_double2(0.0, 0.0);
    const double wgt = (kx == 0) ? 0.5 : 1.0;  // 1/2 * (1 on kx = 0, else 2)
    float2 *om2c = p.om2 + (size_t)kx * N;
    float2 *fnc = p.fnm1 + (size_t)kx * N;
    for (int iz = threadIdx.x; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        const float2 d = sD[sidx<PS>(kzi)];
        const float2 e = sE[sidx<PS>(kzi)];
        float2 fn = make_float2(0.f, 0.f);
        if (kz != -H) {  // STEP2B zeroes the kz = -N/2 row (cuda/step2b_cuda.cu:203-221)
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
        sD[sidx<PS>(kzi)] = u;
        sE[sidx<PS>(kzi)] = w;
        const double pw = (double)on.x * on.x + (double)on.y * on.y;
        ez.x += wgt * pw * invK2;
        ez.y += wgt * pw;
    }
    for (int z = H + threadIdx.x; z < L - H; z += NT) {  // 3/2 zero padding in kz
        sD[sidx<PS>(z)] = make_float2(0.f, 0.f);
        sE[sidx<PS>(z)] = make_float2(0.f, 0.f);
    }
    // energy / enstrophy of the updated field: per-column partials, the last block sums them
    // in column order (deterministic)
    ez = block_sum2<NT>(ez, red);
    if (threadIdx.x == 0) {
        p.part[kx] = ez;
        __threadfence();
        const unsigned int n = atomicAdd(p.counter, 1u);
        am_last = (n == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
        double2 acc = make_double2(0.0, 0.0);
        for (int i = threadIdx.x; i < H; i += NT) {
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
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, 2, NT, PS>(smem, p.tw, Plan{});
    for (int z = threadIdx.x; z < L; z += NT) {
        p.work[widx<L, H>(0, z, kx)] = sD[sidx<PS>(z)];
        p.work[widx<L, H>(1, z, kx)] = sE[sidx<PS>(z)];
    }
}

// ------------------------------------------------------------------------------------------
// Large-grid variants: one row / one column per CTA, one butterfly per thread and stage, three
// stages.  Row pass: inverse plan (R1, R2, R3), forward plan (R3, R2, R1) so that the inverse's
// last stage leaves in registers exactly the stride-L/R3 elements the forward's first stage
// needs: C2R -> products -> R2C runs through shared memory only four times.  The first inverse
// stage reads U, W straight from global memory.  Column pass: plan (R3, R2, R1) both ways, the
// forward's first stage read from global, the inverse's last stage written to global.
// ------------------------------------------------------------------------------------------
template <int N_>
struct Cfg2 {
    static constexpr bool enabled = false;
};

#define DNS2D_CFG2(N_, NT_, R1_, R2_, R3_, MC2_, MC4_, PS_)                                    \
    template <>                                                                                \
    struct Cfg2<N_> {                                                                          \
        static constexpr bool enabled = true;                                                  \
        static constexpr int PS = PS_; /* shared-memory padding: one float2 every 2^PS */       \
        static constexpr int N = N_, H = N_ / 2, L = 3 * N_ / 2, LP = SmemLen<L, PS_>::value;  \
        static constexpr int NT = NT_, R1 = R1_, R2 = R2_, R3 = R3_;                           \
        static constexpr int MC2 = MC2_, MC4 = MC4_; /* CTAs per SM: k_cols_step2, k_cols_step4 */ \
        static_assert(R1_ * R2_ * R3_ == L, "plan");                                           \
        static_assert(L / R1_ <= NT_ && L / R2_ <= NT_ && L / R3_ <= NT_, "one butterfly");    \
    };
// N = 4096 / 2048: plans (16, 24, 16) / (16, 12, 16) with padding every 16 elements make every
// shared-memory access of both passes bank-conflict free (the radix-24 stage has Ns = 16, so its stores are contiguous per
// half-warp, and the stride-16 stores of the Ns = 1 stages spread over all banks); the radix-16
// middle stage of the row pass also holds 16 values in registers instead of 24.
//          N    NT  plan (R1, R2, R3)  column CTAs per SM asked of the register allocator, pad
DNS2D_CFG2(1024, 192, 16, 12, 8,       2, 1, 4)
DNS2D_CFG2(2048, 256, 16, 12, 16,      2, 2, 4)  // two-group columns at 64 registers, 2 CTAs per SM
DNS2D_CFG2(4096, 384, 16, 24, 16,      2, 1, 4)
#undef DNS2D_CFG2

// twiddle catalog of size N: the stages of every plan compiled for it
template <int N>
constexpr TwCatalog make_catalog()
{
    TwCatalog c;
    c.add(typename Cfg<N>::Plan{});
    if constexpr (AltPlans<N>::count > 1) {
        c.add(typename AltPlans<N>::P1{});
        c.add(typename AltPlans<N>::P2{});
    }
    if constexpr (Cfg2<N>::enabled) {
        c.add(Radices<Cfg2<N>::R1, Cfg2<N>::R2, Cfg2<N>::R3>{});
        c.add(Radices<Cfg2<N>::R3, Cfg2<N>::R2, Cfg2<N>::R1>{});
    }
    return c;
}

template <int N>
struct TwCat {
    static constexpr TwCatalog cat = make_catalog<N>();
    static constexpr int off(int R, int NS) { return cat.find(R, NS); }
};

// Inverse x transform of a row pair on the large-grid plan: the half spectra A = U[k], B = W[k]
// (k < H, consecutive k 4 float2 apart, as in the work layout) of two real rows a, b are packed
// Hermitian-wise as A + iB and transformed (C2R semantics: only Re of the k = 0 entries is used).
// Thread j < L/R3 is left holding v[q] = (a(x), b(x)) at x = j + q L/R3; the last inverse stage
// runs in registers.  Used by the row pass (rows u, w of one physical row), NEXTDT (the same,
// for the CFL maximum) and OM2PHYS (two physical rows of one field).
template <int N>
__device__ __forceinline__ void rows_inverse2(const float2 *__restrict__ U, const float2 *__restrict__ W, float2 *s,
                                              const float2 *__restrict__ tw, float2 (&v)[Cfg2<N>::R3])
{
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, R1 = C::R1, R2 = C::R2, R3 = C::R3, PS = C::PS;
    constexpr int LR1 = L / R1, LR3 = L / R3;
    const int j = threadIdx.x;
    // inverse stage 1 (Ns = 1), inputs Z[j + r L/R1] of the Hermitian packing of U + iW.  Z at
    // k > L-H needs U, W at L-k = (L/R1 - j) + (R1-1-r) L/R1: slot R1-1-r of butterfly L/R1 - j.
    // Butterflies j and L/R1 - j share a warp 16 lanes apart, so every thread loads only its
    // k < H slots and receives the mirrored values from its partner lane; butterflies 0 and
    // L/R1/2 are their own mirrors (slots R1 - r and R1-1-r of their own loads).  Half the global
    // loads of reading both mirrors directly (N = 4096 on B200: row pass 0.334 -> 0.309 ms).
    static_assert(R1 == 16 && LR1 % 32 == 0 && C::NT >= LR1, "mirror pairing");
    if (j < LR1) {  // whole warps (L/R1 is a multiple of 32)
        const int lane = j & 31, q = (j >> 5) * 16 + (lane & 15);
        const int jb = (lane < 16) ? (q == 0 ? 0 : q) : (q == 0 ? LR1 / 2 : LR1 - q);
        float2 a[R1], b[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            a[r] = make_float2(0.f, 0.f);
            b[r] = a[r];
            const int k = jb + r * LR1;
            if (!slot_in_band<L, R1, H, L - H>(r) && r * LR1 < H && k < H) {
                a[r] = U[(size_t)k << 2];
                b[r] = W[(size_t)k << 2];
            }
        }
        float2 v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            const int k = jb + r * LR1;
            if (slot_in_band<L, R1, H, L - H>(r)) {
                v[r] = make_float2(0.f, 0.f);
            } else if ((r + 1) * LR1 <= L - H + 1) {  // slot never above L-H: lo or zero
                if (k == 0) v[r] = make_float2(a[r].x, b[r].x);
                else if (k < H) v[r] = make_float2(a[r].x - b[r].y, a[r].y + b[r].x);
                else v[r] = make_float2(0.f, 0.f);
            } else {  // slot r can be above L-H: mirrored value from slot R1-1-r of the partner
                float2 ma, mb;
                ma.x = __shfl_xor_sync(0xffffffffu, a[R1 - 1 - r].x, 16);
                ma.y = __shfl_xor_sync(0xffffffffu, a[R1 - 1 - r].y, 16);
                mb.x = __shfl_xor_sync(0xffffffffu, b[R1 - 1 - r].x, 16);
                mb.y = __shfl_xor_sync(0xffffffffu, b[R1 - 1 - r].y, 16);
                if (jb == 0) {
                    ma = a[(R1 - r) & (R1 - 1)];
                    mb = b[(R1 - r) & (R1 - 1)];
                } else if (jb == LR1 / 2) {
                    ma = a[R1 - 1 - r];
                    mb = b[R1 - 1 - r];
                }
                if (k < H) {
                    v[r] = (k == 0) ? make_float2(a[r].x, b[r].x) : make_float2(a[r].x - b[r].y, a[r].y + b[r].x);
                } else if (k > L - H) {
                    v[r] = make_float2(ma.x + mb.y, mb.x - ma.y);
                } else {
                    v[r] = make_float2(0.f, 0.f);
                }
            }
        }
        DFT<R1, true>::run(v);
        sm_store<L, R1, 1, PS>(s, v, jb);
    }
    stage1<TwCat<N>, L, R2, R1, true, PS>(s, tw);
    __syncthreads();
    if (j < LR3) {
        sm_load<L, R3, PS>(v, s, j);
        bfly<TwCat<N>, L, R3, LR3, true>(v, j, tw);
    }
}

// three CTAs per SM: the register allocator keeps the row pass at 56 registers (36 warps per SM;
// N = 4096: 0.311 -> 0.280 ms against two CTAs at 80 registers)
template <int N>
__global__ void __launch_bounds__(Cfg2<N>::NT, 3) k_rows_step2(Pointers p0)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, R1 = C::R1, R2 = C::R2, R3 = C::R3, PS = C::PS;
    constexpr int LR3 = L / R3;
    extern __shared__ float2 s[];
    const int z = blockIdx.x;
    const int j = threadIdx.x;
    const float2 *__restrict__ U = p.work + widx<L, H>(0, z, 0);
    const float2 *__restrict__ W = p.work + widx<L, H>(1, z, 0);
    // bring to L2 the quarter (z % 4) of the 4-row tile that the CTA pf_rows later reads (two
    // waves of 148 SMs x 2 CTAs by default)
    if (p.pf_rows > 0 && z + p.pf_rows < L) {
        const int t = (z + p.pf_rows) >> 2, part = z & 3;
        constexpr int QB = H * 32 / 4;  // bytes of one quarter tile of one component
        const char *b0 = reinterpret_cast<const char *>(p.work + (size_t)t * H * 4) + part * QB;
        for (int o = j * 128; o < 2 * QB; o += C::NT * 128)
            prefetch_l2(o < QB ? b0 + o : b0 + (size_t)L * H * 8 + (o - QB));
    }
    // inverse x transform; its last stage leaves u + i w in registers -> products -> forward
    // stage 1
    float2 v[R3];
    rows_inverse2<N>(U, W, s, p.tw, v);
    if (j < LR3) {
#pragma unroll
        for (int q = 0; q < R3; ++q) v[q] = make_float2(v[q].x * v[q].x - v[q].y * v[q].y, 2.0f * v[q].x * v[q].y);
        DFT<R3, false>::run(v);
    }
    __syncthreads();
    if (j < LR3) sm_store<L, R3, 1, PS>(s, v, j);
    stage1<TwCat<N>, L, R2, R3, false, PS>(s, p.tw);
    // the unpack reads Q[k] and Q[L-k] for k < H: positions in [H, L-H] are never read
    stage1_last_band<TwCat<N>, L, R1, false, H, L - H, PS>(s, p.tw);
    __syncthreads();
    float2 *__restrict__ Do = p.work + widx<L, H>(0, z, 0);
    float2 *__restrict__ Eo = p.work + widx<L, H>(1, z, 0);
    for (int k = j; k < H; k += C::NT) {
        const float2 q = s[sidx<PS>(k)];
        const float2 m = s[sidx<PS>(k == 0 ? 0 : L - k)];
        Do[(size_t)k << 2] = make_float2(0.5f * (q.x + m.x), 0.5f * (q.y - m.y));
        Eo[(size_t)k << 2] = make_float2(0.25f * (q.y + m.y), -0.25f * (q.x - m.x));
    }
}

template <int N>
__global__ void __launch_bounds__(Cfg2<N>::NT, Cfg2<N>::MC2) k_cols_step2(Pointers p0, int first, int hist_slot)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NT, R1 = C::R1, R2 = C::R2, R3 = C::R3, PS = C::PS;
    constexpr int LR1 = L / R1, LR3 = L / R3;
    extern __shared__ float2 smem[];
    __shared__ double2 red[32];
    __shared__ bool am_last;
    const int kx = blockIdx.x;
    const int j = threadIdx.x;
    float2 *sD = smem, *sE = smem + LP;
    float2 *om2c = p.om2 + (size_t)kx * N;
    float2 *fnc = p.fnm1 + (size_t)kx * N;
    // the state column is only needed after the forward transforms: start bringing it to L2
    for (int o = j * 32; o < N; o += NT * 32) {
        asm volatile("prefetch.global.L2 [%0];" ::"l"(om2c + o));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(fnc + o));
    }
    // forward transforms of D and E along z, plan (R3, R2, R1): the twiddle-free radix-R3 first
    // stage reads straight from global memory
#pragma unroll 1
    for (int a = 0; a < 2; ++a) {
        float2 *s = a ? sE : sD;
        if (j < LR3) {
            // element j + r L/R3 of the column; L/R3 is a multiple of 4, so consecutive r are a
            // fixed stride apart (one live address instead of R3)
            static_assert(LR3 % 4 == 0, "stride");
            constexpr size_t RS = (size_t)(LR3 / 4) * H * 4;
            const float2 *ptr = p.work + widx<L, H>(a, j, kx);
            float2 v[R3];
#pragma unroll
            for (int r = 0; r < R3; ++r, ptr += RS) v[r] = *ptr;
            DFT<R3, false>::run(v);
            sm_store<L, R3, 1, PS>(s, v, j);
        }
        stage1<TwCat<N>, L, R2, R3, false, PS>(s, p.tw);
        stage1<TwCat<N>, L, R1, R3 * R2, false, PS>(s, p.tw);
    }
    __syncthreads();

    const StepParams prm = *p.prm;
    const float dt = prm.dt;
    const float cnm1 = first ? prm.cnm1_first : prm.cn;
    const double hvdt = 0.5 * (double)prm.visc * (double)dt;
    const double c2n = 0.5 * (double)dt * (2.0 + (double)cnm1);
    const double c3n = -0.5 * (double)dt * (double)cnm1;
    const float divxz = (float)(1.0 / ((double)L * (double)L));
    double2 ez = make_double2(0.0, 0.0);
    const double wgt = (kx == 0) ? 0.5 : 1.0;
    for (int iz = j; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        const float2 d = sD[sidx<PS>(kzi)];
        const float2 e = sE[sidx<PS>(kzi)];
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
        sD[sidx<PS>(kzi)] = u;
        sE[sidx<PS>(kzi)] = w;
        const double pw = (double)on.x * on.x + (double)on.y * on.y;
        ez.x += wgt * pw * invK2;
        ez.y += wgt * pw;
    }
    for (int z = H + j; z < L - H; z += NT) {
        sD[sidx<PS>(z)] = make_float2(0.f, 0.f);
        sE[sidx<PS>(z)] = make_float2(0.f, 0.f);
    }
    ez = block_sum2<NT>(ez, red);
    if (threadIdx.x == 0) {
        p.part[kx] = ez;
        __threadfence();
        const unsigned int n = atomicAdd(p.counter, 1u);
        am_last = (n == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
        double2 acc = make_double2(0.0, 0.0);
        for (int i = threadIdx.x; i < H; i += NT) {
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
    // inverse transforms along z, plan (R3, R2, R1), the last stage straight to global memory
#pragma unroll 1
    for (int a = 0; a < 2; ++a) {
        float2 *s = a ? sE : sD;
        stage1<TwCat<N>, L, R3, 1, true, PS>(s, p.tw);
        stage1<TwCat<N>, L, R2, R3, true, PS>(s, p.tw);
        __syncthreads();
        if (j < LR1) {
            float2 v[R1];
            sm_load<L, R1, PS>(v, s, j);
            bfly<TwCat<N>, L, R1, LR1, true>(v, j, p.tw);
            static_assert(LR1 % 4 == 0, "stride");
            constexpr size_t QS = (size_t)(LR1 / 4) * H * 4;
            float2 *ptr = p.work + widx<L, H>(a, j, kx);
#pragma unroll
            for (int q = 0; q < R1; ++q, ptr += QS) *ptr = v[q];
        }
    }
}

// ------------------------------------------------------------------------------------------
// Column pass with one CTA of two thread groups per column: group 0 transforms D (then U),
// group 1 E (then W), each group synchronising on its own named barrier; the spectral update
// uses the whole CTA.  Same arithmetic as k_cols_step2.  One 768-thread CTA per SM holds half
// the shared memory of two 384-thread CTAs with the same number of warps, which leaves L1 room
// for the twiddle tables (N = 4096 on B200: 0.680 -> 0.655 ms per step; no register spills at
// 80 registers, where the single-group kernel spilled 272 bytes).  The columns arrive by
// cp.async (no registers held by loads in flight) and the state column is prefetched to L2.
// ------------------------------------------------------------------------------------------
template <int NTH>
__device__ __forceinline__ void group_sync(int id)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(NTH) : "memory");
}

template <class Cat, int L, int R, int NS, bool INV, int NTH, int PS = 5>
__device__ __forceinline__ void stage1g(float2 *s, const float2 *tw, int j, int bar)
{
    constexpr int LR = L / R;
    float2 v[R];
    group_sync<NTH>(bar);
    if (j < LR) {
        sm_load<L, R, PS>(v, s, j);
        bfly<Cat, L, R, NS, INV>(v, j, tw);
    }
    group_sync<NTH>(bar);
    if (j < LR) sm_store<L, R, NS, PS>(s, v, j);
}

// group stage variants with a compile-time band [B0, B1]: a first stage (Ns = 1) whose inputs in
// the band are zero, and a last stage (Ns = L/R) whose outputs in the band are never read
template <class Cat, int L, int R, bool INV, int NTH, int B0, int B1, int PS = 5>
__device__ __forceinline__ void stage1g_first_band(float2 *s, const float2 *tw, int j, int bar)
{
    constexpr int LR = L / R;
    float2 v[R];
    group_sync<NTH>(bar);
    if (j < LR) {
#pragma unroll
        for (int r = 0; r < R; ++r)
            v[r] = slot_in_band<L, R, B0, B1>(r) ? make_float2(0.f, 0.f) : s[sidx<PS>(j + r * LR)];
        DFT<R, INV>::run(v);
    }
    group_sync<NTH>(bar);
    if (j < LR) sm_store<L, R, 1, PS>(s, v, j);
}

template <class Cat, int L, int R, bool INV, int NTH, int B0, int B1, int PS = 5>
__device__ __forceinline__ void stage1g_last_band(float2 *s, const float2 *tw, int j, int bar)
{
    constexpr int LR = L / R;
    float2 v[R];
    group_sync<NTH>(bar);
    if (j < LR) {
        sm_load<L, R, PS>(v, s, j);
        bfly<Cat, L, R, LR, INV>(v, j, tw);
    }
    group_sync<NTH>(bar);
    if (j < LR) {
#pragma unroll
        for (int q = 0; q < R; ++q)
            if (!slot_in_band<L, R, B0, B1>(q)) s[sidx<PS>(j + q * LR)] = v[q];
    }
}

// Where one column CTA holds an SM (MC4 = 1), the column's om2 / fnm1 are brought into shared
// memory by cp.async at the start of the column pass, behind the D, E columns, so the spectral
// update reads them with no global-load latency left (N = 4096 on B200: column pass 0.299 ->
// 0.294 ms).  With two CTAs per SM the 2 x 16 N bytes more shrink L1 below the twiddle tables
// (N = 2048: 0.075 -> 0.076 ms), so there the state is read from global memory, prefetched to L2.
template <int N>
constexpr bool cols4_stage_state()
{
    return Cfg2<N>::MC4 == 1;
}

// dynamic shared memory of k_cols_step4: the D / E (then U / W) arrays and the staged state
template <int N>
constexpr size_t cols4_smem_bytes()
{
    return (2 * (size_t)Cfg2<N>::LP + (cols4_stage_state<N>() ? 2 * (size_t)N : 0)) * sizeof(float2);
}

template <int N>
__global__ void __launch_bounds__(2 * Cfg2<N>::NT, Cfg2<N>::MC4) k_cols_step4(Pointers p0, int first, int hist_slot)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NT, NT2 = 2 * C::NT, PS = C::PS;
    constexpr int R1 = C::R1, R2 = C::R2, R3 = C::R3, LR1 = L / R1;
    static_assert(NT % 32 == 0, "groups must be whole warps");
    extern __shared__ float2 smem[];
    __shared__ double2 red[32];
    __shared__ bool am_last;
    const int kx = blockIdx.x;
    const int g = (int)threadIdx.x / NT;  // 0: D / U, 1: E / W
    const int j = (int)threadIdx.x - g * NT;
    const int bar = 1 + g;
    float2 *sD = smem, *sE = smem + LP;
    float2 *sg = smem + g * LP;
    float2 *om2c = p.om2 + (size_t)kx * N;
    float2 *fnc = p.fnm1 + (size_t)kx * N;
    for (int z = j; z < L; z += NT) cp_async8(sg + sidx<PS>(z), p.work + widx<L, H>(g, z, kx));
    cp_async_commit();
    constexpr bool STAGE = cols4_stage_state<N>();
    float2 *so = smem + 2 * LP, *sf = so + N;  // the staged state column, dense (read at consecutive iz)
    if constexpr (STAGE) {
        for (int i = (int)threadIdx.x; i < N; i += NT2) {
            cp_async8(so + i, om2c + i);
            cp_async8(sf + i, fnc + i);
        }
        cp_async_commit();
    } else {
        for (int o = (int)threadIdx.x * 16; o < N; o += NT2 * 16) {
            prefetch_l2(om2c + o);
            prefetch_l2(fnc + o);
        }
    }
    if (p.pf_cols > 0 && kx + p.pf_cols < (int)gridDim.x) {  // the column pf_cols CTAs later
        const int kp = kx + p.pf_cols;
        for (int q = (int)threadIdx.x; q < 2 * (L / 4); q += NT2) {
            const int a = q / (L / 4), gg = q - a * (L / 4);
            prefetch_l2(p.work + (size_t)a * L * H + (((size_t)gg * H + kp) << 2));
        }
    }
    cp_async_wait<STAGE ? 1 : 0>();  // this thread's D / E copies have landed
    stage1g<TwCat<N>, L, R3, 1, false, NT, PS>(sg, p.tw, j, bar);
    stage1g<TwCat<N>, L, R2, R3, false, NT, PS>(sg, p.tw, j, bar);
    // the update reads kz_i < H and kz_i >= L - H only: the 3/2 band [H, L-H-1] is not stored
    stage1g_last_band<TwCat<N>, L, R1, false, NT, H, L - H - 1, PS>(sg, p.tw, j, bar);
    cp_async_wait<0>();  // and the state copies
    __syncthreads();

    const StepParams prm = *p.prm;
    const float dt = prm.dt;
    const float cnm1 = first ? prm.cnm1_first : prm.cn;
    const double hvdt = 0.5 * (double)prm.visc * (double)dt;
    const double c2n = 0.5 * (double)dt * (2.0 + (double)cnm1);
    const double c3n = -0.5 * (double)dt * (double)cnm1;
    const float divxz = (float)(1.0 / ((double)L * (double)L));
    double2 ez = make_double2(0.0, 0.0);
    const double wgt = (kx == 0) ? 0.5 : 1.0;
    for (int iz = (int)threadIdx.x; iz < N; iz += NT2) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        const float2 d = sD[sidx<PS>(kzi)];
        const float2 e = sE[sidx<PS>(kzi)];
        float2 fn = make_float2(0.f, 0.f);
        if (kz != -H) {
            const float ga = (float)kz * (float)kx;
            const float g2a2 = (float)kz * (float)kz - (float)kx * (float)kx;
            fn.x = (ga * d.x + g2a2 * e.x) * divxz;
            fn.y = (ga * d.y + g2a2 * e.y) * divxz;
            if (p.force) fn = add_forcing(fn, p, kx, iz, N);
        }
        const double K2 = (double)kx * kx + (double)kz * kz;
        const float2 on = STAGE ? cn_update(so[iz], fn, sf[iz], K2, hvdt, c2n, c3n)
                                : cn_update(om2c[iz], fn, fnc[iz], K2, hvdt, c2n, c3n);
        om2c[iz] = on;
        fnc[iz] = fn;
        float2 u, w;
        double invK2;
        recover_velocity(kx, kz, on, u, w, invK2);
        sD[sidx<PS>(kzi)] = u;
        sE[sidx<PS>(kzi)] = w;
        const double pw = (double)on.x * on.x + (double)on.y * on.y;
        ez.x += wgt * pw * invK2;
        ez.y += wgt * pw;
    }
    ez = block_sum2<NT2>(ez, red);
    if (threadIdx.x == 0) {
        p.part[kx] = ez;
        __threadfence();
        const unsigned int n = atomicAdd(p.counter, 1u);
        am_last = (n == gridDim.x - 1);
    }
    __syncthreads();
    if (am_last) {
        double2 acc = make_double2(0.0, 0.0);
        for (int i = (int)threadIdx.x; i < H; i += NT2) {
            const double2 q = __ldcg(&p.part[i]);
            acc.x += q.x;
            acc.y += q.y;
        }
        acc = block_sum2<NT2>(acc, red);
        if (threadIdx.x == 0) {
            p.hist[hist_slot] = acc;
            *p.counter = 0u;
        }
    }
    // 3/2 zero padding: the band [H, L-H-1] enters the first inverse stage as compile-time zeros
    // where whole radix-R3 slots lie in it; band positions in a slot that also holds retained
    // modes are read from shared memory, so they are cleared here (none when the slots tile the
    // band exactly, as with R3 = 12 or 24)
    for (int z = H + (int)threadIdx.x; z < L - H; z += NT2) {
        if (!slot_in_band<L, R3, H, L - H - 1>(z / (L / R3))) {
            sD[sidx<PS>(z)] = make_float2(0.f, 0.f);
            sE[sidx<PS>(z)] = make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    // inverse transform of this group's column, plan (R3, R2, R1), last stage straight to HBM
    stage1g_first_band<TwCat<N>, L, R3, true, NT, H, L - H - 1, PS>(sg, p.tw, j, bar);
    stage1g<TwCat<N>, L, R2, R3, true, NT, PS>(sg, p.tw, j, bar);
    group_sync<NT>(bar);
    if (j < LR1) {
        float2 v[R1];
        sm_load<L, R1, PS>(v, sg, j);
        bfly<TwCat<N>, L, R1, LR1, true>(v, j, p.tw);
        static_assert(LR1 % 4 == 0, "stride");
        constexpr size_t QS = (size_t)(LR1 / 4) * H * 4;
        float2 *ptr = p.work + widx<L, H>(g, j, kx);
#pragma unroll
        for (int q = 0; q < R1; ++q, ptr += QS) *ptr = v[q];
    }
}

// ------------------------------------------------------------------------------------------
// Diagnostics on the large-grid plans (the sizes with Cfg2): NEXTDT's CFL maximum and the
// physical velocity planes (as k_rows_velocity), and OM2PHYS / the stream function (as
// k_cols_scalar + k_rows_scalar), on the step kernels' transforms.
// ------------------------------------------------------------------------------------------
// one physical row: u, w into phys[0..1] (when phys != nullptr) and the CFL maximum
// max |u|/dx + |w|/dx (cuda/dns_cuda.cu:486-522) into cflm (when cflm != nullptr)
template <int N>
__global__ void __launch_bounds__(Cfg2<N>::NT, 3) k_rows_velocity2(Pointers p0, float *phys, float *cflm, float dx)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, R3 = C::R3, LR3 = L / R3, NT = C::NT;
    extern __shared__ float2 s[];
    __shared__ float red[32];
    const int z = blockIdx.x, j = threadIdx.x;
    float2 v[R3];
    rows_inverse2<N>(p.work + widx<L, H>(0, z, 0), p.work + widx<L, H>(1, z, 0), s, p.tw, v);
    float m = 0.0f;
    if (j < LR3) {
#pragma unroll
        for (int q = 0; q < R3; ++q) {
            if (phys) {
                const size_t o = (size_t)z * L + j + q * LR3;
                phys[o] = v[q].x;
                phys[(size_t)L * L + o] = v[q].y;
            }
            m = fmaxf(m, cfl_term(v[q].x, v[q].y, dx));
        }
    }
    if (cflm) {
        m = block_max<NT>(m, red);
        if (threadIdx.x == 0) atomic_max_nonneg(cflm + blockIdx.y, m);
    }
}

// one column: om2 (kind 0) or the stream function om2 / K^2 (kind 1; 0 at k = 0) -> inverse z
// transform -> scratch component 0 in the work layout
template <int N>
__global__ void __launch_bounds__(Cfg2<N>::NT) k_cols_scalar2(Pointers p, float2 *scratch, int kind)
{
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, NT = C::NT, R1 = C::R1, R2 = C::R2, R3 = C::R3, PS = C::PS, LR1 = L / R1;
    extern __shared__ float2 s[];
    const int kx = blockIdx.x, j = threadIdx.x;
    for (int iz = j; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        float2 v = p.om2[(size_t)kx * N + iz];
        if (kind == 1) {
            const float k2 = (float)kx * (float)kx + (float)kz * (float)kz + 1.0e-30f;
            v = make_float2(v.x / k2, v.y / k2);
            if (kx == 0 && iz == 0) v = make_float2(0.f, 0.f);
        }
        s[sidx<PS>(kzi)] = v;
    }
    for (int z = H + j; z < L - H; z += NT)
        if (!slot_in_band<L, R3, H, L - H - 1>(z / (L / R3))) s[sidx<PS>(z)] = make_float2(0.f, 0.f);
    stage1g_first_band<TwCat<N>, L, R3, true, NT, H, L - H - 1, PS>(s, p.tw, j, 1);
    stage1g<TwCat<N>, L, R2, R3, true, NT, PS>(s, p.tw, j, 1);
    group_sync<NT>(1);
    if (j < LR1) {
        float2 v[R1];
        sm_load<L, R1, PS>(v, s, j);
        bfly<TwCat<N>, L, R1, LR1, true>(v, j, p.tw);
        constexpr size_t QS = (size_t)(LR1 / 4) * H * 4;
        float2 *ptr = scratch + widx<L, H>(0, j, kx);
#pragma unroll
        for (int q = 0; q < R1; ++q, ptr += QS) *ptr = v[q];
    }
}

// two physical rows z = 2 blockIdx.x, z + 1 of a real field from its x half spectra (scratch
// component 0) -> out, with the CTA's min / max into minmax[blockIdx.x]
template <int N>
__global__ void __launch_bounds__(Cfg2<N>::NT, 3) k_rows_pair2(Pointers p, const float2 *scratch, float *out,
                                                             float2 *minmax)
{
    using C = Cfg2<N>;
    constexpr int L = C::L, H = C::H, R3 = C::R3, LR3 = L / R3, NT = C::NT;
    extern __shared__ float2 s[];
    __shared__ float red[32];
    const int z = 2 * blockIdx.x, j = threadIdx.x;
    float2 v[R3];
    rows_inverse2<N>(scratch + widx<L, H>(0, z, 0), scratch + widx<L, H>(0, z + 1, 0), s, p.tw, v);
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    if (j < LR3) {
#pragma unroll
        for (int q = 0; q < R3; ++q) {
            const size_t o = (size_t)z * L + j + q * LR3;
            out[o] = v[q].x;
            out[o + L] = v[q].y;
            mn = fminf(mn, fminf(v[q].x, v[q].y));
            mx = fmaxf(mx, fmaxf(v[q].x, v[q].y));
        }
    }
    __shared__ float s_nmn;
    const float nmn = block_max<NT>(-mn, red);
    if (threadIdx.x == 0) s_nmn = nmn;
    const float bmx = block_max<NT>(mx, red);
    if (threadIdx.x == 0) minmax[blockIdx.x] = make_float2(-s_nmn, bmx);
}

// ------------------------------------------------------------------------------------------
// Column set-up: velocity spectrum -> U, W columns.
// mode 0: from the compact velocity spectrum uw[iz][ix][2] (PAO); om2 = i (kz u - kx w)
//         (CALCOM, cuda/calcom_cuda.cu:117-131), fnm1 = 0.
// mode 1: from om2 (already in [kx][kz] layout): velocity recovery; om2/fnm1 left unchanged.
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTA) k_cols_init(Pointers p0, const float2 *__restrict__ uw,
                                                           int mode)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NTA;
    extern __shared__ float2 smem[];
    const int kx = blockIdx.x;
    float2 *sU = smem, *sW = smem + LP;
    for (int iz = threadIdx.x; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        float2 u, w;
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
        sU[sidx<PS>(kzi)] = u;
        sW[sidx<PS>(kzi)] = w;
    }
    for (int z = H + threadIdx.x; z < L - H; z += NT) {
        sU[sidx<PS>(z)] = make_float2(0.f, 0.f);
        sW[sidx<PS>(z)] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, 2, NT, PS>(smem, p.tw, typename C::Plan{});
    for (int z = threadIdx.x; z < L; z += NT) {
        p.work[widx<L, H>(0, z, kx)] = sU[sidx<PS>(z)];
        p.work[widx<L, H>(1, z, kx)] = sW[sidx<PS>(z)];
    }
}

// ------------------------------------------------------------------------------------------
// Velocity rows: U,W rows -> u,w physical (STEP2A's x-inverse).  Optionally writes u, w into
// phys[0], phys[1] ([L][L] float each) and/or reduces the CFL maximum (NEXTDT, DX = 2 pi / N).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_velocity(Pointers p0, float *phys, float *cflm,
                                                               float dx)
{
    const Pointers p = p0.member(blockIdx.y);
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, ROWS = C::ROWS, NT = C::NTB;
    extern __shared__ float2 smem[];
    __shared__ float red[32];
    const int z0 = blockIdx.x * ROWS;
    rows_load_pack<L, H, ROWS, NT, LP, PS>(smem, p.work, z0);
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, ROWS, NT, PS>(smem, p.tw, typename C::Plan{});
    float m = 0.0f;
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        const float2 z = smem[r * LP + sidx<PS>(x)];
        if (phys) {
            const size_t o = (size_t)(z0 + r) * L + x;
            phys[o] = z.x;
            phys[(size_t)L * L + o] = z.y;
        }
        m = fmaxf(m, cfl_term(z.x, z.y, dx));
    }
    if (cflm) {
        m = block_max<NT>(m, red);
        if (threadIdx.x == 0) atomic_max_nonneg(cflm + blockIdx.y, m);
    }
}

// ------------------------------------------------------------------------------------------
// Physical rows -> U,W rows (x-forward of u, w scaled by 1/L): loading a restart file's UR.
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_from_phys(Pointers p, const float *phys)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, ROWS = C::ROWS, NT = C::NTB;
    extern __shared__ float2 smem[];
    const int z0 = blockIdx.x * ROWS;
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        const size_t o = (size_t)(z0 + r) * L + x;
        smem[r * LP + sidx<PS>(x)] = make_float2(phys[o], phys[(size_t)L * L + o]);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, ROWS, NT, PS>(smem, p.tw, typename C::Plan{});
    const float sc = 1.0f / (float)L;
    for (int e = threadIdx.x; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 *x = smem + r * LP;
        const float2 q = x[sidx<PS>(k)];
        const float2 m = x[sidx<PS>(k == 0 ? 0 : L - k)];
        p.work[widx<L, H>(0, z0 + r, k)] = make_float2(0.5f * sc * (q.x + m.x), 0.5f * sc * (q.y - m.y));
        p.work[widx<L, H>(1, z0 + r, k)] = make_float2(0.5f * sc * (q.y + m.y), -0.5f * sc * (q.x - m.x));
    }
}

// ------------------------------------------------------------------------------------------
// Scalar field to physical space (OM2PHYS, stream function): one compact spectrum column ->
// z-inverse -> scratch (component 0 of a work-shaped buffer).  kind 0: om2; kind 1: om2/K^2
// with the (0,0) mode zeroed (cuda/om2phys_cuda.cu:232-256).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTA) k_cols_scalar(Pointers p, float2 *scratch, int kind)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NTA;
    extern __shared__ float2 smem[];
    const int kx = blockIdx.x;
    for (int iz = threadIdx.x; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        float2 v = p.om2[(size_t)kx * N + iz];
        if (kind == 1) {
            const float k2 = (float)kx * (float)kx + (float)kz * (float)kz + 1.0e-30f;
            v = make_float2(v.x / k2, v.y / k2);
            if (kx == 0 && iz == 0) v = make_float2(0.f, 0.f);
        }
        smem[sidx<PS>(kzi)] = v;
    }
    for (int z = H + threadIdx.x; z < L - H; z += NT) smem[sidx<PS>(z)] = make_float2(0.f, 0.f);
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, 1, NT, PS>(smem, p.tw, typename C::Plan{});
    for (int z = threadIdx.x; z < L; z += NT) scratch[widx<L, H>(0, z, kx)] = smem[sidx<PS>(z)];
}

// scratch rows -> real field rows written to out ([L][L]); per-block min/max partials
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_scalar(Pointers p, const float2 *scratch, float *out,
                                                             float2 *minmax)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, ROWS = C::ROWS, NT = C::NTB;
    extern __shared__ float2 smem[];
    __shared__ float red[32];
    const int z0 = blockIdx.x * ROWS;
    for (int e = threadIdx.x; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 a = scratch[widx<L, H>(0, z0 + r, k)];
        float2 *x = smem + r * LP;
        if (k == 0) {
            x[sidx<PS>(0)] = make_float2(a.x, 0.f);
        } else {
            x[sidx<PS>(k)] = a;
            x[sidx<PS>(L - k)] = make_float2(a.x, -a.y);
        }
    }
    constexpr int NZ = L - 2 * H + 1;
    for (int e = threadIdx.x; e < ROWS * NZ; e += NT) {
        const int r = e / NZ, k = H + (e - r * NZ);
        smem[r * LP + sidx<PS>(k)] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, ROWS, NT, PS>(smem, p.tw, typename C::Plan{});
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        const float v = smem[r * LP + sidx<PS>(x)].x;
        out[(size_t)(z0 + r) * L + x] = v;
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
    // block min/max (max of -min)
    __shared__ float s_nmn;
    const float nmn = block_max<NT>(-mn, red);
    if (threadIdx.x == 0) s_nmn = nmn;
    const float bmx = block_max<NT>(mx, red);
    if (threadIdx.x == 0) minmax[blockIdx.x] = make_float2(-s_nmn, bmx);
}


// ------------------------------------------------------------------------------------------
// Closure support: a real field on the L x L grid -> its retained spectrum F(kx,kz) in the
// compact [kx][kz] layout, normalised like FN: F = (1/L^2) sum_x f(x) e^{-i k.x}.
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_fwd_scalar(Pointers p, const float *f, float2 *scratch)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, ROWS = C::ROWS, NT = C::NTB;
    extern __shared__ float2 smem[];
    const int z0 = blockIdx.x * ROWS;
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        smem[r * LP + sidx<PS>(x)] = make_float2(f[(size_t)(z0 + r) * L + x], 0.f);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, ROWS, NT, PS>(smem, p.tw, typename C::Plan{});
    const float sc = 1.0f / (float)L;
    for (int e = threadIdx.x; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 q = smem[r * LP + sidx<PS>(k)];
        scratch[widx<L, H>(0, z0 + r, k)] = make_float2(q.x * sc, q.y * sc);
    }
}

// Energy gate of the closure, folded into the forcing's column transform (GateArgs.om2 set): the
// forcing F changes the energy at the rate P = sum w Re(conj(om / K^2) F); the resolved energy of
// an unforced step can only fall (dE/dt = -2 nu Z, Z = sum 0.5 w |om|^2; w = 1 at kx = 0, else 2;
// the mean mode left out), so the closure is kept for this step only when P <= 2 nu Z.  scale 0:
// otherwise the step runs as the plain coarse step (gate 0); scale 1: the forcing is scaled by
// 2 nu Z / P so that its input equals the loss.  Each column adds its modes in FP64, the partials
// (one per column) are summed by a fixed tree in the last column CTA to arrive, which decides.
__host__ __device__ constexpr int pow2_ceil(int n)
{
    int p = 1;
    while (p < n) p *= 2;
    return p;
}

struct GateArgs {
    const float2 *om2 = nullptr;       // the state's vorticity modes [kx][kz]; nullptr: no gate
    float visc = 0.0f;
    int scale = 0;
    float *gate = nullptr;              // the factor the step applies to the forcing
    unsigned long long *off = nullptr;  // steps whose forcing was dropped or scaled
    double2 *part = nullptr;            // (P, Z) per column, [H]
    unsigned int *counter = nullptr;    // arrival counter, reset by the last CTA
};

template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTA) k_cols_fwd_scalar(Pointers p, const float2 *scratch, float2 *out,
                                                                  GateArgs g)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = C::NTA;
    extern __shared__ float2 smem[];
    __shared__ double sp[NT], sz[NT];
    __shared__ bool last;
    const int kx = blockIdx.x;
    for (int z = threadIdx.x; z < L; z += NT) smem[sidx<PS>(z)] = scratch[widx<L, H>(0, z, kx)];
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, 1, NT, PS>(smem, p.tw, typename C::Plan{});
    const float sc = 1.0f / (float)L;
    double P = 0.0, Z = 0.0;
    const double w = (kx == 0) ? 1.0 : 2.0;
    for (int iz = threadIdx.x; iz < N; iz += NT) {
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        const float2 v = smem[sidx<PS>(kzi)];
        const float2 f = (kz == -H) ? make_float2(0.f, 0.f) : make_float2(v.x * sc, v.y * sc);
        out[(size_t)kx * N + iz] = f;
        if (g.om2) {
            const double k2 = (double)kx * kx + (double)kz * kz;
            if (k2 != 0.0) {
                const float2 o = g.om2[(size_t)kx * N + iz];
                P += w * ((double)o.x * f.x + (double)o.y * f.y) / k2;
                Z += 0.5 * w * ((double)o.x * o.x + (double)o.y * o.y);
            }
        }
    }
    if (!g.om2) return;
    // block sums by a fixed tree (NT need not be a power of two), then the column's partial
    constexpr int P2 = pow2_ceil(NT);
    sp[threadIdx.x] = P;
    sz[threadIdx.x] = Z;
    __syncthreads();
    for (int o = P2 / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o && (int)threadIdx.x + o < NT) {
            sp[threadIdx.x] += sp[threadIdx.x + o];
            sz[threadIdx.x] += sz[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        g.part[kx] = make_double2(sp[0], sz[0]);
        __threadfence();
        last = (atomicAdd(g.counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    // the last CTA: each thread adds the partials of columns threadIdx.x, + NT, ..., then the tree
    double2 q = make_double2(0.0, 0.0);
    for (int c = threadIdx.x; c < (int)gridDim.x; c += NT) {
        const double2 r = __ldcg(&g.part[c]);
        q.x += r.x;
        q.y += r.y;
    }
    sp[threadIdx.x] = q.x;
    sz[threadIdx.x] = q.y;
    __syncthreads();
    for (int o = P2 / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o && (int)threadIdx.x + o < NT) {
            sp[threadIdx.x] += sp[threadIdx.x + o];
            sz[threadIdx.x] += sz[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double Ps = sp[0], Zs = sz[0];
        *g.counter = 0u;
        const double loss = 2.0 * (double)g.visc * Zs;
        const bool keep = Ps <= loss;  // P > loss >= 0 below: the ratio is in [0, 1)
        *g.gate = keep ? 1.0f : (g.scale ? (float)(loss / Ps) : 0.0f);
        if (!keep) *g.off += 1ULL;
    }
}

// ------------------------------------------------------------------------------------------
// Dump path: the unnormalised forward 2D R2C of the physical velocity planes u, w, every mode
// kx in [0, L/2], kz in [0, L) -- the transform the reference's energy_spectrum.csv is binned
// from (cuda/mem_cuda.cu:579-581).  Output spec[c][z][kx] complex64, pitch L/2 + 1.
// Rows: u + i w through one complex FFT per row, U = (Q[k] + conj Q[L-k]) / 2,
// W = (Q[k] - conj Q[L-k]) / 2i; columns: one forward C2C per (kx, component).
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTB) k_rows_r2c_full(Pointers p, const float *phys, float2 *spec)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, LP = C::LP, ROWS = C::ROWS, NT = C::NTB, NK = L / 2 + 1;
    extern __shared__ float2 smem[];
    const int z0 = blockIdx.x * ROWS;
    const float *u = phys, *w = phys + (size_t)L * L;
    for (int e = threadIdx.x; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        const size_t i = (size_t)(z0 + r) * L + x;
        smem[r * LP + sidx<PS>(x)] = make_float2(u[i], w[i]);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, ROWS, NT, PS>(smem, p.tw, typename C::Plan{});
    for (int e = threadIdx.x; e < ROWS * NK; e += NT) {
        const int r = e / NK, k = e - r * NK;
        const float2 q = smem[r * LP + sidx<PS>(k)];
        const float2 m = smem[r * LP + sidx<PS>(k == 0 ? 0 : L - k)];
        const size_t o = (size_t)(z0 + r) * NK + k;
        spec[o] = make_float2(0.5f * (q.x + m.x), 0.5f * (q.y - m.y));
        spec[(size_t)L * NK + o] = make_float2(0.5f * (q.y + m.y), -0.5f * (q.x - m.x));
    }
}

template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTA) k_cols_c2c_full(Pointers p, float2 *spec)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    constexpr int L = C::L, LP = C::LP, NT = C::NTA, NK = L / 2 + 1;
    extern __shared__ float2 smem[];
    float2 *col = spec + (size_t)blockIdx.y * L * NK + blockIdx.x;
    for (int z = threadIdx.x; z < L; z += NT) smem[sidx<PS>(z)] = col[(size_t)z * NK];
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, 1, NT, PS>(smem, p.tw, typename C::Plan{});
    for (int z = threadIdx.x; z < L; z += NT) col[(size_t)z * NK] = smem[sidx<PS>(z)];
}

}  // namespace dns2d
