// ensemble.cu — the persistent ensemble launch (ensemble.cuh): device work items, the kernel
// and its cooperative, occupancy-sized launch.
#include "ensemble.cuh"

#include <algorithm>

namespace dns2d {
namespace {

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// wait until *c >= target: false when this wait ran out (recorded in *status) or another CTA's did
__device__ bool ens_wait(const unsigned int *c, unsigned int target, const EnsLaunch &q)
{
    long long n = 0;
    while (ld_acquire(c) < target) {
        if (*(volatile int *)q.status != 0) return false;
        if (++n > q.spin_limit) {
            atomicExch(q.status, 1);
            return false;
        }
        __nanosleep(256);
    }
    return true;
}

// rows z0 .. z0 + kEnsRows - 1 of one member: the row pass of k_rows_step (U, W rows -> C2R ->
// (u + iw)^2 -> R2C -> D, E rows), inputs loaded through L2
template <int N, class Plan>
__device__ __forceinline__ void ens_rows(const Pointers &p, int z0, float2 *smem)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    const int tid = opaque_tid();  // nothing of it hoisted out of the work loop
    constexpr int L = C::L, H = C::H, LP = C::LP, ROWS = kEnsRows, NT = kEnsThreads;
    for (int e = tid; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 a = __ldcg(p.work + widx<L, H>(0, z0 + r, k));
        const float2 b = __ldcg(p.work + widx<L, H>(1, z0 + r, k));
        float2 *x = smem + r * LP;
        if (k == 0) {
            x[sidx<PS>(0)] = make_float2(a.x, b.x);
        } else {
            x[sidx<PS>(k)] = make_float2(a.x - b.y, a.y + b.x);
            x[sidx<PS>(L - k)] = make_float2(a.x + b.y, b.x - a.y);
        }
    }
    constexpr int NZ = L - 2 * H + 1;  // zero band kx in [H, L-H]
    for (int e = tid; e < ROWS * NZ; e += NT) {
        const int r = e / NZ, k = H + (e - r * NZ);
        smem[r * LP + sidx<PS>(k)] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, ROWS, NT, PS, true>(smem, p.tw, Plan{});
    for (int e = tid; e < ROWS * L; e += NT) {
        const int r = e / L, x = e - r * L;
        float2 *a = smem + r * LP + sidx<PS>(x);
        const float2 z = *a;
        *a = make_float2(z.x * z.x - z.y * z.y, 2.0f * z.x * z.y);
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, ROWS, NT, PS, true>(smem, p.tw, Plan{});
    for (int e = tid; e < ROWS * H; e += NT) {
        const int r = e % ROWS, k = e / ROWS;
        const float2 *x = smem + r * LP;
        const float2 q = x[sidx<PS>(k)];
        const float2 m = x[sidx<PS>(k == 0 ? 0 : L - k)];
        p.work[widx<L, H>(0, z0 + r, k)] = make_float2(0.5f * (q.x + m.x), 0.5f * (q.y - m.y));
        p.work[widx<L, H>(1, z0 + r, k)] = make_float2(0.25f * (q.y + m.y), -0.25f * (q.x - m.x));
    }
}

// columns kx0 .. kx0 + CG - 1 of one member: the column pass of k_cols_step (D, E columns ->
// z-forward -> FN, Crank-Nicolson/AB2, FNM1 <- FN, velocity recovery -> 3/2 padding -> z-inverse
// -> U, W columns).  Shared-memory arrays 2c and 2c + 1 hold column c's D (then U) and E (then W).
// The item's FP64 energy/enstrophy partial goes to part[item]; the member's last item to finish
// sums the partials in item order (deterministic) into hist[slot].
template <int N, class Plan>
__device__ __forceinline__ void ens_cols(const Pointers &p, int item, int first, int slot, int nitems, float2 *smem,
                                         double2 *red, int *last)
{
    using C = Cfg<N>;
    constexpr int PS = C::PS;
    const int tid = opaque_tid();  // nothing of it hoisted out of the work loop
    constexpr int L = C::L, H = C::H, LP = C::LP, NT = kEnsThreads, CG = ens_cols_per_item<N>(), B = 2 * CG;
    const int kx0 = item * CG;
    // (z, kx0 + c) for c < CG and z%4 are CG * 4 consecutive float2 of a 4-row tile: read them so
    for (int e = tid; e < CG * L; e += NT) {
        const int z4 = e / (CG * 4), rem = e - z4 * (CG * 4), c = rem >> 2, z = 4 * z4 + (rem & 3);
        smem[(2 * c) * LP + sidx<PS>(z)] = __ldcg(p.work + widx<L, H>(0, z, kx0 + c));
        smem[(2 * c + 1) * LP + sidx<PS>(z)] = __ldcg(p.work + widx<L, H>(1, z, kx0 + c));
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, false, B, NT, PS, true>(smem, p.tw, Plan{});

    const StepParams prm = *p.prm;
    const float dt = prm.dt;
    const float cnm1 = first ? prm.cnm1_first : prm.cn;
    const double hvdt = 0.5 * (double)prm.visc * (double)dt;
    const double c2n = 0.5 * (double)dt * (2.0 + (double)cnm1);
    const double c3n = -0.5 * (double)dt * (double)cnm1;
    const float divxz = (float)(1.0 / ((double)L * (double)L));
    double2 ez = make_double2(0.0, 0.0);
    for (int e = tid; e < CG * N; e += NT) {
        const int c = e / N, iz = e - c * N, kx = kx0 + c;
        const int kz = (iz < H) ? iz : iz - N;
        const int kzi = (kz >= 0) ? kz : kz + L;
        float2 *sD = smem + (2 * c) * LP, *sE = smem + (2 * c + 1) * LP;
        const float2 d = sD[sidx<PS>(kzi)];
        const float2 ee = sE[sidx<PS>(kzi)];
        float2 fn = make_float2(0.f, 0.f);
        if (kz != -H) {  // STEP2B zeroes the kz = -N/2 row (cuda/step2b_cuda.cu:203-221)
            const float ga = (float)kz * (float)kx;
            const float g2a2 = (float)kz * (float)kz - (float)kx * (float)kx;
            fn.x = (ga * d.x + g2a2 * ee.x) * divxz;
            fn.y = (ga * d.y + g2a2 * ee.y) * divxz;
        }
        const double K2 = (double)kx * kx + (double)kz * kz;
        float2 *om2c = p.om2 + (size_t)kx * N;
        float2 *fnc = p.fnm1 + (size_t)kx * N;
        const float2 on = cn_update(__ldcg(om2c + iz), fn, __ldcg(fnc + iz), K2, hvdt, c2n, c3n);
        om2c[iz] = on;
        fnc[iz] = fn;
        float2 u, w;
        double invK2;
        recover_velocity(kx, kz, on, u, w, invK2);
        sD[sidx<PS>(kzi)] = u;
        sE[sidx<PS>(kzi)] = w;
        const double pw = (double)on.x * on.x + (double)on.y * on.y;
        const double wgt = (kx == 0) ? 0.5 : 1.0;  // 1/2 * (1 on kx = 0, else 2)
        ez.x += wgt * pw * invK2;
        ez.y += wgt * pw;
    }
    constexpr int NZ = L - 2 * H;  // 3/2 zero padding in kz
    for (int e = tid; e < CG * NZ; e += NT) {
        const int c = e / NZ, z = H + (e - c * NZ);
        smem[(2 * c) * LP + sidx<PS>(z)] = make_float2(0.f, 0.f);
        smem[(2 * c + 1) * LP + sidx<PS>(z)] = make_float2(0.f, 0.f);
    }
    ez = block_sum2<NT>(ez, red);
    if (tid == 0) {
        p.part[item] = ez;
        __threadfence();
        const unsigned int n = atomicAdd(p.counter, 1u);
        *last = (n == (unsigned int)nitems - 1u) ? 1 : 0;
    }
    __syncthreads();
    if (*last) {
        double2 acc = make_double2(0.0, 0.0);
        for (int i = tid; i < nitems; i += NT) {
            const double2 q = __ldcg(&p.part[i]);
            acc.x += q.x;
            acc.y += q.y;
        }
        acc = block_sum2<NT>(acc, red);
        if (tid == 0) {
            p.hist[slot] = acc;
            *p.counter = 0u;
        }
    }
    __syncthreads();
    fft_run<TwCat<N>, L, LP, true, B, NT, PS, true>(smem, p.tw, Plan{});
    for (int e = tid; e < CG * L; e += NT) {
        const int z4 = e / (CG * 4), rem = e - z4 * (CG * 4), c = rem >> 2, z = 4 * z4 + (rem & 3);
        p.work[widx<L, H>(0, z, kx0 + c)] = smem[(2 * c) * LP + sidx<PS>(z)];
        p.work[widx<L, H>(1, z, kx0 + c)] = smem[(2 * c + 1) * LP + sidx<PS>(z)];
    }
}

// a member's row / column item, on the size's default radix plan (Cfg<N>::Plan)
template <int N>
__device__ __forceinline__ void ens_row_item(const Pointers &p, int tile, float2 *smem)
{
    ens_rows<N, typename Cfg<N>::Plan>(p, tile * kEnsRows, smem);
}

template <int N>
__device__ __forceinline__ void ens_col_item(const Pointers &p, int item, int first, int slot, int nitems, float2 *smem,
                                             double2 *red, int *last)
{
    ens_cols<N, typename Cfg<N>::Plan>(p, item, first, slot, nitems, smem, red, last);
}

__global__ void __launch_bounds__(kEnsThreads, 2) k_ensemble(const __grid_constant__ EnsLaunch q)
{
    extern __shared__ float2 smem[];
    __shared__ double2 red[32];
    __shared__ int s_item, s_ok, s_last;
    const int per_step = q.rows_per_step + q.cols_per_step;
    const int total = per_step * q.steps;
    for (;;) {
        if (threadIdx.x == 0) {
            int it = (int)atomicAdd(q.ticket, 1u);
            if (it < total && *(volatile int *)q.status != 0) it = total;  // a wait ran out: stop
            s_item = it;
        }
        __syncthreads();
        const int item = s_item;
        if (item >= total) return;
        const int s = item / per_step;
        int r = item - s * per_step;
        const bool rows = r < q.rows_per_step;
        if (!rows) r -= q.rows_per_step;
        int gi = 0;
        for (int k = 1; k < q.ngroups; ++k)
            if ((rows ? q.g[k].row_begin : q.g[k].col_begin) <= r) gi = k;
        const EnsGroupDev &G = q.g[gi];
        const int per = rows ? G.row_items : G.col_items;
        const int rel = r - (rows ? G.row_begin : G.col_begin);
        const int m = rel / per, t = rel - m * per;
        const int gm = G.member0 + m;
        if (threadIdx.x == 0) {
            // rows of (m, s) after every column item of (m, s - 1); columns of (m, s) after every
            // row item of (m, s)
            const bool ok = rows ? ens_wait(q.cols_done + gm, (unsigned int)(s * G.col_items), q)
                                 : ens_wait(q.rows_done + gm,
                                            gm == q.stall_member ? 0xffffffffu : (unsigned int)((s + 1) * G.row_items), q);
            __threadfence();
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) return;
        const Pointers p = G.p.member(m);
        if (rows) {
            for (int u = 0; u < G.tiles_per_item; ++u) {
                const int tile = t * G.tiles_per_item + u;
                if (u > 0) __syncthreads();  // the previous tile's reads of shared memory are done
                switch (G.N) {
                case 64: ens_row_item<64>(p, tile, smem); break;
                case 128: ens_row_item<128>(p, tile, smem); break;
                case 256: ens_row_item<256>(p, tile, smem); break;
                default: ens_row_item<512>(p, tile, smem); break;
                }
            }
        } else {
            const int first = (q.first && s == 0) ? 1 : 0;
            const int ngroups = G.col_items * G.groups_per_item;  // column groups per member
            for (int u = 0; u < G.groups_per_item; ++u) {
                const int grp = t * G.groups_per_item + u;
                if (u > 0) __syncthreads();
                switch (G.N) {
                case 64: ens_col_item<64>(p, grp, first, s, ngroups, smem, red, &s_last); break;
                case 128: ens_col_item<128>(p, grp, first, s, ngroups, smem, red, &s_last); break;
                case 256: ens_col_item<256>(p, grp, first, s, ngroups, smem, red, &s_last); break;
                default: ens_col_item<512>(p, grp, first, s, ngroups, smem, red, &s_last); break;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd((rows ? q.rows_done : q.cols_done) + gm, 1u);
        }
    }
}

constexpr size_t kEnsSmem = std::max(std::max(ens_smem_bytes<64>(), ens_smem_bytes<128>()),
                                     std::max(ens_smem_bytes<256>(), ens_smem_bytes<512>()));

}  // namespace

// The grid is every CTA that fits on the GPU at once (occupancy x SMs), no more than there are
// items; a cooperative launch, which the driver refuses rather than run with CTAs that are not
// all resident, so no wait can depend on a CTA that never starts.
cudaError_t ens_launch(const EnsLaunch &q, cudaStream_t stream, int *grid_out)
{
    cudaError_t e = cudaFuncSetAttribute(k_ensemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEnsSmem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ensemble, kEnsThreads, kEnsSmem)) != cudaSuccess)
        return e;
    const long long items = (long long)(q.rows_per_step + q.cols_per_step) * q.steps;
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm, items));
    if (grid_out) *grid_out = grid;
    void *args[] = {const_cast<EnsLaunch *>(&q)};
    return cudaLaunchCooperativeKernel((void *)k_ensemble, grid, kEnsThreads, args, kEnsSmem, stream);
}

}  // namespace dns2d
