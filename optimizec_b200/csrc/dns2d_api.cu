// dns2d_api.cu — host side of the B200 2D vorticity solver: the C ABI of include/dns2d.h.
//
// The state owns its device buffers, one non-blocking CUDA stream and a cache of captured CUDA
// graphs (one per segment length).  The scalar bookkeeping (it, t, dt, cn, cnm1, cflm) is kept
// on the host in float and updated with the same expressions, in the same order, as the
// reference's host code (cuda/mem_cuda.cu:1848-1862, cuda/dns_cuda.cu:553-580,
// cuda/step3_cuda.cu:172), so printed T/DT/CN values follow the reference.  The device sees
// dt/cn/cnm1 through a small parameter block written by a one-thread kernel at the start of
// every dns2d_step call, which lets one captured graph serve every segment.
//
// Sections, in order: kernel configuration and tuning; small kernels and FP64 reductions; the
// state and its life cycle; initial conditions; time stepping; movie frames; diagnostics; state
// transfer; restart.bin through pinned staging; phase timing; batched ensembles; the closure
// network, the autotuner and the closure coupling; the time step without device allocation.
// The kernels of the passes are in dns2d_kernels.cuh / cluster.cuh, their launch tables in
// kernel_sets.cuh (instantiated by sets_*.cu).
#include "kernel_sets.cuh"
#include "ensemble.cuh"
#include "cnn.cuh"
#include "cnn_gemm.cuh"
#include "cnn_net.cuh"
#include "cnn_tc.cuh"
#include "../../include/dns2d.h"

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

using namespace dns2d;

// ============================================================================================
// kernel configuration and the table of compiled sizes (kernel_sets.cuh, sets_*.cu)
// ============================================================================================
namespace {

// kernel configuration of one size on one device; every variant computes the same arithmetic,
// so the choice changes speed only
struct Tuning {
    int rows_tile = 0, cols_groups = 0, pf_rows = 296, pf_cols = 74;
    int plan_rows = 0, plan_cols = 0;  // radix plans (these change the rounding)
};

std::mutex g_tune_mu;
std::map<std::pair<int, int>, Tuning> g_tune;  // (device, N) -> autotuned configuration
thread_local bool t_in_autotune = false;       // the autotuner's own scratch state is untuned

Tuning tuning_for(int device, int N)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({device, N});
    return it == g_tune.end() ? Tuning() : it->second;
}

void apply_tuning(Pointers &p, const Tuning &t)
{
    p.rows_tile = t.rows_tile;
    p.cols_groups = t.cols_groups;
    p.pf_rows = t.pf_rows;
    p.pf_cols = t.pf_cols;
    p.plan_rows = t.plan_rows;
    p.plan_cols = t.plan_cols;
}

// Small-grid tuning: rows per CTA x radix plan for the row pass, radix plan for the column pass.
// time(t, rows) returns the time of one pass under configuration t.  An alternative plan (which
// rounds differently) replaces plan 0 only when it is at least 3 % faster.
template <class F>
Tuning tune_small(int nplans, Tuning best, F time)
{
    float t0 = 1e30f, tb = 1e30f;
    Tuning b0 = best, bb = best;
    for (int pl = 0; pl < nplans; ++pl)
        for (int rt : {2, 4, 8}) {
            Tuning t = best;
            t.plan_rows = pl;
            t.rows_tile = rt;
            const float ms = time(t, true);
            if (pl == 0 && ms < t0) t0 = ms, b0.rows_tile = rt, b0.plan_rows = 0;
            if (ms < tb) tb = ms, bb.rows_tile = rt, bb.plan_rows = pl;
        }
    if (bb.plan_rows != 0 && tb > 0.97f * t0) bb = b0;
    best.rows_tile = bb.rows_tile;
    best.plan_rows = bb.plan_rows;
    t0 = tb = 1e30f;
    int pb = 0;
    for (int pl = 0; pl < nplans; ++pl) {
        Tuning t = best;
        t.plan_cols = pl;
        const float ms = time(t, false);
        if (pl == 0) t0 = ms;
        if (ms < tb) tb = ms, pb = pl;
    }
    best.plan_cols = (pb != 0 && tb > 0.97f * t0) ? 0 : pb;
    return best;
}

const KernelSet *kernel_set(int N)
{
    // one translation unit per group of sizes (sets_*.cu), compiled in parallel
    for (const KernelSet *(*part)(int) : {kernel_sets_small, kernel_sets_256, kernel_sets_mid, kernel_sets_4096,
                                          kernel_sets_cluster, kernel_sets_16384, kernel_sets_29400})
        if (const KernelSet *k = part(N)) return k;
    return nullptr;
}

// sizes served by the 4-CTA cluster kernels (one configuration each: not autotuned)
bool cluster_size(int N) { return N == 840 || N == 8192 || N == 9216 || N == 16384 || N == 29400; }

// ============================================================================================
// small non-templated kernels
// ============================================================================================
__global__ void k_set_params(StepParams *prm, float dt, float cnm1_first, float cn, float visc)
{
    prm->dt = dt;
    prm->cnm1_first = cnm1_first;
    prm->cn = cn;
    prm->visc = visc;
}

// |u| into phys[2] (cuda/om2phys_cuda.cu:331-355)
__global__ void k_kinetic(float *phys, size_t plane)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        const float u = phys[i], w = phys[plane + i];
        phys[2 * plane + i] = sqrtf(u * u + w * w);
    }
}

__global__ void k_minmax(const float *f, size_t n, float2 *out)
{
    __shared__ float smn[256], smx[256];
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = f[i];
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
    smn[threadIdx.x] = mn;
    smx[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            smn[threadIdx.x] = fminf(smn[threadIdx.x], smn[threadIdx.x + o]);
            smx[threadIdx.x] = fmaxf(smx[threadIdx.x], smx[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = make_float2(smn[0], smx[0]);
}

// 8-bit display quantisation sums (cuda/mem_cuda.cu:691-740): same IEEE operation sequence
__device__ __forceinline__ void sigma_pixel_sums(const float *f, size_t n, float minv, float rng, int is_constant,
                                                 unsigned long long *sums)
{
    __shared__ unsigned long long s1[256], s2[256];
    unsigned long long a = 0, b = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        int pix = 128;
        if (!is_constant) {
            const float norm = __fdiv_rn(__fsub_rn(f[i], minv), rng);
            float pf = __fadd_rn(1.0f, __fmul_rn(norm, 254.0f));
            if (pf < 1.0f) pf = 1.0f;
            if (pf > 255.0f) pf = 255.0f;
            pix = (int)pf;
        }
        a += (unsigned long long)pix;
        b += (unsigned long long)(pix * pix);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[2 * blockIdx.x] = s1[0];
        sums[2 * blockIdx.x + 1] = s2[0];
    }
}

__global__ void k_sigma_pixels(const float *f, size_t n, float minv, float rng, int is_constant,
                               unsigned long long *sums)
{
    sigma_pixel_sums(f, n, minv, rng, is_constant, sums);
}

// the same from min / max partials already on the device (every block reduces them itself, in
// float like the host: min / max are exact, so the result equals a separate min / max pass)
__global__ void k_sigma_pixels_mm(const float *f, size_t n, const float2 *mm, int nparts, unsigned long long *sums)
{
    __shared__ float smn[256], smx[256];
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        const float2 q = mm[i];
        mn = fminf(mn, q.x);
        mx = fmaxf(mx, q.y);
    }
    smn[threadIdx.x] = mn;
    smx[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            smn[threadIdx.x] = fminf(smn[threadIdx.x], smn[threadIdx.x + o]);
            smx[threadIdx.x] = fmaxf(smx[threadIdx.x], smx[threadIdx.x + o]);
        }
        __syncthreads();
    }
    const float minv = smn[0], maxv = smx[0];
    const float rng = __fsub_rn(maxv, minv);
    sigma_pixel_sums(f, n, minv, rng, fabsf(rng) <= 1.0e-12f ? 1 : 0, sums);
}

// FP64 reductions over the [kx][kz] vorticity: out[block] = {E, Z, pal, total_full, k00, kmax2}
__global__ void k_om2_reduce(const float2 *om2, int N, double *out)
{
    const int H = N / 2;
    __shared__ double sh[6][256];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    const size_t n = (size_t)N * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i / N), iz = (int)(i % N);
        const int kz = (iz < H) ? iz : iz - N;
        const float2 o = om2[i];
        const double p = (double)o.x * o.x + (double)o.y * o.y;
        const double k2 = (double)kx * kx + (double)kz * kz;
        const double w = (kx == 0) ? 1.0 : 2.0;
        acc[1] += 0.5 * w * p;
        if (k2 > 0) acc[0] += 0.5 * w * p / k2;
        // palinstrophy weights of cuda/mem_cuda.cu:912-916 (1 on x = 0 and x = N/2-1)
        const double wp = (kx == 0 || kx == H - 1) ? 1.0 : 2.0;
        acc[2] += wp * k2 * p;
        acc[3] += wp * p;
        if (kx == 0 && iz == 0) acc[4] += p;
        acc[5] = fmax(acc[5], k2);
    }
    for (int j = 0; j < 6; ++j) sh[j][threadIdx.x] = acc[j];
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            for (int j = 0; j < 5; ++j) sh[j][threadIdx.x] += sh[j][threadIdx.x + o];
            sh[5][threadIdx.x] = fmax(sh[5][threadIdx.x], sh[5][threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int j = 0; j < 6; ++j) out[6 * blockIdx.x + j] = sh[j][0];
}

__global__ void k_shell(const float2 *om2, int N, double *Ek, int nb)
{
    const int H = N / 2;
    const size_t n = (size_t)N * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i / N), iz = (int)(i % N);
        const int kz = (iz < H) ? iz : iz - N;
        const double k2 = (double)kx * kx + (double)kz * kz;
        if (k2 == 0.0) continue;
        const int sh = (int)(sqrt(k2) + 0.5);
        if (sh >= nb) continue;
        const float2 o = om2[i];
        const double w = (kx == 0) ? 1.0 : 2.0;
        atomicAdd(&Ek[sh], 0.5 * w * ((double)o.x * o.x + (double)o.y * o.y) / k2);
    }
}

// energy_spectrum.csv bins (cuda/mem_cuda.cu:593-629) over the full L x (L/2+1) grid.  The
// velocity is band limited, so F[u](kz,kx) = L^2 u_hat for retained modes and 0 elsewhere;
// every grid mode is still counted, as in the reference.
__global__ void k_vel_bins(const float2 *om2, int N, double *esum, int *cnt, int nbins)
{
    const int H = N / 2, L = 3 * N / 2, Nk = L / 2 + 1;
    const double r_max = sqrt(2.0), k_nyq = 0.5 * (double)L;
    const double L2 = (double)L * (double)L;
    const size_t n = (size_t)L * Nk;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(i / Nk), kx = (int)(i % Nk);
        const int kz = (z <= L / 2) ? z : z - L;
        if (kx == 0 && kz == 0) continue;
        const double r = sqrt((double)kx * kx + (double)kz * kz) / k_nyq;
        int bin = (int)floor((r / r_max) * nbins);
        if (bin < 0) bin = 0;
        if (bin >= nbins) bin = nbins - 1;
        const bool dbl = (kx > 0 && 2 * kx < L);
        atomicAdd(&cnt[bin], dbl ? 2 : 1);
        if (kx < H && kz >= -H && kz < H) {
            const int iz = (kz >= 0) ? kz : kz + N;
            const float2 o = om2[(size_t)kx * N + iz];
            const double K2 = (double)kx * kx + (double)kz * kz;
            const double ox = o.x, oy = o.y;
            double uu, ww;
            if (kx >= 1) {
                uu = (double)kz * kz * (ox * ox + oy * oy) / (K2 * K2);
                ww = (double)kx * kx * (ox * ox + oy * oy) / (K2 * K2);
            } else {
                uu = (kz != 0) ? (ox * ox + oy * oy) / ((double)kz * kz) : 0.0;
                ww = 0.0;
            }
            double p = (uu + ww) * L2 * L2;
            if (dbl) p *= 2.0;
            if (p != 0.0) atomicAdd(&esum[bin], p);
        }
    }
}

// [iz][ix] <-> [ix][iz] transposes of the compact spectra
__global__ void k_transpose_c64(const float2 *in, float2 *out, int rows, int cols)
{
    __shared__ float2 t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < rows && c < cols) t[j][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = t[threadIdx.x][j];
    }
}

}  // namespace

// ============================================================================================
// state
// ============================================================================================
struct dns2d_state {
    int N = 0, H = 0, L = 0, Nk = 0, device = 0;
    float Re = 0, K0 = 0, visc = 0, t = 0, dt = 0, cn = 1, cnm1 = 0, cflnum = 0, cflm = 0;
    int it = 0, ifn = 1;
    bool initialised = false;
    const KernelSet *ks = nullptr;
    cudaStream_t stream = nullptr;
    // device buffers
    float2 *om2 = nullptr, *fnm1 = nullptr, *work = nullptr, *tw = nullptr, *scratch = nullptr;
    float *phys = nullptr;
    // min/max partials of phys plane 2 in `minmax` left by OM2PHYS / the stream function (0: none
    // valid); display_sigma of plane 2 then needs no min/max pass of its own
    int mm_plane2 = 0;
    StepParams *prm = nullptr;
    double2 *part = nullptr, *hist = nullptr;
    unsigned int *counter = nullptr;
    float *cflm_dev = nullptr;
    float2 *minmax = nullptr;
    unsigned long long *sums = nullptr;
    double *red = nullptr;
    int hist_cap = 0;
    // pinned host
    double2 *hist_host = nullptr;
    unsigned char *stage = nullptr;  // restart file staging: kStageBufs buffers of stage_chunk bytes
    size_t stage_chunk = 0;
    cudaEvent_t stage_ev[3] = {nullptr, nullptr, nullptr};
    // graphs keyed by (first, K)
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    // phase timing
    bool timing = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double phase_ms[4] = {0, 0, 0, 0};
    long long phase_n[4] = {0, 0, 0, 0};
    // learned closure (dns2d_closure_attach)
    dns2d_cnn *cnn = nullptr;
    float in_scale[3] = {1, 1, 1}, out_scale = 1;
    int closure_check = 1;
    int closure_tc = 1;  // BF16 tensor-core CNN inference where the grid allows it
    float closure_clamp = 0.0f;  // forcing limited to this multiple of |FN| per mode (0: off)
    Tuning tune;         // kernel configuration (from the autotuner's table at creation)
    float2 *force = nullptr, *bk_om2 = nullptr, *bk_fnm1 = nullptr, *bk_work = nullptr;
    float *gate = nullptr;                  // device 0/1 per step (energy gate)
    double2 *gate_part = nullptr;           // per-column partials of the gate reduction, [H]
    unsigned int *gate_counter = nullptr;
    unsigned long long *gate_off = nullptr; // device count of gated-off steps
    std::map<int, cudaGraphExec_t> closure_graphs;
    float *closure_in = nullptr;
    long long closure_steps = 0, closure_fallbacks = 0;
    double closure_E = -1.0;
    std::string err;

    Pointers ptrs() const
    {
        Pointers p;
        p.om2 = om2;
        p.fnm1 = fnm1;
        p.work = work;
        p.tw = tw;
        p.prm = prm;
        p.part = part;
        p.counter = counter;
        p.hist = hist;
        p.force = nullptr;
        p.gate = nullptr;
        p.s_state = 0;
        p.s_work = 0;
        p.s_part = 0;
        p.s_hist = 0;
        apply_tuning(p, tune);
        return p;
    }
};

namespace {

constexpr int kHistCap = 4096;
constexpr int kSigmaBlocks = 1024;
constexpr int kRedBlocks = 512;
constexpr int kChunk = 128;  // steps per captured graph

int fail(dns2d_state *s, int code, const char *fmt, ...)
{
    if (s) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        s->err = buf;
    }
    return code;
}

int cuda_check(dns2d_state *s, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return DNS2D_OK;
    return fail(s, DNS2D_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define DNS2D_CUDA(call, what)                                      \
    do {                                                            \
        int rc_ = cuda_check(s, (call), what);                      \
        if (rc_ != DNS2D_OK) return rc_;                            \
    } while (0)

#define DNS2D_LAUNCHED(what) DNS2D_CUDA(cudaGetLastError(), what)

void free_graphs(dns2d_state *s)
{
    for (auto &kv : s->graphs) cudaGraphExecDestroy(kv.second);
    s->graphs.clear();
}

// per-stage twiddle tables of a catalog: entry off + (r-1) Ns + k = W_{Ns R}^{r k}, built in
// FP64 from the exactly reduced fraction (r k mod Ns R) / (Ns R) and rounded once
std::vector<float2> twiddles(const TwCatalog &c)
{
    std::vector<float2> t((size_t)std::max(c.total, 1));
    for (int i = 0; i < c.n; ++i) {
        const int R = c.R[i], NS = c.NS[i], M = R * NS;
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < NS; ++k) {
                const long long m = ((long long)r * k) % M;
                const double a = 2.0 * M_PI * (double)m / (double)M;
                t[(size_t)c.off[i] + (size_t)(r - 1) * NS + k] = make_float2((float)std::cos(a), (float)-std::sin(a));
            }
    }
    return t;
}

void phase_begin(dns2d_state *s)
{
    if (s->timing) cudaEventRecord(s->ev0, s->stream);
}

void phase_end(dns2d_state *s, int id)
{
    if (!s->timing) return;
    cudaEventRecord(s->ev1, s->stream);
    cudaEventSynchronize(s->ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    s->phase_ms[id] += ms;
    s->phase_n[id] += 1;
}

}  // namespace

// ============================================================================================
// life cycle
// ============================================================================================
extern "C" const char *dns2d_strerror(int code)
{
    switch (code) {
    case DNS2D_OK: return "ok";
    case DNS2D_ERR_ARG: return "invalid argument";
    case DNS2D_ERR_SIZE: return "unsupported grid size";
    case DNS2D_ERR_CUDA: return "CUDA error";
    case DNS2D_ERR_NOMEM: return "device allocation failed";
    case DNS2D_ERR_IO: return "file I/O error";
    case DNS2D_ERR_FORMAT: return "restart format mismatch";
    case DNS2D_ERR_STATE: return "call out of order";
    case DNS2D_ERR_TIMEOUT: return "device watchdog timeout";
    default: return "unknown error";
    }
}

extern "C" const char *dns2d_last_error(const dns2d_state *s) { return s ? s->err.c_str() : "null state"; }

extern "C" int dns2d_supported(int N) { return kernel_set(N) != nullptr ? 1 : 0; }

extern "C" size_t dns2d_device_bytes(int N)
{
    const size_t H = N / 2, L = 3 * (size_t)N / 2;
    return 2 * (size_t)N * H * 8      // om2, fnm1
           + 2 * L * H * 8            // work
           + L * H * 8                // scratch
           + 3 * L * L * 4            // phys
           + 2 * L * 8 + H * 16 + kHistCap * 16;
}

extern "C" int dns2d_create(dns2d_state **out, int N, float Re, float K0, float cflnum, int device)
{
    if (!out) return DNS2D_ERR_ARG;
    *out = nullptr;
    const KernelSet *ks = kernel_set(N);
    if (!ks) return DNS2D_ERR_SIZE;
    if (!t_in_autotune) {
        const char *env = std::getenv("DNS2D_AUTOTUNE");
        bool tuned;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            tuned = g_tune.count({device, N}) > 0;
        }
        if (env && env[0] == '1' && !tuned) {
            const int rc = dns2d_autotune(N, device, nullptr);
            if (rc) return rc;
        }
    }
    dns2d_state *s = new dns2d_state();
    s->N = N;
    s->H = N / 2;
    s->L = 3 * N / 2;
    s->Nk = 3 * N / 4 + 1;
    s->Re = Re;
    s->K0 = K0;
    s->visc = 0.0f;
    s->cflnum = cflnum;
    s->device = device;
    s->ks = ks;
    s->tune = tuning_for(device, N);
    auto bail = [&](int rc) {
        dns2d_destroy(s);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (ks->setup() != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    const size_t H = s->H, L = s->L;
    const size_t nom = (size_t)N * H;
    auto dalloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
    if (!dalloc((void **)&s->om2, nom * 8) || !dalloc((void **)&s->fnm1, nom * 8) ||
        !dalloc((void **)&s->work, 2 * L * H * 8) || !dalloc((void **)&s->scratch, L * H * 8) ||
        !dalloc((void **)&s->phys, 3 * L * L * 4) || !dalloc((void **)&s->tw, (size_t)std::max(ks->cat->total, 1) * 8) ||
        !dalloc((void **)&s->prm, sizeof(StepParams)) || !dalloc((void **)&s->part, H * 16) ||
        !dalloc((void **)&s->hist, (size_t)kHistCap * 16) || !dalloc((void **)&s->counter, 4) ||
        !dalloc((void **)&s->cflm_dev, 4) || !dalloc((void **)&s->minmax, (size_t)std::max(kSigmaBlocks, ks->rows_blocks) * 8) ||
        !dalloc((void **)&s->sums, (size_t)kSigmaBlocks * 16) || !dalloc((void **)&s->red, (size_t)kRedBlocks * 6 * 8)) {
        cudaGetLastError();
        return bail(DNS2D_ERR_NOMEM);
    }
    s->hist_cap = kHistCap;
    if (cudaMallocHost((void **)&s->hist_host, (size_t)kHistCap * 16) != cudaSuccess) return bail(DNS2D_ERR_NOMEM);
    std::vector<float2> tw = twiddles(*ks->cat);
    if (cudaMemcpy(s->tw, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaMemset(s->counter, 0, 4) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaMemset(s->om2, 0, nom * 8) != cudaSuccess || cudaMemset(s->fnm1, 0, nom * 8) != cudaSuccess ||
        cudaMemset(s->work, 0, 2 * L * H * 8) != cudaSuccess || cudaMemset(s->phys, 0, 3 * L * L * 4) != cudaSuccess)
        return bail(DNS2D_ERR_CUDA);
    if (cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    *out = s;
    return DNS2D_OK;
}

extern "C" void dns2d_destroy(dns2d_state *s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_graphs(s);
    cudaFree(s->om2);
    cudaFree(s->fnm1);
    cudaFree(s->work);
    cudaFree(s->scratch);
    cudaFree(s->phys);
    cudaFree(s->tw);
    cudaFree(s->prm);
    cudaFree(s->part);
    cudaFree(s->hist);
    cudaFree(s->counter);
    cudaFree(s->cflm_dev);
    cudaFree(s->minmax);
    cudaFree(s->sums);
    cudaFree(s->red);
    for (auto &kv : s->closure_graphs) cudaGraphExecDestroy(kv.second);
    cudaFree(s->gate);
    cudaFree(s->gate_off);
    cudaFree(s->gate_part);
    cudaFree(s->gate_counter);
    cudaFree(s->force);
    cudaFree(s->bk_om2);
    cudaFree(s->bk_fnm1);
    cudaFree(s->bk_work);
    cudaFree(s->closure_in);
    if (s->hist_host) cudaFreeHost(s->hist_host);
    if (s->stage) cudaFreeHost(s->stage);
    for (cudaEvent_t e : s->stage_ev)
        if (e) cudaEventDestroy(e);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// ============================================================================================
// initial conditions
// ============================================================================================
namespace {

void reset_scalars(dns2d_state *s)
{
    s->it = 0;
    s->t = 0.0f;
    s->dt = 0.0f;
    s->cn = 1.0f;
    s->cnm1 = 0.0f;
    s->ifn = 1;
}

// upload [iz][ix] c64 host arrays into the [kx][kz] device layout
int upload_compact(dns2d_state *s, const float *host, float2 *dst)
{
    const size_t n = (size_t)s->N * s->H;
    DNS2D_CUDA(cudaMemcpyAsync(s->scratch, host, n * 8, cudaMemcpyHostToDevice, s->stream), "upload");
    dim3 b(32, 8), g((s->H + 31) / 32, (s->N + 31) / 32);
    k_transpose_c64<<<g, b, 0, s->stream>>>(s->scratch, dst, s->N, s->H);
    DNS2D_LAUNCHED("transpose");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "upload sync");
    return DNS2D_OK;
}

int download_compact(dns2d_state *s, const float2 *src, float *host)
{
    const size_t n = (size_t)s->N * s->H;
    dim3 b(32, 8), g((s->N + 31) / 32, (s->H + 31) / 32);
    k_transpose_c64<<<g, b, 0, s->stream>>>(src, s->scratch, s->H, s->N);
    DNS2D_LAUNCHED("transpose");
    DNS2D_CUDA(cudaMemcpyAsync(host, s->scratch, n * 8, cudaMemcpyDeviceToHost, s->stream), "download");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "download sync");
    return DNS2D_OK;
}

// PAO-k^-3 host initial condition with the reference's float/double arithmetic
// (cuda/pao_km3_cuda.cu:59-424).  uw: [z][x][2] complex float.
void pao_host(int N, float K0, float Re, std::vector<std::complex<float>> &uw, double *stats, int *seed_out)
{
    const int NE = N, ND2 = N / 2, NED2 = NE / 2;
    const float PI = 3.14159265358979f;
    const float DXZ = 2.0f * PI / float(N);
    const float NORM = PI * K0 * K0;
    const float AMP2_FLOOR = 1.0e-40f;
    std::vector<float> alfa(ND2), gamma(NE);
    const float E1 = 1.0f, E3 = 1.0f / E1;
    for (int x = 0; x < NED2; ++x) alfa[x] = float(x) * (1.0f / E1);
    gamma[0] = 0.0f;
    for (int z = 1; z <= NED2; ++z) {
        gamma[z] = float(z) * (1.0f / E3);
        gamma[NE - z] = -gamma[z];
    }
    uw.assign((size_t)ND2 * NE * 2, std::complex<float>(0.0f, 0.0f));
    auto at = [&](int x, int z, int c) -> std::complex<float> & { return uw[(size_t)c + 2 * ((size_t)x + (size_t)ND2 * z)]; };

    // Fortran-style LCG and the 97-entry shuffle table
    int seed = 1;
    const int seed_init = 1;
    auto frand = [&]() {
        seed = (seed * 420029 + 2017) % 5011;
        return float(seed) / float(5011);
    };
    float ranvec[97];
    for (int i = 0; i < 97; ++i) frand();
    for (int i = 0; i < 97; ++i) ranvec[i] = frand();
    for (int z = 0; z < NE; ++z) {
        for (int x = 0; x < NED2; ++x) {
            const float r = frand();
            int idx = int(r * 97.0f);
            idx = std::min(96, std::max(0, idx));
            const float pick = ranvec[idx];
            ranvec[idx] = r;
            const float th = 2.0f * PI * pick;
            const std::complex<float> arg(std::cos(th), std::sin(th));
            const float ax = alfa[x], gz = gamma[z];
            const float K = std::sqrt(ax * ax + gz * gz);
            if (ax == 0.0f) {
                at(x, z, 1) = std::complex<float>(0.0f, 0.0f);
                float a2 = std::exp(-(K / K0) * (K / K0)) / NORM;
                if (a2 < AMP2_FLOOR) a2 = AMP2_FLOOR;
                at(x, z, 0) = std::sqrt(a2) * arg;
            } else {
                const float denom = 1.0f + (gz * gz) / (ax * ax);
                float a2 = std::exp(-(K / K0) * (K / K0)) / (denom * NORM);
                if (a2 < AMP2_FLOOR) a2 = AMP2_FLOOR;
                const std::complex<float> w = std::sqrt(a2) * arg;
                at(x, z, 1) = w;
                at(x, z, 0) = -(gz / ax) * w;
            }
        }
    }
    at(0, 0, 0) = at(0, 0, 1) = std::complex<float>(0.0f, 0.0f);
    for (int z = 1; z < NED2; ++z) {
        at(0, NE - z, 0) = std::conj(at(0, z, 0));
        at(0, NE - z, 1) = std::conj(at(0, z, 1));
    }
    for (int x = 0; x < ND2; ++x) at(x, NED2, 0) = at(x, NED2, 1) = std::complex<float>(0.0f, 0.0f);

    // shell re-weighting toward E(k) ~ k^-3 with hashed jitter and phases
    auto hash01 = [](int x, int z, int sd, int salt) {
        const double a = (double(x) + 1.0) * 12.9898 + (double(z) + 1.0) * 78.233 +
                         (double(sd) + 1.0) * 0.010001 + (double(salt) + 1.0) * 37.719;
        const double v = std::sin(a) * 43758.5453123;
        return v - std::floor(v);
    };
    const double knyq = double(ND2);
    const int kmax = ND2;
    std::vector<double> shell_e(kmax + 1, 0.0), shell_w(kmax + 1, 0.0), target(kmax + 1, 0.0);
    for (int x = 0; x < ND2; ++x) {
        const double m = (x == 0) ? 1.0 : 2.0;
        const double ax2 = double(alfa[x]) * double(alfa[x]);
        for (int z = 0; z < NE; ++z) {
            const double gz = double(gamma[z]);
            const double k = std::sqrt(ax2 + gz * gz);
            const int sh = int(k + 0.5);
            const std::complex<float> U1 = at(x, z, 0), U3 = at(x, z, 1);
            const double e1 = double(U1.real()) * double(U1.real()) + double(U1.imag()) * double(U1.imag());
            const double e3 = double(U3.real()) * double(U3.real()) + double(U3.imag()) * double(U3.imag());
            if (k > 0.0 && k <= knyq && sh <= kmax) {
                const int zh = (x == 0 && z > NED2) ? NE - z : z;
                shell_e[sh] += m * (e1 + e3);
                shell_w[sh] += m * (0.75 + 0.50 * hash01(x, zh, seed_init, 17));
            }
        }
    }
    const double k0 = std::max(1.0, double(K0));
    for (int sh = 1; sh <= kmax; ++sh) {
        const double k = double(sh);
        target[sh] = (k < k0) ? std::pow(k / k0, 4) / (k0 * k0 * k0) : 1.0 / (k * k * k);
        if (k < k0) {
            const double low = k / k0;
            target[sh] = (low * low * low * low) / (k0 * k0 * k0);
        }
    }
    double e_orig = 0.0, e_tgt = 0.0;
    for (int sh = 1; sh <= kmax; ++sh) {
        e_orig += shell_e[sh];
        e_tgt += target[sh];
    }
    if (e_orig > 0.0 && e_tgt > 0.0) {
        const double norm = e_orig / e_tgt;
        for (int x = 0; x < ND2; ++x) {
            const double ax = double(alfa[x]), ax2 = ax * ax;
            for (int z = 0; z < NE; ++z) {
                const double gz = double(gamma[z]), gz2 = gz * gz;
                const double k = std::sqrt(ax2 + gz2);
                const int sh = int(k + 0.5);
                if (k > 0.0 && k <= knyq && sh <= kmax && shell_w[sh] > 0.0) {
                    int zh = z;
                    double sgn = 1.0;
                    if (x == 0 && z > NED2) {
                        zh = NE - z;
                        sgn = -1.0;
                    }
                    const double jit = 0.75 + 0.50 * hash01(x, zh, seed_init, 17);
                    const double me = (norm * target[sh]) * jit / shell_w[sh];
                    const double th = sgn * 2.0 * 3.14159265358979323846 * hash01(x, zh, seed_init, 53);
                    const std::complex<float> ph(float(std::cos(th)), float(std::sin(th)));
                    if (ax == 0.0) {
                        at(x, z, 0) = float(std::sqrt(me)) * ph;
                        at(x, z, 1) = std::complex<float>(0.0f, 0.0f);
                    } else {
                        const std::complex<float> w = float(std::sqrt(me / (1.0 + gz2 / ax2))) * ph;
                        at(x, z, 0) = float(-gz / ax) * w;
                        at(x, z, 1) = w;
                    }
                } else {
                    at(x, z, 0) = at(x, z, 1) = std::complex<float>(0.0f, 0.0f);
                }
            }
        }
    }
    // statistics block (cuda/pao_km3_cuda.cu:345-424)
    double A[8] = {0, 0, 0, 0, 0, 0, 0, 0}, E110 = 0.0;
    for (int x = 0; x < ND2; ++x) {
        for (int z = 0; z < N; ++z) {
            const double e1 = std::norm(at(x, z, 0)), e3 = std::norm(at(x, z, 1));
            const double ax2 = double(alfa[x]) * double(alfa[x]);
            const double gz2 = double(gamma[z]) * double(gamma[z]);
            const double K2 = ax2 + gz2;
            const double m = (x == 0) ? 1.0 : 2.0;
            A[1] += m * e1;
            A[2] += m * e3;
            A[3] += m * e1 * ax2;
            A[4] += m * e1 * gz2;
            A[5] += m * e3 * ax2;
            A[6] += m * e3 * gz2;
            A[7] += m * (e1 + e3) * K2 * K2;
            if (x == 0) E110 += e1;
        }
    }
    const double Q2 = A[1] + A[2], W2 = A[3] + A[4] + A[5] + A[6];
    const double visc = 1.0 / Re;
    const double EP = visc * W2, De = 2.0 * visc * visc * A[7];
    const double KOL = std::pow(visc * visc * visc / EP, 0.25);
    if (stats) {
        const double v[19] = {double(Re), Q2, W2, EP, 2.0 * A[1] / Q2 - 1.0, 2.0 * (A[3] + A[4]) / W2 - 1.0,
                              0.5 * Q2 / EP, KOL, visc, DXZ / KOL, (E110 != 0.0) ? 2.0 * A[1] / E110 : 0.0,
                              2.0 * PI / std::sqrt(2.0 * A[1] / A[3]), 2.0 * PI / std::sqrt(2.0 * A[1] / A[4]),
                              2.0 * PI / std::sqrt(2.0 * A[2] / A[5]), 2.0 * PI / std::sqrt(2.0 * A[2] / A[6]),
                              De, 0.5 * Q2 * De / (EP * EP), double(E1), double(E3)};
        std::memcpy(stats, v, sizeof(v));
    }
    if (seed_out) *seed_out = seed;
}

}  // namespace

extern "C" int dns2d_init_pao(dns2d_state *s, double *stats19, int *pao_seed)
{
    if (!s) return DNS2D_ERR_ARG;
    std::vector<std::complex<float>> uw;
    pao_host(s->N, s->K0, s->Re, uw, stats19, pao_seed);
    s->visc = float(1.0 / s->Re);
    reset_scalars(s);
    const size_t bytes = uw.size() * sizeof(std::complex<float>);
    float2 *d_uw = nullptr;
    // the compact velocity spectrum (2 N^2/2 complex) is staged in the phys buffer
    if (bytes > 3 * (size_t)s->L * s->L * 4) return fail(s, DNS2D_ERR_NOMEM, "PAO staging");
    d_uw = reinterpret_cast<float2 *>(s->phys);
    s->mm_plane2 = 0;
    DNS2D_CUDA(cudaMemcpyAsync(d_uw, uw.data(), bytes, cudaMemcpyHostToDevice, s->stream), "PAO upload");
    s->ks->cols_init(s->ptrs(), d_uw, 0, s->stream, 1);
    DNS2D_LAUNCHED("cols_init(PAO)");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "PAO init");
    s->initialised = true;
    return DNS2D_OK;
}

extern "C" int dns2d_init_vorticity(dns2d_state *s, const float *om2, const float *fnm1)
{
    if (!s || !om2) return DNS2D_ERR_ARG;
    if (s->visc == 0.0f) s->visc = float(1.0 / s->Re);
    reset_scalars(s);
    int rc = upload_compact(s, om2, s->om2);
    if (rc) return rc;
    if (fnm1) {
        rc = upload_compact(s, fnm1, s->fnm1);
        if (rc) return rc;
    } else {
        DNS2D_CUDA(cudaMemsetAsync(s->fnm1, 0, (size_t)s->N * s->H * 8, s->stream), "fnm1 clear");
    }
    s->ks->cols_init(s->ptrs(), nullptr, 1, s->stream, 1);
    DNS2D_LAUNCHED("cols_init(om2)");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "vorticity init");
    s->initialised = true;
    return DNS2D_OK;
}

extern "C" int dns2d_k4_spectrum(int N, float K0, uint64_t seed, float *om2)
{
    if (!om2 || N < 8 || N % 8) return DNS2D_ERR_ARG;
    const int H = N / 2;
    std::vector<double> re((size_t)N * H), im((size_t)N * H);
    // splitmix64: the i-th draw (row-major over [iz][ix]) mixes the state seed + (i+1) * gamma, so
    // rows are generated independently (in parallel at large N) with the same values
    const double k0 = K0;
    auto rows = [&](int iz0, int iz1) {
        for (int iz = iz0; iz < iz1; ++iz)
            for (int ix = 0; ix < H; ++ix) {
                const size_t i = (size_t)iz * H + ix;
                uint64_t z = seed + (uint64_t)(i + 1) * 0x9E3779B97F4A7C15ULL;
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
                z ^= z >> 31;
                const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0);
                const double th = 2.0 * M_PI * u;
                const int kz = (iz < H) ? iz : iz - N;
                const double k2 = (double)ix * ix + (double)kz * kz;
                if (k2 == 0.0 || kz == -H) {
                    re[i] = im[i] = 0.0;
                    continue;
                }
                const double k = std::sqrt(k2), q = k / k0;
                const double a = std::sqrt(k * q * q * q * q * std::exp(-2.0 * q * q));
                re[i] = a * std::cos(th);
                im[i] = a * std::sin(th);
            }
    };
    const int nth = (N >= 2048) ? (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency())) : 1;
    if (nth == 1) {
        rows(0, N);
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nth; ++t) pool.emplace_back(rows, (int)((long long)N * t / nth), (int)((long long)N * (t + 1) / nth));
        for (auto &th : pool) th.join();
    }
    for (int iz = H + 1; iz < N; ++iz) {  // Hermitian kx = 0 column
        re[(size_t)iz * H] = re[(size_t)(N - iz) * H];
        im[(size_t)iz * H] = -im[(size_t)(N - iz) * H];
    }
    double E = 0.0;
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const int kz = (iz < H) ? iz : iz - N;
            const double k2 = (double)ix * ix + (double)kz * kz;
            if (k2 == 0.0) continue;
            const size_t i = (size_t)iz * H + ix;
            E += 0.5 * (ix == 0 ? 1.0 : 2.0) * (re[i] * re[i] + im[i] * im[i]) / k2;
        }
    const double sc = (E > 0.0) ? std::sqrt(0.5 / E) : 0.0;
    for (size_t i = 0; i < (size_t)N * H; ++i) {
        om2[2 * i] = (float)(re[i] * sc);
        om2[2 * i + 1] = (float)(im[i] * sc);
    }
    return DNS2D_OK;
}

extern "C" int dns2d_init_k4(dns2d_state *s, uint64_t seed)
{
    if (!s) return DNS2D_ERR_ARG;
    std::vector<float> om((size_t)s->N * s->H * 2);
    int rc = dns2d_k4_spectrum(s->N, s->K0, seed, om.data());
    if (rc) return rc;
    return dns2d_init_vorticity(s, om.data(), nullptr);
}

// ============================================================================================
// time stepping
// ============================================================================================
namespace {

int get_graph(dns2d_state *s, int first, int K, cudaGraphExec_t *out)
{
    auto key = std::make_pair(first, K);
    auto itg = s->graphs.find(key);
    if (itg != s->graphs.end()) {
        *out = itg->second;
        return DNS2D_OK;
    }
    cudaGraph_t g = nullptr;
    DNS2D_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    const Pointers p = s->ptrs();
    for (int i = 0; i < K; ++i) {
        s->ks->rows_step(p, s->stream, 1);
        s->ks->cols_step(p, (first && i == 0) ? 1 : 0, i, s->stream, 1);
    }
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) return cuda_check(s, e, "end capture");
    cudaGraphExec_t ex = nullptr;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_check(s, e, "graph instantiate");
    s->graphs[key] = ex;
    *out = ex;
    return DNS2D_OK;
}

}  // namespace

static int closure_run(dns2d_state *s, int nsteps, double *E_hist, double *Z_hist);

// Capture (and instantiate) the CUDA graphs that dns2d_step(s, nsteps) will launch, without
// running anything: a caller that times dns2d_step keeps the one-time graph set-up out of the
// timed region.  With a closure attached nothing is prepared.
extern "C" int dns2d_prepare(dns2d_state *s, int nsteps)
{
    if (!s || nsteps < 0) return DNS2D_ERR_ARG;
    if (s->cnn) return DNS2D_OK;
    for (int done = 0; done < nsteps;) {
        const int K = std::min(kChunk, nsteps - done);
        cudaGraphExec_t ex = nullptr;
        const int rc = get_graph(s, done == 0 ? 1 : 0, K, &ex);
        if (rc) return rc;
        done += K;
    }
    return DNS2D_OK;
}

extern "C" int dns2d_step(dns2d_state *s, int nsteps, double *E_hist, double *Z_hist)
{
    if (!s || nsteps < 0) return DNS2D_ERR_ARG;
    if (!s->initialised) return fail(s, DNS2D_ERR_STATE, "no initial condition");
    if (s->cnn) return closure_run(s, nsteps, E_hist, Z_hist);
    int done = 0;
    while (done < nsteps) {
        const int K = std::min(kChunk, nsteps - done);
        const int first = (done == 0) ? 1 : 0;
        // parameters of this chunk: within a dns2d_step call dt is constant; after the first
        // step of the call CNM1 == CN (cuda/step3_cuda.cu:172)
        const float cnm1_first = (done == 0) ? s->cnm1 : s->cn;
        k_set_params<<<1, 1, 0, s->stream>>>(s->prm, s->dt, cnm1_first, s->cn, s->visc);
        DNS2D_LAUNCHED("set params");
        if (s->timing) {
            const Pointers p = s->ptrs();
            for (int i = 0; i < K; ++i) {
                phase_begin(s);
                s->ks->rows_step(p, s->stream, 1);
                DNS2D_LAUNCHED("rows_step");
                phase_end(s, 0);
                phase_begin(s);
                s->ks->cols_step(p, (first && i == 0) ? 1 : 0, i, s->stream, 1);
                DNS2D_LAUNCHED("cols_step");
                phase_end(s, 1);
            }
        } else {
            cudaGraphExec_t ex = nullptr;
            int rc = get_graph(s, first, K, &ex);
            if (rc) return rc;
            DNS2D_CUDA(cudaGraphLaunch(ex, s->stream), "graph launch");
        }
        if (E_hist || Z_hist) {
            DNS2D_CUDA(cudaMemcpyAsync(s->hist_host, s->hist, (size_t)K * 16, cudaMemcpyDeviceToHost, s->stream),
                       "history copy");
            DNS2D_CUDA(cudaStreamSynchronize(s->stream), "history sync");
            for (int i = 0; i < K; ++i) {
                if (E_hist) E_hist[done + i] = s->hist_host[i].x;
                if (Z_hist) Z_hist[done + i] = s->hist_host[i].y;
            }
        }
        // host scalars, step by step like the reference loop
        for (int i = 0; i < K; ++i) {
            s->it += 1;
            const float dt_old = s->dt;
            s->cnm1 = s->cn;
            s->t += dt_old;
        }
        done += K;
    }
    return DNS2D_OK;
}

extern "C" void *dns2d_stream(dns2d_state *s) { return s ? (void *)s->stream : nullptr; }

extern "C" int dns2d_sync(dns2d_state *s, int timeout_ms)
{
    if (!s) return DNS2D_ERR_ARG;
    if (timeout_ms <= 0) {
        DNS2D_CUDA(cudaStreamSynchronize(s->stream), "sync");
        return DNS2D_OK;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        const cudaError_t e = cudaStreamQuery(s->stream);
        if (e == cudaSuccess) return DNS2D_OK;
        if (e != cudaErrorNotReady) return cuda_check(s, e, "sync");
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > timeout_ms) return fail(s, DNS2D_ERR_TIMEOUT, "device did not finish within %d ms", timeout_ms);
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

namespace {

int compute_cflm(dns2d_state *s, float *out)
{
    const float PI = 3.14159265358979323846f;
    const float DX = 2.0f * PI / float(s->N);
    DNS2D_CUDA(cudaMemsetAsync(s->cflm_dev, 0, 4, s->stream), "cflm clear");
    s->ks->rows_velocity(s->ptrs(), nullptr, s->cflm_dev, DX, s->stream, 1);
    DNS2D_LAUNCHED("rows_velocity(cfl)");
    float h = 0.0f;
    DNS2D_CUDA(cudaMemcpyAsync(&h, s->cflm_dev, 4, cudaMemcpyDeviceToHost, s->stream), "cflm copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "cflm sync");
    *out = h;
    return DNS2D_OK;
}

}  // namespace

extern "C" int dns2d_next_dt(dns2d_state *s, float *cflm_out)
{
    if (!s) return DNS2D_ERR_ARG;
    if (!s->initialised) return fail(s, DNS2D_ERR_STATE, "no initial condition");
    const float PI = 3.14159265358979323846f;
    phase_begin(s);
    float CFLM = 0.0f;
    // NEXTDT init branch (cuda/dns_cuda.cu:562-569) and regular update (:572-579)
    if (s->it == 0 && s->dt == 0.0f) {
        int rc = compute_cflm(s, &CFLM);
        if (rc) return rc;
        s->dt = s->cflnum / CFLM / PI;
        s->cflm = CFLM;
    } else if (s->ifn > 0 && (s->it % s->ifn) == 0) {
        int rc = compute_cflm(s, &CFLM);
        if (rc) return rc;
        const float CFL = CFLM * s->dt * PI;
        s->cn = 0.8f + 0.2f * (s->cflnum / CFL);
        s->dt = s->dt * s->cn;
        s->cflm = CFLM;
    }
    phase_end(s, 2);
    if (cflm_out) *cflm_out = s->cflm;
    return DNS2D_OK;
}

// ============================================================================================
// movie frames: inferno colour map of a physical plane (cuda/color_cuda.cu:37-232, :491-597)
// ============================================================================================
namespace {

__constant__ unsigned char c_inferno[256 * 3];

// five colour stops, linear in between, truncated to bytes (cuda/color_cuda.cu:37-70)
void inferno_lut(unsigned char lut[768])
{
    const float pos[5] = {0.00f, 0.25f, 0.50f, 0.75f, 1.00f};
    const unsigned char col[5][3] = {{0, 0, 4}, {87, 15, 109}, {187, 55, 84}, {249, 142, 8}, {252, 255, 164}};
    for (int i = 0; i < 256; ++i) {
        const float x = (float)i / 255.0f;
        int k = 0;
        while (k + 1 < 5 && x > pos[k + 1]) ++k;
        const int k1 = std::min(k + 1, 4);
        const float span = std::max(1.0e-12f, pos[k1] - pos[k]);
        const float t = std::max(0.0f, std::min(1.0f, (x - pos[k]) / span));
        for (int c = 0; c < 3; ++c) lut[3 * i + c] = (unsigned char)((1.0f - t) * col[k][c] + t * col[k1][c]);
    }
}

constexpr int kFrameBlocks = 1024;

// per-block min/max over the finite values
__global__ void k_frame_minmax(const float *f, size_t n, float2 *out)
{
    __shared__ float smn[256], smx[256];
    float mn = 3.402823466e38f, mx = -3.402823466e38f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = f[i];
        if (isfinite(v)) {
            mn = fminf(mn, v);
            mx = fmaxf(mx, v);
        }
    }
    smn[threadIdx.x] = mn;
    smx[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            smn[threadIdx.x] = fminf(smn[threadIdx.x], smn[threadIdx.x + o]);
            smx[threadIdx.x] = fmaxf(smx[threadIdx.x], smx[threadIdx.x + o]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = make_float2(smn[0], smx[0]);
}

// pixel value 1..255 of v (cuda/color_cuda.cu:150-160); 1 + 254 norm is one fused multiply-add, as the
// reference's nvcc build contracts it
__device__ __forceinline__ int frame_pixel(float v, float minv, float inv_range, int is_constant)
{
    if (is_constant || !isfinite(v)) return 128;
    const float norm = (v - minv) * inv_range;
    float pf = fmaf(norm, 254.0f, 1.0f);
    if (pf < 1.0f) pf = 1.0f;
    if (pf > 255.0f) pf = 255.0f;
    return (int)pf;
}

// per-block sums of pix and pix^2 (integers: exact in FP64, independent of the order)
__global__ void k_frame_stats(const float *f, size_t n, float minv, float inv_range, int is_constant, double2 *out)
{
    __shared__ double s1[256], s2[256];
    double a = 0.0, b = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double p = (double)frame_pixel(f[i], minv, inv_range, is_constant);
        a += p;
        b += p * p;
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = make_double2(s1[0], s2[0]);
}

// one output pixel per thread, sampling every F-th point; the colour index stretches
// [mean - 2.5 sigma, mean + 2.5 sigma] of the pixel values over the table when sigma >= 1
// rows [oy0, oy1) of the frame, written from rgb[0]
__global__ void k_frame_render(const float *f, unsigned char *rgb, int nx, int nz, int out_w, int oy0, int oy1, int F,
                               float minv, float inv_range, int is_constant, double mean, double sigma)
{
    const int ox = blockIdx.x * blockDim.x + threadIdx.x, oy = oy0 + blockIdx.y * blockDim.y + threadIdx.y;
    if (ox >= out_w || oy >= oy1) return;
    const int x = min(ox * F, nx - 1), y = min(oy * F, nz - 1);
    const int pix = frame_pixel(f[(size_t)y * nx + x], minv, inv_range, is_constant);
    int ci = pix;
    const double lo = mean - 2.5 * sigma, hi = mean + 2.5 * sigma;
    if (sigma >= 1.0 && hi > lo) {
        ci = (int)floor(((double)pix - lo) * 255.0 / (hi - lo) + 0.5);
        ci = ci < 0 ? 0 : (ci > 255 ? 255 : ci);
    }
    const size_t d = 3 * ((size_t)(oy - oy0) * out_w + ox);
    rgb[d] = c_inferno[3 * ci];
    rgb[d + 1] = c_inferno[3 * ci + 1];
    rgb[d + 2] = c_inferno[3 * ci + 2];
}

}  // namespace

// frame downsampling factor for size N (cuda/color_cuda.cu:491-498)
extern "C" int dns2d_movie_scale(int N)
{
    if (N == 9216) return 8;
    if (N == 16384) return 12;
    if (N == 29400) return 14;
    return std::max(1, (3 * N / 2 + 3839) / 3840);
}

extern "C" int dns2d_movie_frame(dns2d_state *s, int comp, int scale_f, unsigned char *rgb, int *width, int *height,
                                 double *sigma_out)
{
    if (!s || comp < 0 || comp > 2) return DNS2D_ERR_ARG;
    const int F = scale_f > 0 ? scale_f : 1;
    const int L = s->L;
    const int out_w = (L + F - 1) / F, out_h = (L + F - 1) / F;
    if (width) *width = out_w;
    if (height) *height = out_h;
    if (!rgb) return DNS2D_OK;
    const size_t plane = (size_t)L * L;
    const float *f = s->phys + (size_t)comp * plane;
    const int nb = (int)std::min<size_t>(kFrameBlocks, std::max<size_t>(1, (plane + 255) / 256));
    static_assert(kFrameBlocks <= kSigmaBlocks, "frame partials share the sigma buffers");
    s->mm_plane2 = 0;
    k_frame_minmax<<<nb, 256, 0, s->stream>>>(f, plane, s->minmax);
    DNS2D_LAUNCHED("frame minmax");
    std::vector<float2> mm((size_t)nb);
    DNS2D_CUDA(cudaMemcpyAsync(mm.data(), s->minmax, (size_t)nb * 8, cudaMemcpyDeviceToHost, s->stream), "minmax copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "minmax sync");
    float minv = mm[0].x, maxv = mm[0].y;
    for (int i = 1; i < nb; ++i) {
        minv = std::min(minv, mm[(size_t)i].x);
        maxv = std::max(maxv, mm[(size_t)i].y);
    }
    const float range = maxv - minv;
    const int is_constant = !(range > 1.0e-12f);
    const float inv_range = is_constant ? 1.0f : 1.0f / range;
    double2 *sums = reinterpret_cast<double2 *>(s->sums);
    k_frame_stats<<<nb, 256, 0, s->stream>>>(f, plane, minv, inv_range, is_constant, sums);
    DNS2D_LAUNCHED("frame stats");
    std::vector<double2> st((size_t)nb);
    DNS2D_CUDA(cudaMemcpyAsync(st.data(), sums, (size_t)nb * 16, cudaMemcpyDeviceToHost, s->stream), "stats copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "stats sync");
    double a = 0.0, b = 0.0;
    for (int i = 0; i < nb; ++i) {
        a += st[(size_t)i].x;
        b += st[(size_t)i].y;
    }
    const double mean = a / (double)plane;
    const double sigma = std::sqrt(std::max(0.0, b / (double)plane - mean * mean));
    if (sigma_out) *sigma_out = sigma;
    unsigned char lut[768];
    inferno_lut(lut);
    DNS2D_CUDA(cudaMemcpyToSymbolAsync(c_inferno, lut, sizeof(lut), 0, cudaMemcpyHostToDevice, s->stream), "lut copy");
    // the frame goes through the scratch buffer (8 L H bytes) in bands of rows: at F = 1 the whole
    // frame (3 L^2 bytes) is larger than the buffer
    unsigned char *d_rgb = reinterpret_cast<unsigned char *>(s->scratch);
    const int band = (int)std::min<size_t>(out_h, (size_t)8 * L * s->H / ((size_t)3 * out_w));
    for (int oy0 = 0; oy0 < out_h; oy0 += band) {
        const int oy1 = std::min(out_h, oy0 + band);
        const dim3 blk(16, 16), grd((out_w + 15) / 16, (oy1 - oy0 + 15) / 16);
        k_frame_render<<<grd, blk, 0, s->stream>>>(f, d_rgb, L, L, out_w, oy0, oy1, F, minv, inv_range, is_constant,
                                                   mean, sigma);
        DNS2D_LAUNCHED("movie frame");
        DNS2D_CUDA(cudaMemcpyAsync(rgb + (size_t)3 * out_w * oy0, d_rgb, (size_t)3 * out_w * (oy1 - oy0),
                                   cudaMemcpyDeviceToHost, s->stream),
                   "rgb copy");
    }
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "rgb sync");
    return DNS2D_OK;
}

// ============================================================================================
// diagnostics
// ============================================================================================
extern "C" int dns2d_om2phys(dns2d_state *s)
{
    if (!s) return DNS2D_ERR_ARG;
    phase_begin(s);
    const size_t plane = (size_t)s->L * s->L;
    s->ks->cols_scalar(s->ptrs(), s->scratch, 0, s->stream);
    DNS2D_LAUNCHED("cols_scalar");
    s->ks->rows_scalar(s->ptrs(), s->scratch, s->phys + 2 * plane, s->minmax, s->stream);
    DNS2D_LAUNCHED("rows_scalar");
    s->mm_plane2 = s->ks->scalar_parts;
    phase_end(s, 3);
    return DNS2D_OK;
}

extern "C" int dns2d_stream_func(dns2d_state *s)
{
    if (!s) return DNS2D_ERR_ARG;
    const size_t plane = (size_t)s->L * s->L;
    s->ks->cols_scalar(s->ptrs(), s->scratch, 1, s->stream);
    DNS2D_LAUNCHED("cols_scalar(psi)");
    s->ks->rows_scalar(s->ptrs(), s->scratch, s->phys + 2 * plane, s->minmax, s->stream);
    DNS2D_LAUNCHED("rows_scalar(psi)");
    s->mm_plane2 = s->ks->scalar_parts;
    return DNS2D_OK;
}

extern "C" int dns2d_velocity_phys(dns2d_state *s)
{
    if (!s) return DNS2D_ERR_ARG;
    if (!s->initialised) return fail(s, DNS2D_ERR_STATE, "no initial condition");
    s->ks->rows_velocity(s->ptrs(), s->phys, nullptr, 1.0f, s->stream, 1);
    DNS2D_LAUNCHED("rows_velocity(phys)");
    return DNS2D_OK;
}

extern "C" int dns2d_kinetic(dns2d_state *s)
{
    if (!s) return DNS2D_ERR_ARG;
    const size_t plane = (size_t)s->L * s->L;
    s->mm_plane2 = 0;
    k_kinetic<<<1024, 256, 0, s->stream>>>(s->phys, plane);
    DNS2D_LAUNCHED("kinetic");
    return DNS2D_OK;
}

namespace {
// sigma = sqrt(E[pix^2] - E[pix]^2) from the per-block pixel sums (integers: exact)
int sigma_finish(dns2d_state *s, int nb, size_t plane, double *sigma)
{
    std::vector<unsigned long long> hs((size_t)nb * 2);
    DNS2D_CUDA(cudaMemcpyAsync(hs.data(), s->sums, (size_t)nb * 16, cudaMemcpyDeviceToHost, s->stream), "sums copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "sums sync");
    unsigned long long a = 0, b = 0;
    for (int i = 0; i < nb; ++i) {
        a += hs[2 * (size_t)i];
        b += hs[2 * (size_t)i + 1];
    }
    const double mean = (double)a / (double)plane;
    const double var = std::max(0.0, (double)b / (double)plane - mean * mean);
    *sigma = std::sqrt(var);
    phase_end(s, 3);
    return DNS2D_OK;
}
}  // namespace

extern "C" int dns2d_display_sigma(dns2d_state *s, int comp, double *sigma)
{
    if (!s || !sigma || comp < 0 || comp > 2) return DNS2D_ERR_ARG;
    phase_begin(s);
    const size_t plane = (size_t)s->L * s->L;
    const float *f = s->phys + (size_t)comp * plane;
    const int nb = (int)std::min<size_t>(kSigmaBlocks, std::max<size_t>(1, (plane + 255) / 256));
    if (comp == 2 && s->mm_plane2 > 0) {  // min / max partials of this plane from OM2PHYS
        k_sigma_pixels_mm<<<nb, 256, 0, s->stream>>>(f, plane, s->minmax, s->mm_plane2, s->sums);
        DNS2D_LAUNCHED("sigma pixels");
        return sigma_finish(s, nb, plane, sigma);
    }
    s->mm_plane2 = 0;
    k_minmax<<<nb, 256, 0, s->stream>>>(f, plane, s->minmax);
    DNS2D_LAUNCHED("minmax");
    std::vector<float2> mm((size_t)nb);
    DNS2D_CUDA(cudaMemcpyAsync(mm.data(), s->minmax, (size_t)nb * 8, cudaMemcpyDeviceToHost, s->stream), "minmax copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "minmax sync");
    float minv = mm[0].x, maxv = mm[0].y;
    for (int i = 1; i < nb; ++i) {
        minv = std::min(minv, mm[(size_t)i].x);
        maxv = std::max(maxv, mm[(size_t)i].y);
    }
    const float rng = maxv - minv;
    const int is_constant = (std::fabs(rng) <= 1.0e-12f) ? 1 : 0;
    k_sigma_pixels<<<nb, 256, 0, s->stream>>>(f, plane, minv, rng, is_constant, s->sums);
    DNS2D_LAUNCHED("sigma pixels");
    return sigma_finish(s, nb, plane, sigma);
}

namespace {
int om2_reduce(dns2d_state *s, double *v6)
{
    k_om2_reduce<<<kRedBlocks, 256, 0, s->stream>>>(s->om2, s->N, s->red);
    DNS2D_LAUNCHED("om2 reduce");
    std::vector<double> h((size_t)kRedBlocks * 6);
    DNS2D_CUDA(cudaMemcpyAsync(h.data(), s->red, h.size() * 8, cudaMemcpyDeviceToHost, s->stream), "reduce copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "reduce sync");
    for (int j = 0; j < 6; ++j) v6[j] = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) {
        for (int j = 0; j < 5; ++j) v6[j] += h[6 * (size_t)b + j];
        v6[5] = std::max(v6[5], h[6 * (size_t)b + 5]);
    }
    return DNS2D_OK;
}
}  // namespace

extern "C" int dns2d_energy_enstrophy(dns2d_state *s, double *E, double *Z)
{
    if (!s) return DNS2D_ERR_ARG;
    double v[6];
    int rc = om2_reduce(s, v);
    if (rc) return rc;
    if (E) *E = v[0];
    if (Z) *Z = v[1];
    return DNS2D_OK;
}

extern "C" int dns2d_palin(dns2d_state *s, double *out)
{
    if (!s || !out) return DNS2D_ERR_ARG;
    double v[6];
    int rc = om2_reduce(s, v);
    if (rc) return rc;
    const double total = v[3] - v[4];
    *out = (total <= 0.0 || v[5] <= 0.0) ? 0.0 : v[2] / (total * v[5]);
    return DNS2D_OK;
}

extern "C" int dns2d_shell_spectrum(dns2d_state *s, double *Ek, int nb)
{
    if (!s || !Ek || nb <= 0) return DNS2D_ERR_ARG;
    double *d = nullptr;
    DNS2D_CUDA(cudaMallocAsync((void **)&d, (size_t)nb * 8, s->stream), "shell alloc");
    DNS2D_CUDA(cudaMemsetAsync(d, 0, (size_t)nb * 8, s->stream), "shell clear");
    k_shell<<<512, 256, 0, s->stream>>>(s->om2, s->N, d, nb);
    DNS2D_LAUNCHED("shell");
    DNS2D_CUDA(cudaMemcpyAsync(Ek, d, (size_t)nb * 8, cudaMemcpyDeviceToHost, s->stream), "shell copy");
    DNS2D_CUDA(cudaFreeAsync(d, s->stream), "shell free");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "shell sync");
    return DNS2D_OK;
}

extern "C" int dns2d_velocity_spectrum_bins(dns2d_state *s, double *esum, int *count, int nbins)
{
    if (!s || !esum || !count || nbins <= 0) return DNS2D_ERR_ARG;
    if (s->ks->velocity_r2c_full) {
        // the reference's procedure (cuda/mem_cuda.cu:579-649): forward R2C of the physical u, w
        // over every mode of the L x L grid, then the shell sums on the host in its loop order
        // (z outer, kx inner), so every bin it writes -- the retained band and the transform's
        // rounding noise beyond it -- is formed the same way
        const int L = s->L, NK = L / 2 + 1;
        const size_t plane = (size_t)L * NK;
        int rc = dns2d_velocity_phys(s);
        if (rc) return rc;
        float2 *d = nullptr;
        DNS2D_CUDA(cudaMallocAsync((void **)&d, 2 * plane * sizeof(float2), s->stream), "spectrum alloc");
        s->ks->velocity_r2c_full(s->ptrs(), s->phys, d, s->stream);
        DNS2D_LAUNCHED("velocity r2c");
        std::vector<float2> h(2 * plane);
        DNS2D_CUDA(cudaMemcpyAsync(h.data(), d, 2 * plane * sizeof(float2), cudaMemcpyDeviceToHost, s->stream),
                   "spectrum copy");
        DNS2D_CUDA(cudaFreeAsync(d, s->stream), "spectrum free");
        DNS2D_CUDA(cudaStreamSynchronize(s->stream), "spectrum sync");
        std::fill(esum, esum + nbins, 0.0);
        std::fill(count, count + nbins, 0);
        const double r_max = std::sqrt(2.0), k_nyq = 0.5 * (double)L;
        for (int z = 0; z < L; ++z) {
            const int kz = (z <= L / 2) ? z : z - L;
            for (int kx = 0; kx < NK; ++kx) {
                if (kx == 0 && kz == 0) continue;
                const double r = std::sqrt((double)(kx * kx + kz * kz)) / k_nyq;
                int bin = (int)std::floor((r / r_max) * nbins);
                bin = std::min(std::max(bin, 0), nbins - 1);
                const float2 u = h[(size_t)z * NK + kx], v = h[plane + (size_t)z * NK + kx];
                double p = (double)u.x * u.x + (double)u.y * u.y + (double)v.x * v.x + (double)v.y * v.y;
                const bool dbl = kx > 0 && kx < L / 2;
                if (dbl) p *= 2.0;
                esum[bin] += p;
                count[bin] += dbl ? 2 : 1;
            }
        }
        return DNS2D_OK;
    }
    // cluster sizes: the retained modes from the spectral state (exact; the bins beyond the
    // retained radius, which hold only transform rounding noise, stay empty)
    double *d = nullptr;
    int *c = nullptr;
    DNS2D_CUDA(cudaMallocAsync((void **)&d, (size_t)nbins * 8, s->stream), "bins alloc");
    DNS2D_CUDA(cudaMallocAsync((void **)&c, (size_t)nbins * 4, s->stream), "bins alloc");
    DNS2D_CUDA(cudaMemsetAsync(d, 0, (size_t)nbins * 8, s->stream), "bins clear");
    DNS2D_CUDA(cudaMemsetAsync(c, 0, (size_t)nbins * 4, s->stream), "bins clear");
    k_vel_bins<<<1024, 256, 0, s->stream>>>(s->om2, s->N, d, c, nbins);
    DNS2D_LAUNCHED("velocity bins");
    DNS2D_CUDA(cudaMemcpyAsync(esum, d, (size_t)nbins * 8, cudaMemcpyDeviceToHost, s->stream), "bins copy");
    DNS2D_CUDA(cudaMemcpyAsync(count, c, (size_t)nbins * 4, cudaMemcpyDeviceToHost, s->stream), "bins copy");
    DNS2D_CUDA(cudaFreeAsync(d, s->stream), "bins free");
    DNS2D_CUDA(cudaFreeAsync(c, s->stream), "bins free");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "bins sync");
    return DNS2D_OK;
}

// ============================================================================================
// state transfer
// ============================================================================================
extern "C" int dns2d_get_scalars(const dns2d_state *s, dns2d_scalars *o)
{
    if (!s || !o) return DNS2D_ERR_ARG;
    o->N = s->N;
    o->NX_full = s->L;
    o->NK_full = s->Nk;
    o->it = s->it;
    o->ifn = s->ifn;
    o->Re = s->Re;
    o->K0 = s->K0;
    o->visc = s->visc;
    o->t = s->t;
    o->dt = s->dt;
    o->cn = s->cn;
    o->cnm1 = s->cnm1;
    o->cflnum = s->cflnum;
    o->cflm = s->cflm;
    return DNS2D_OK;
}

extern "C" int dns2d_set_scalars(dns2d_state *s, const dns2d_scalars *i)
{
    if (!s || !i) return DNS2D_ERR_ARG;
    if (i->N != s->N) return fail(s, DNS2D_ERR_ARG, "scalars for N=%d on a state of N=%d", i->N, s->N);
    s->it = i->it;
    s->ifn = i->ifn;
    s->Re = i->Re;
    s->K0 = i->K0;
    s->visc = i->visc;
    s->t = i->t;
    s->dt = i->dt;
    s->cn = i->cn;
    s->cnm1 = i->cnm1;
    s->cflnum = i->cflnum;
    s->cflm = i->cflm;
    return DNS2D_OK;
}

extern "C" int dns2d_get_om2(dns2d_state *s, float *om2)
{
    if (!s || !om2) return DNS2D_ERR_ARG;
    return download_compact(s, s->om2, om2);
}

extern "C" int dns2d_get_fnm1(dns2d_state *s, float *fnm1)
{
    if (!s || !fnm1) return DNS2D_ERR_ARG;
    return download_compact(s, s->fnm1, fnm1);
}

extern "C" int dns2d_get_phys(dns2d_state *s, int comp, float *plane)
{
    if (!s || !plane || comp < 0 || comp > 2) return DNS2D_ERR_ARG;
    const size_t n = (size_t)s->L * s->L;
    DNS2D_CUDA(cudaMemcpyAsync(plane, s->phys + (size_t)comp * n, n * 4, cudaMemcpyDeviceToHost, s->stream), "phys copy");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "phys sync");
    return DNS2D_OK;
}

extern "C" int dns2d_set_velocity_phys(dns2d_state *s, const float *u, const float *w)
{
    if (!s || !u || !w) return DNS2D_ERR_ARG;
    const size_t n = (size_t)s->L * s->L;
    DNS2D_CUDA(cudaMemcpyAsync(s->phys, u, n * 4, cudaMemcpyHostToDevice, s->stream), "u upload");
    DNS2D_CUDA(cudaMemcpyAsync(s->phys + n, w, n * 4, cudaMemcpyHostToDevice, s->stream), "w upload");
    s->ks->rows_from_phys(s->ptrs(), s->phys, s->stream);
    DNS2D_LAUNCHED("rows_from_phys");
    DNS2D_CUDA(cudaStreamSynchronize(s->stream), "velocity upload");
    s->initialised = true;
    return DNS2D_OK;
}

// ============================================================================================
// restart.bin (cuda/mem_cuda.cu:1019-1054 header, :1236-1394 writer/reader).
// Little-endian, natural alignment: v1 header 136 bytes, v2 adds ur_full_count (144 bytes).
// ============================================================================================
namespace {

#pragma pack(push, 4)
struct RestartV1 {
    char magic[16];
    uint32_t version, header_bytes, real_bytes, cplx_bytes;
    int32_t Nbase, N, NX, NZ, NK, NX_full, NZ_full, NK_full, it, ifn;
    float Re, K0, visc, t, dt, cn, cnm1, cflnum, cflm;
    uint32_t pad_;
    uint64_t uc_full_count, om2_count, fnm1_count;
};
#pragma pack(pop)
static_assert(sizeof(RestartV1) == 136, "restart v1 header size");
struct RestartV2 {
    RestartV1 v1;
    uint64_t ur_full_count;
};
static_assert(sizeof(RestartV2) == 144, "restart v2 header size");

}  // namespace

namespace {

// Restart files move through pinned staging buffers: file chunk k (stage_chunk bytes from the
// start of the payload range) lives in buffer k % kStageBufs. Saving keeps kStageBufs
// device->host copies in flight while the host writes the oldest finished chunk; loading reads
// chunk k from the file (kReadThreads preads in parallel) while the host->device copies of the
// chunks before it run. Each region of the file is one contiguous device range, so a chunk is at
// most a few cudaMemcpyAsync calls; the file's [iz][ix] OM2/FNM1 and the state's [ix][iz] are
// transposed on the device, one array at a time through the scratch buffer.
constexpr int kStageBufs = 3;
constexpr size_t kStageChunkMax = 64ull << 20;
constexpr int kReadThreads = 4;

// file bytes [off, off + len) are dev[0, len) (or host[0, len) for the header); `before` (save)
// is enqueued ahead of the region's first copy, `after` (load) behind its last
struct FileRegion {
    uint64_t off, len;
    unsigned char *dev;
    const unsigned char *host;
    std::function<void()> before, after;
};

int stage_reserve(dns2d_state *s, uint64_t bytes)
{
    const size_t want = std::min<size_t>(
        kStageChunkMax, std::max<size_t>(4096, ((bytes + kStageBufs - 1) / kStageBufs + 4095) / 4096 * 4096));
    if (s->stage && s->stage_chunk >= want) return DNS2D_OK;
    if (s->stage) cudaFreeHost(s->stage);
    s->stage = nullptr;
    s->stage_chunk = 0;
    DNS2D_CUDA(cudaHostAlloc((void **)&s->stage, want * kStageBufs, cudaHostAllocDefault), "staging buffers");
    s->stage_chunk = want;
    for (cudaEvent_t &e : s->stage_ev)
        if (!e) DNS2D_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "staging events");
    return DNS2D_OK;
}

bool write_all(int fd, const unsigned char *p, size_t n)
{
    while (n > 0) {
        const ssize_t w = ::write(fd, p, std::min<size_t>(n, 1ull << 30));
        if (w < 0 && errno == EINTR) continue;
        if (w <= 0) return false;
        p += w;
        n -= (size_t)w;
    }
    return true;
}

bool pread_all(int fd, unsigned char *p, size_t n, uint64_t off)
{
    while (n > 0) {
        const ssize_t r = ::pread(fd, p, std::min<size_t>(n, 1ull << 30), (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return false;
        p += r;
        n -= (size_t)r;
        off += (uint64_t)r;
    }
    return true;
}

// file bytes [lo, hi) into buf, by up to kReadThreads threads reading contiguous slices
bool pread_parallel(int fd, unsigned char *buf, uint64_t lo, uint64_t hi)
{
    const uint64_t n = hi - lo;
    const int t = n >= (8ull << 20) ? kReadThreads : 1;
    if (t == 1) return pread_all(fd, buf, n, lo);
    const uint64_t part = (n + t - 1) / t;
    bool ok[kReadThreads];
    std::vector<std::thread> th;
    for (int i = 0; i < t; ++i) {
        const uint64_t a = std::min<uint64_t>(n, i * part), b = std::min<uint64_t>(n, a + part);
        ok[i] = true;
        th.emplace_back([&ok, fd, buf, lo, i, a, b] { ok[i] = pread_all(fd, buf + a, b - a, lo + a); });
    }
    for (auto &x : th) x.join();
    return std::all_of(ok, ok + t, [](bool v) { return v; });
}

void transpose_c64(dns2d_state *s, const float2 *in, float2 *out, int rows, int cols)
{
    dim3 b(32, 8), g((cols + 31) / 32, (rows + 31) / 32);
    k_transpose_c64<<<g, b, 0, s->stream>>>(in, out, rows, cols);
}

}  // namespace

extern "C" int dns2d_save_restart(dns2d_state *s, const char *path)
{
    if (!s || !path) return DNS2D_ERR_ARG;
    const size_t n = (size_t)s->L * s->L, nom = (size_t)s->N * s->H;
    RestartV2 h;
    std::memset(&h, 0, sizeof(h));
    std::snprintf(h.v1.magic, sizeof(h.v1.magic), "CTRB_RESTART");
    h.v1.version = 2;
    h.v1.header_bytes = sizeof(RestartV2);
    h.v1.real_bytes = 4;
    h.v1.cplx_bytes = 8;
    h.v1.Nbase = h.v1.N = h.v1.NX = h.v1.NZ = s->N;
    h.v1.NK = h.v1.NK_full = s->Nk;
    h.v1.NX_full = h.v1.NZ_full = s->L;
    h.v1.it = s->it;
    h.v1.ifn = s->ifn;
    h.v1.Re = s->Re;
    h.v1.K0 = s->K0;
    h.v1.visc = s->visc;
    h.v1.t = s->t;
    h.v1.dt = s->dt;
    h.v1.cn = s->cn;
    h.v1.cnm1 = s->cnm1;
    h.v1.cflnum = s->cflnum;
    h.v1.cflm = s->cflm;
    h.v1.uc_full_count = 0;
    h.v1.om2_count = h.v1.fnm1_count = nom;
    h.ur_full_count = 3 * n;
    int rc = dns2d_velocity_phys(s);
    if (rc) return rc;
    const uint64_t hb = sizeof(h), ur = 3 * n * 4, om = nom * 8, total = hb + ur + 2 * om;
    unsigned char *scr = reinterpret_cast<unsigned char *>(s->scratch);
    // file order: header, UR_full (three planes), OM2, FNM1 in [iz][ix]; the scratch buffer holds
    // OM2 then FNM1 (stream order keeps FNM1's transpose behind OM2's last copy out of it)
    const FileRegion reg[4] = {
        {0, hb, nullptr, reinterpret_cast<const unsigned char *>(&h), nullptr, nullptr},
        {hb, ur, reinterpret_cast<unsigned char *>(s->phys), nullptr, nullptr, nullptr},
        {hb + ur, om, scr, nullptr, [&] { transpose_c64(s, s->om2, s->scratch, s->H, s->N); }, nullptr},
        {hb + ur + om, om, scr, nullptr, [&] { transpose_c64(s, s->fnm1, s->scratch, s->H, s->N); }, nullptr},
    };
    rc = stage_reserve(s, total);
    if (rc) return rc;
    const uint64_t C = s->stage_chunk, nch = (total + C - 1) / C;
    const int fd = ::open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return fail(s, DNS2D_ERR_IO, "cannot open %s: %s", path, std::strerror(errno));
    cudaError_t ce = cudaSuccess;
    auto enqueue = [&](uint64_t k) {
        unsigned char *buf = s->stage + (k % kStageBufs) * C;
        const uint64_t lo = k * C, hi = std::min(total, lo + C);
        for (const FileRegion &r : reg) {
            const uint64_t a = std::max(lo, r.off), b = std::min(hi, r.off + r.len);
            if (a >= b) continue;
            if (a == r.off && r.before) r.before();
            if (r.host)
                std::memcpy(buf + (a - lo), r.host + (a - r.off), b - a);
            else if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(buf + (a - lo), r.dev + (a - r.off), b - a, cudaMemcpyDeviceToHost, s->stream);
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(s->stage_ev[k % kStageBufs], s->stream);
    };
    bool ok = true;
    for (uint64_t k = 0; k < std::min<uint64_t>(nch, kStageBufs); ++k) enqueue(k);
    for (uint64_t k = 0; k < nch && ok && ce == cudaSuccess; ++k) {
        ce = cudaEventSynchronize(s->stage_ev[k % kStageBufs]);
        if (ce != cudaSuccess) break;
        const uint64_t lo = k * C, hi = std::min(total, lo + C);
        ok = write_all(fd, s->stage + (k % kStageBufs) * C, hi - lo);
        if (ok && k + kStageBufs < nch) enqueue(k + kStageBufs);  // into the buffer just written
    }
    if (ce == cudaSuccess) ce = cudaGetLastError();  // the transposes
    const cudaError_t se = cudaStreamSynchronize(s->stream);
    if (::close(fd) != 0) ok = false;
    if (ce == cudaSuccess) ce = se;
    if (ce != cudaSuccess) return cuda_check(s, ce, "restart staging");
    return ok ? DNS2D_OK : fail(s, DNS2D_ERR_IO, "write failed: %s", path);
}

extern "C" int dns2d_load_restart(dns2d_state *s, const char *path)
{
    if (!s || !path) return DNS2D_ERR_ARG;
    s->mm_plane2 = 0;  // the file's UR planes replace the physical planes
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return fail(s, DNS2D_ERR_IO, "cannot open %s", path);
    RestartV2 h;
    std::memset(&h, 0, sizeof(h));
    auto bad = [&](int code, const char *msg) {
        ::close(fd);
        return fail(s, code, "%s: %s", path, msg);
    };
    struct stat st;
    if (fstat(fd, &st) != 0) return bad(DNS2D_ERR_IO, "stat");
    if (!pread_all(fd, reinterpret_cast<unsigned char *>(&h.v1), sizeof(h.v1), 0))
        return bad(DNS2D_ERR_IO, "short header");
    if (std::strncmp(h.v1.magic, "CTRB_RESTART", 12) != 0) return bad(DNS2D_ERR_FORMAT, "bad magic");
    if (h.v1.version == 2) {
        if (h.v1.header_bytes != sizeof(RestartV2)) return bad(DNS2D_ERR_FORMAT, "header size");
        if (!pread_all(fd, reinterpret_cast<unsigned char *>(&h.ur_full_count), 8, sizeof(h.v1)))
            return bad(DNS2D_ERR_IO, "short header");
    }
    if (h.v1.version < 1 || h.v1.version > 2 || (h.v1.version == 1 && h.v1.header_bytes != sizeof(RestartV1)) ||
        h.v1.real_bytes != 4 || h.v1.cplx_bytes != 8)
        return bad(DNS2D_ERR_FORMAT, "unsupported format");
    if (h.v1.Nbase != s->N || h.v1.N != s->N || h.v1.NX != s->N || h.v1.NZ != s->N || h.v1.NK != s->Nk ||
        h.v1.NX_full != s->L || h.v1.NZ_full != s->L || h.v1.NK_full != s->Nk)
        return bad(DNS2D_ERR_FORMAT, "dimensions do not match this run");
    const uint64_t ucn = (uint64_t)s->Nk * s->L * 3, urn = (uint64_t)s->L * s->L * 3, omn = (uint64_t)s->N * s->H;
    const bool has_uc = h.v1.uc_full_count != 0;
    if ((h.v1.version == 1 && h.v1.uc_full_count != ucn) || (h.v1.version >= 2 && has_uc && h.v1.uc_full_count != ucn) ||
        (h.v1.version >= 2 && h.ur_full_count != urn) || h.v1.om2_count != omn || h.v1.fnm1_count != omn)
        return bad(DNS2D_ERR_FORMAT, "array sizes do not match this run");
    // the UC_full payload (v1, or v2 with one) is not read: the velocity is rebuilt from UR or OM2
    const uint64_t hb = h.v1.header_bytes, uc = (h.v1.version == 1 || has_uc) ? h.v1.uc_full_count * 8 : 0;
    const uint64_t ur = h.v1.version >= 2 ? urn * 4 : 0, om = omn * 8;
    const uint64_t first = hb + uc, end = first + ur + 2 * om;
    if ((uint64_t)st.st_size < end) return bad(DNS2D_ERR_IO, "short payload");
    int rc = stage_reserve(s, end - first);
    if (rc) {
        ::close(fd);
        return rc;
    }
    unsigned char *scr = reinterpret_cast<unsigned char *>(s->scratch);
    const FileRegion reg[3] = {
        {first, ur, reinterpret_cast<unsigned char *>(s->phys), nullptr, nullptr, nullptr},
        {first + ur, om, scr, nullptr, nullptr, [&] { transpose_c64(s, s->scratch, s->om2, s->N, s->H); }},
        {first + ur + om, om, scr, nullptr, nullptr, [&] { transpose_c64(s, s->scratch, s->fnm1, s->N, s->H); }},
    };
    // from here on the device state is overwritten: a failure leaves it without an initial condition
    s->initialised = false;
    const uint64_t C = s->stage_chunk, nch = (end - first + C - 1) / C;
    cudaError_t ce = cudaSuccess;
    bool ok = true;
    for (uint64_t k = 0; k < nch && ok && ce == cudaSuccess; ++k) {
        unsigned char *buf = s->stage + (k % kStageBufs) * C;
        if (k >= kStageBufs) ce = cudaEventSynchronize(s->stage_ev[k % kStageBufs]);  // its last copies done
        if (ce != cudaSuccess) break;
        const uint64_t lo = first + k * C, hi = std::min(end, lo + C);
        ok = pread_parallel(fd, buf, lo, hi);
        if (!ok) break;
        for (const FileRegion &r : reg) {
            const uint64_t a = std::max(lo, r.off), b = std::min(hi, r.off + r.len);
            if (a >= b) continue;
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(r.dev + (a - r.off), buf + (a - lo), b - a, cudaMemcpyHostToDevice, s->stream);
            if (b == r.off + r.len && r.after) r.after();
        }
        if (ce == cudaSuccess) ce = cudaEventRecord(s->stage_ev[k % kStageBufs], s->stream);
    }
    ::close(fd);
    if (ok && ce == cudaSuccess) {
        if (h.v1.version >= 2)
            s->ks->rows_from_phys(s->ptrs(), s->phys, s->stream);
        else
            s->ks->cols_init(s->ptrs(), nullptr, 1, s->stream, 1);  // velocity from OM2 (v1)
        ce = cudaGetLastError();
    }
    const cudaError_t se = cudaStreamSynchronize(s->stream);
    if (ce == cudaSuccess) ce = se;
    if (ce != cudaSuccess) return cuda_check(s, ce, "restart staging");
    if (!ok) return fail(s, DNS2D_ERR_IO, "%s: read failed", path);
    s->Re = h.v1.Re;
    s->K0 = h.v1.K0;
    s->visc = h.v1.visc;
    s->t = h.v1.t;
    s->dt = h.v1.dt;
    s->cn = h.v1.cn;
    s->cnm1 = h.v1.cnm1;
    s->cflnum = h.v1.cflnum;
    s->cflm = h.v1.cflm;
    s->it = h.v1.it;
    s->ifn = h.v1.ifn;
    s->initialised = true;
    return DNS2D_OK;
}

// ============================================================================================
// phase timing
// ============================================================================================
extern "C" int dns2d_phase_timing(dns2d_state *s, int enable)
{
    if (!s) return DNS2D_ERR_ARG;
    s->timing = enable != 0;
    for (int i = 0; i < 4; ++i) {
        s->phase_ms[i] = 0.0;
        s->phase_n[i] = 0;
    }
    return DNS2D_OK;
}

extern "C" int dns2d_phase_report(dns2d_state *s, double *ms, long long *counts)
{
    if (!s) return DNS2D_ERR_ARG;
    for (int i = 0; i < 4; ++i) {
        if (ms) ms[i] = s->phase_ms[i];
        if (counts) counts[i] = s->phase_n[i];
    }
    return DNS2D_OK;
}

// ============================================================================================
// Batched ensembles: independent runs of (possibly different) N, Re, K0, CFL advanced together.
// Members are grouped by N; each group's state, work buffer and parameter blocks are contiguous
// and every kernel of a group covers all its members in one launch (member = blockIdx.y).  A
// chunk of up to 128 ensemble steps (row + column pass of every group) is one captured CUDA
// graph.  Each member keeps the reference's float scalar bookkeeping on the host.
// ============================================================================================
namespace {

struct BatchGroup {
    int N = 0, H = 0, L = 0, count = 0;
    const KernelSet *ks = nullptr;
    std::vector<int> members;  // batch indices of this group's members, in group order
    float2 *om2 = nullptr, *fnm1 = nullptr, *work = nullptr, *tw = nullptr;
    StepParams *prm = nullptr;
    double2 *part = nullptr, *hist = nullptr;
    unsigned int *counter = nullptr;
    float *cflm = nullptr;
    Tuning tune;

    Pointers ptrs() const
    {
        Pointers p;
        p.om2 = om2;
        p.fnm1 = fnm1;
        p.work = work;
        p.tw = tw;
        p.prm = prm;
        p.part = part;
        p.counter = counter;
        p.hist = hist;
        p.force = nullptr;
        p.gate = nullptr;
        p.s_state = (size_t)N * H;
        p.s_work = 2 * (size_t)L * H;
        p.s_part = H;
        p.s_hist = kChunk;
        apply_tuning(p, tune);
        return p;
    }
};

struct MemberScalars {
    float Re, K0, visc, t, dt, cn, cnm1, cflnum, cflm;
    int it, ifn;
    uint64_t seed;
};

}  // namespace

struct dns2d_batch {
    int count = 0, device = 0;
    cudaStream_t stream = nullptr;
    std::vector<MemberScalars> sc;
    std::vector<std::pair<int, int>> where;  // member -> (group, index in group)
    std::vector<BatchGroup> groups;
    StepParams *prm_host = nullptr;  // pinned, count entries (group order)
    double2 *hist_host = nullptr;    // pinned, count * kChunk entries
    float *cflm_host = nullptr;      // pinned, count entries
    cudaEvent_t prm_copied = nullptr;
    // one capture stream per size group: the groups' step chains are independent, so a chunk's
    // graph holds them as parallel branches (forked from and joined back into `stream`)
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    // stepping mode: 0 = one CUDA graph per chunk with each size group's row / column kernels as
    // a branch; 1 = one persistent launch per chunk (ensemble.cuh)
    int mode = 0;
    unsigned int *ens = nullptr;  // persistent launch: ticket, rows_done[count], cols_done[count], status
    int *ens_status_host = nullptr;
    long long spin_limit = 1ll << 22;  // polls of a dependency counter (~1 s) before a wait gives up
    int stall_member = -1;
    int ens_grid = 0;
    int tiles_per_item = 8, groups_per_item = 4;  // persistent launch work-item size (powers of two)
    bool initialised = false;
    std::string err;
};

namespace {

int bfail(dns2d_batch *b, int code, const char *what, cudaError_t e = cudaSuccess)
{
    if (b) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s%s%s", what, e != cudaSuccess ? ": " : "",
                      e != cudaSuccess ? cudaGetErrorString(e) : "");
        b->err = buf;
    }
    return code;
}

#define BATCH_CUDA(call, what)                                                   \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return bfail(b, DNS2D_ERR_CUDA, what, e_);        \
    } while (0)

}  // namespace

extern "C" void dns2d_batch_destroy(dns2d_batch *b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    for (BatchGroup &g : b->groups) {
        cudaFree(g.om2);
        cudaFree(g.fnm1);
        cudaFree(g.work);
        cudaFree(g.tw);
        cudaFree(g.prm);
        cudaFree(g.part);
        cudaFree(g.hist);
        cudaFree(g.counter);
        cudaFree(g.cflm);
    }
    cudaFree(b->ens);
    if (b->ens_status_host) cudaFreeHost(b->ens_status_host);
    if (b->prm_host) cudaFreeHost(b->prm_host);
    if (b->hist_host) cudaFreeHost(b->hist_host);
    if (b->cflm_host) cudaFreeHost(b->cflm_host);
    if (b->prm_copied) cudaEventDestroy(b->prm_copied);
    for (cudaStream_t q : b->side)
        if (q) cudaStreamDestroy(q);
    for (cudaEvent_t e : b->joins)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

extern "C" const char *dns2d_batch_last_error(const dns2d_batch *b) { return b ? b->err.c_str() : "null batch"; }

extern "C" void *dns2d_batch_stream(dns2d_batch *b) { return b ? (void *)b->stream : nullptr; }

extern "C" int dns2d_batch_create(dns2d_batch **out, const dns2d_member *members, int count, int device)
{
    if (!out || !members || count <= 0) return DNS2D_ERR_ARG;
    *out = nullptr;
    for (int i = 0; i < count; ++i)
        if (!kernel_set(members[i].N)) return DNS2D_ERR_SIZE;
    dns2d_batch *b = new dns2d_batch();
    b->count = count;
    b->device = device;
    auto bail = [&](int rc) {
        dns2d_batch_destroy(b);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaEventCreateWithFlags(&b->prm_copied, cudaEventDisableTiming) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    b->sc.resize((size_t)count);
    b->where.resize((size_t)count);
    for (int i = 0; i < count; ++i) {
        const dns2d_member &m = members[i];
        int gi = -1;
        for (size_t k = 0; k < b->groups.size(); ++k)
            if (b->groups[k].N == m.N) gi = (int)k;
        if (gi < 0) {
            BatchGroup g;
            g.N = m.N;
            g.H = m.N / 2;
            g.L = 3 * m.N / 2;
            g.ks = kernel_set(m.N);
            g.tune = tuning_for(device, m.N);
            b->groups.push_back(g);
            gi = (int)b->groups.size() - 1;
        }
        BatchGroup &g = b->groups[(size_t)gi];
        b->where[(size_t)i] = {gi, g.count};
        g.members.push_back(i);
        g.count += 1;
        MemberScalars &c = b->sc[(size_t)i];
        c = MemberScalars{m.Re, m.K0, float(1.0 / m.Re), 0.0f, 0.0f, 1.0f, 0.0f, m.cflnum, 0.0f, 0, 1, m.seed};
    }
    for (BatchGroup &g : b->groups) {
        if (g.ks->setup() != cudaSuccess) return bail(DNS2D_ERR_CUDA);
        const size_t H = g.H, L = g.L, nom = (size_t)g.N * H, c = (size_t)g.count;
        auto dalloc = [&](void **p, size_t bytes) { return cudaMalloc(p, bytes) == cudaSuccess; };
        if (!dalloc((void **)&g.om2, c * nom * 8) || !dalloc((void **)&g.fnm1, c * nom * 8) ||
            !dalloc((void **)&g.work, c * 2 * L * H * 8) ||
            !dalloc((void **)&g.tw, (size_t)std::max(g.ks->cat->total, 1) * 8) ||
            !dalloc((void **)&g.prm, c * sizeof(StepParams)) || !dalloc((void **)&g.part, c * H * 16) ||
            !dalloc((void **)&g.hist, c * kChunk * 16) || !dalloc((void **)&g.counter, c * 4) ||
            !dalloc((void **)&g.cflm, c * 4)) {
            cudaGetLastError();
            return bail(DNS2D_ERR_NOMEM);
        }
        std::vector<float2> tw = twiddles(*g.ks->cat);
        if (cudaMemcpy(g.tw, tw.data(), tw.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(g.counter, 0, c * 4) != cudaSuccess || cudaMemset(g.fnm1, 0, c * nom * 8) != cudaSuccess)
            return bail(DNS2D_ERR_CUDA);
    }
    if (cudaMallocHost((void **)&b->prm_host, (size_t)count * sizeof(StepParams)) != cudaSuccess ||
        cudaMallocHost((void **)&b->hist_host, (size_t)count * kChunk * 16) != cudaSuccess ||
        cudaMallocHost((void **)&b->cflm_host, (size_t)count * 4) != cudaSuccess ||
        cudaMallocHost((void **)&b->ens_status_host, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&b->ens, (size_t)(2 + 2 * count) * 4) != cudaSuccess)
        return bail(DNS2D_ERR_NOMEM);
    if (b->groups.size() > 1) {
        if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
        b->side.assign(b->groups.size(), nullptr);
        b->joins.assign(b->groups.size(), nullptr);
        for (size_t i = 0; i < b->groups.size(); ++i)
            if (cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming) != cudaSuccess)
                return bail(DNS2D_ERR_CUDA);
    }
    *out = b;
    return DNS2D_OK;
}

extern "C" int dns2d_batch_init_vorticity(dns2d_batch *b, int member, const float *om2)
{
    if (!b || !om2 || member < 0 || member >= b->count) return DNS2D_ERR_ARG;
    const auto [gi, k] = b->where[(size_t)member];
    BatchGroup &g = b->groups[(size_t)gi];
    const size_t nom = (size_t)g.N * g.H;
    float2 *stage = g.work + (size_t)k * 2 * g.L * g.H;  // the member's work buffer as staging
    BATCH_CUDA(cudaMemcpyAsync(stage, om2, nom * 8, cudaMemcpyHostToDevice, b->stream), "om2 upload");
    dim3 tb(32, 8), tg((g.H + 31) / 32, (g.N + 31) / 32);
    k_transpose_c64<<<tg, tb, 0, b->stream>>>(stage, g.om2 + (size_t)k * nom, g.N, g.H);
    BATCH_CUDA(cudaGetLastError(), "transpose");
    BATCH_CUDA(cudaMemsetAsync(g.fnm1 + (size_t)k * nom, 0, nom * 8, b->stream), "fnm1 clear");
    MemberScalars &c = b->sc[(size_t)member];
    c.it = 0;
    c.t = 0.0f;
    c.dt = 0.0f;
    c.cn = 1.0f;
    c.cnm1 = 0.0f;
    c.visc = float(1.0 / c.Re);
    BATCH_CUDA(cudaStreamSynchronize(b->stream), "vorticity upload");
    return DNS2D_OK;
}

// velocity of every member from its vorticity (after the vorticity uploads)
static int batch_velocity(dns2d_batch *b)
{
    for (BatchGroup &g : b->groups) g.ks->cols_init(g.ptrs(), nullptr, 1, b->stream, g.count);
    BATCH_CUDA(cudaGetLastError(), "cols_init(batch)");
    BATCH_CUDA(cudaStreamSynchronize(b->stream), "batch velocity");
    b->initialised = true;
    return DNS2D_OK;
}

// Autotuner for a batch: each size group's kernel variants timed with the group's own member
// count on the batch's own buffers.  Call before the initial fields are set (the timing runs
// the passes on the buffers); every variant computes the same arithmetic.
extern "C" int dns2d_batch_autotune(dns2d_batch *b)
{
    if (!b) return DNS2D_ERR_ARG;
    if (b->initialised) return DNS2D_ERR_STATE;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        return DNS2D_ERR_CUDA;
    }
    auto timed = [&](auto fn, int reps) {
        for (int i = 0; i < 2; ++i) fn();
        cudaEventRecord(e0, b->stream);
        for (int i = 0; i < reps; ++i) fn();
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / (float)reps;
    };
    for (BatchGroup &g : b->groups) {
        if (cluster_size(g.N)) continue;
        const int reps = g.N >= 2048 ? 10 : 50;
        Tuning best = g.tune;
        float tb = 1e30f;
        if (g.N >= 1024) {
            for (int pf : {0, 148, 296, 444, 592}) {
                g.tune = best;
                g.tune.pf_rows = pf;
                const Pointers p = g.ptrs();
                const float t = timed([&] { g.ks->rows_step(p, b->stream, g.count); }, reps);
                if (t < tb) tb = t, best.pf_rows = pf;
            }
            tb = 1e30f;
            for (int gr : {1, 2})
                for (int pf : {0, 37, 74, 148}) {
                    g.tune = best;
                    g.tune.cols_groups = gr;
                    g.tune.pf_cols = pf;
                    const Pointers p = g.ptrs();
                    const float t = timed([&] { g.ks->cols_step(p, 0, 0, b->stream, g.count); }, reps);
                    if (t < tb) tb = t, best.cols_groups = gr, best.pf_cols = pf;
                }
        } else {
            best = tune_small(g.ks->nplans, best, [&](const Tuning &t, bool rows) {
                g.tune = t;
                const Pointers p = g.ptrs();
                if (rows) return timed([&] { g.ks->rows_step(p, b->stream, g.count); }, reps);
                return timed([&] { g.ks->cols_step(p, 0, 0, b->stream, g.count); }, reps);
            });
        }
        g.tune = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the buffers hold timing leftovers: clear them as at creation
    for (BatchGroup &g : b->groups) {
        const size_t nom = (size_t)g.count * g.N * g.H, nwork = (size_t)g.count * 2 * g.L * g.H;
        if (cudaMemsetAsync(g.om2, 0, nom * 8, b->stream) != cudaSuccess ||
            cudaMemsetAsync(g.fnm1, 0, nom * 8, b->stream) != cudaSuccess ||
            cudaMemsetAsync(g.work, 0, nwork * 8, b->stream) != cudaSuccess)
            return DNS2D_ERR_CUDA;
    }
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    return cudaStreamSynchronize(b->stream) == cudaSuccess ? DNS2D_OK : DNS2D_ERR_CUDA;
}

extern "C" int dns2d_batch_init_k4(dns2d_batch *b)
{
    if (!b) return DNS2D_ERR_ARG;
    for (int i = 0; i < b->count; ++i) {
        const auto [gi, k] = b->where[(size_t)i];
        const int N = b->groups[(size_t)gi].N;
        std::vector<float> om((size_t)N * (N / 2) * 2);
        dns2d_k4_spectrum(N, b->sc[(size_t)i].K0, b->sc[(size_t)i].seed, om.data());
        int rc = dns2d_batch_init_vorticity(b, i, om.data());
        if (rc) return rc;
    }
    return batch_velocity(b);
}

extern "C" int dns2d_batch_next_dt(dns2d_batch *b, float *cflm_out)
{
    if (!b) return DNS2D_ERR_ARG;
    if (!b->initialised) return bfail(b, DNS2D_ERR_STATE, "no initial condition");
    for (BatchGroup &g : b->groups) {
        BATCH_CUDA(cudaMemsetAsync(g.cflm, 0, (size_t)g.count * 4, b->stream), "cflm clear");
        const float DX = 2.0f * 3.14159265358979323846f / float(g.N);
        g.ks->rows_velocity(g.ptrs(), nullptr, g.cflm, DX, b->stream, g.count);
        BATCH_CUDA(cudaGetLastError(), "rows_velocity(batch)");
    }
    int off = 0;
    for (BatchGroup &g : b->groups) {
        BATCH_CUDA(cudaMemcpyAsync(b->cflm_host + off, g.cflm, (size_t)g.count * 4, cudaMemcpyDeviceToHost, b->stream),
                   "cflm copy");
        off += g.count;
    }
    BATCH_CUDA(cudaStreamSynchronize(b->stream), "cflm sync");
    const float PI = 3.14159265358979323846f;
    off = 0;
    for (BatchGroup &g : b->groups) {
        for (int k = 0; k < g.count; ++k) {
            MemberScalars &c = b->sc[(size_t)g.members[(size_t)k]];
            const float CFLM = b->cflm_host[off + k];
            if (c.it == 0 && c.dt == 0.0f) {  // NEXTDT init branch (cuda/dns_cuda.cu:562-569)
                c.dt = c.cflnum / CFLM / PI;
                c.cflm = CFLM;
            } else if (c.ifn > 0 && (c.it % c.ifn) == 0) {  // regular update (:572-579)
                const float CFL = CFLM * c.dt * PI;
                c.cn = 0.8f + 0.2f * (c.cflnum / CFL);
                c.dt = c.dt * c.cn;
                c.cflm = CFLM;
            }
            if (cflm_out) cflm_out[g.members[(size_t)k]] = c.cflm;
        }
        off += g.count;
    }
    return DNS2D_OK;
}

namespace {

// the instantiated graph of a chunk of K steps (first: the chunk opens a dns2d_batch_step call),
// captured on first use: every size group's step chain as its own branch
int batch_graph(dns2d_batch *b, int first, int K, cudaGraphExec_t *out)
{
    const auto key = std::make_pair(first, K);
    const auto itg = b->graphs.find(key);
    if (itg != b->graphs.end()) {
        *out = itg->second;
        return DNS2D_OK;
    }
    cudaGraph_t gr = nullptr;
    BATCH_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    const bool par = !b->side.empty();
    // a failure inside the capture still ends it (the stream leaves capture mode)
    cudaError_t ce = par ? cudaEventRecord(b->fork, b->stream) : cudaSuccess;
    for (size_t gi = 0; gi < b->groups.size() && ce == cudaSuccess; ++gi) {
        BatchGroup &g = b->groups[gi];
        cudaStream_t q = par ? b->side[gi] : b->stream;
        if (par) ce = cudaStreamWaitEvent(q, b->fork, 0);
        for (int i = 0; i < K && ce == cudaSuccess; ++i) {
            g.ks->rows_step(g.ptrs(), q, g.count);
            g.ks->cols_step(g.ptrs(), (first && i == 0) ? 1 : 0, i, q, g.count);
        }
        if (par && ce == cudaSuccess) ce = cudaEventRecord(b->joins[gi], q);
        if (par && ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->joins[gi], 0);
    }
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &gr);
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (gr) cudaGraphDestroy(gr);
        return bfail(b, DNS2D_ERR_CUDA, "graph capture", ce != cudaSuccess ? ce : ee);
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return bfail(b, DNS2D_ERR_CUDA, "graph instantiate", e);
    b->graphs[key] = ex;
    *out = ex;
    return DNS2D_OK;
}

}  // namespace

namespace {

int ens_cols_per_item_of(int N)
{
    switch (N) {
    case 64: return ens_cols_per_item<64>();
    case 128: return ens_cols_per_item<128>();
    case 256: return ens_cols_per_item<256>();
    default: return ens_cols_per_item<512>();
    }
}

bool ens_batch_supported(const dns2d_batch *b)
{
    if (b->groups.size() > (size_t)kEnsMaxGroups) return false;
    for (const BatchGroup &g : b->groups)
        if (!ens_supported(g.N)) return false;
    return true;
}

// K steps of every member in one persistent launch (first: the chunk opens a dns2d_batch_step call)
int ens_chunk(dns2d_batch *b, int first, int K)
{
    EnsLaunch q;
    q.ngroups = (int)b->groups.size();
    q.steps = K;
    q.first = first;
    int member = 0;
    for (size_t i = 0; i < b->groups.size(); ++i) {
        const BatchGroup &g = b->groups[i];
        EnsGroupDev &d = q.g[i];
        d.N = g.N;
        d.count = g.count;
        d.member0 = member;
        // a few row tiles / column groups per item, so the per-item ticket, wait and completion
        // count are spread over more work (the items of the small sizes are tiny)
        const int tiles = g.L / kEnsRows, groups = g.H / ens_cols_per_item_of(g.N);
        d.tiles_per_item = b->tiles_per_item;
        while (tiles % d.tiles_per_item) d.tiles_per_item /= 2;
        d.groups_per_item = b->groups_per_item;
        while (groups % d.groups_per_item) d.groups_per_item /= 2;
        d.row_items = tiles / d.tiles_per_item;
        d.col_items = groups / d.groups_per_item;
        d.row_begin = q.rows_per_step;
        d.col_begin = q.cols_per_step;
        d.p = g.ptrs();
        q.rows_per_step += g.count * d.row_items;
        q.cols_per_step += g.count * d.col_items;
        member += g.count;
    }
    q.ticket = b->ens;
    q.rows_done = b->ens + 1;
    q.cols_done = b->ens + 1 + b->count;
    q.status = reinterpret_cast<int *>(b->ens + 1 + 2 * b->count);
    q.spin_limit = b->spin_limit;
    q.stall_member = b->stall_member;
    BATCH_CUDA(cudaMemsetAsync(b->ens, 0, (size_t)(2 + 2 * b->count) * 4, b->stream), "counter reset");
    BATCH_CUDA(ens_launch(q, b->stream, &b->ens_grid), "persistent ensemble launch");
    return DNS2D_OK;
}

}  // namespace

extern "C" int dns2d_batch_set_mode(dns2d_batch *b, int mode)
{
    if (!b || mode < 0 || mode > 1) return DNS2D_ERR_ARG;
    if (mode == 1 && !ens_batch_supported(b))
        return bfail(b, DNS2D_ERR_SIZE, "persistent launch: sizes 64, 128, 256, 512 and at most 8 size groups");
    b->mode = mode;
    return DNS2D_OK;
}

extern "C" int dns2d_batch_set_items(dns2d_batch *b, int tiles_per_item, int groups_per_item)
{
    auto pow2 = [](int v) { return v >= 1 && v <= 64 && (v & (v - 1)) == 0; };
    if (!b || !pow2(tiles_per_item) || !pow2(groups_per_item)) return DNS2D_ERR_ARG;
    b->tiles_per_item = tiles_per_item;
    b->groups_per_item = groups_per_item;
    return DNS2D_OK;
}

extern "C" int dns2d_batch_set_waits(dns2d_batch *b, long long spin_limit, int stall_member)
{
    if (!b || spin_limit < 1 || stall_member >= b->count) return DNS2D_ERR_ARG;
    b->spin_limit = spin_limit;
    b->stall_member = stall_member;
    return DNS2D_OK;
}

extern "C" int dns2d_batch_prepare(dns2d_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return DNS2D_ERR_ARG;
    for (int done = 0; done < nsteps;) {
        const int K = std::min(kChunk, nsteps - done);
        cudaGraphExec_t ex = nullptr;
        const int rc = batch_graph(b, done == 0 ? 1 : 0, K, &ex);
        if (rc) return rc;
        done += K;
    }
    return DNS2D_OK;
}

extern "C" int dns2d_batch_step(dns2d_batch *b, int nsteps, double *E_hist, double *Z_hist)
{
    if (!b || nsteps < 0) return DNS2D_ERR_ARG;
    if (!b->initialised) return bfail(b, DNS2D_ERR_STATE, "no initial condition");
    // parameter blocks of every member (group order), copied once per call
    BATCH_CUDA(cudaEventSynchronize(b->prm_copied), "parameter buffer");
    int off = 0;
    for (BatchGroup &g : b->groups) {
        for (int k = 0; k < g.count; ++k) {
            const MemberScalars &c = b->sc[(size_t)g.members[(size_t)k]];
            b->prm_host[off + k] = StepParams{c.dt, c.cnm1, c.cn, c.visc};
        }
        BATCH_CUDA(cudaMemcpyAsync(g.prm, b->prm_host + off, (size_t)g.count * sizeof(StepParams),
                                   cudaMemcpyHostToDevice, b->stream),
                   "parameter copy");
        off += g.count;
    }
    BATCH_CUDA(cudaEventRecord(b->prm_copied, b->stream), "parameter event");
    int done = 0;
    while (done < nsteps) {
        const int K = std::min(kChunk, nsteps - done);
        const int first = (done == 0) ? 1 : 0;
        if (b->mode == 1) {
            const int rc = ens_chunk(b, first, K);
            if (rc) return rc;
        } else {
            cudaGraphExec_t ex = nullptr;
            const int rc = batch_graph(b, first, K, &ex);
            if (rc) return rc;
            BATCH_CUDA(cudaGraphLaunch(ex, b->stream), "graph launch");
        }
        if (b->mode == 1) {
            // the launch's status: a dependency wait that ran out stops every CTA
            BATCH_CUDA(cudaMemcpyAsync(b->ens_status_host, b->ens + 1 + 2 * b->count, sizeof(int),
                                       cudaMemcpyDeviceToHost, b->stream),
                       "status copy");
            BATCH_CUDA(cudaStreamSynchronize(b->stream), "status sync");
            if (*b->ens_status_host != 0)
                return bfail(b, DNS2D_ERR_TIMEOUT, "persistent ensemble launch: a dependency wait ran out");
        }
        if (E_hist || Z_hist) {
            off = 0;
            for (BatchGroup &g : b->groups) {
                BATCH_CUDA(cudaMemcpyAsync(b->hist_host + (size_t)off * kChunk, g.hist, (size_t)g.count * kChunk * 16,
                                           cudaMemcpyDeviceToHost, b->stream),
                           "history copy");
                off += g.count;
            }
            BATCH_CUDA(cudaStreamSynchronize(b->stream), "history sync");
            off = 0;
            for (BatchGroup &g : b->groups) {
                for (int k = 0; k < g.count; ++k) {
                    const int m = g.members[(size_t)k];
                    for (int i = 0; i < K; ++i) {
                        const double2 v = b->hist_host[(size_t)(off + k) * kChunk + i];
                        if (E_hist) E_hist[(size_t)m * nsteps + done + i] = v.x;
                        if (Z_hist) Z_hist[(size_t)m * nsteps + done + i] = v.y;
                    }
                }
                off += g.count;
            }
        }
        for (MemberScalars &c : b->sc)
            for (int i = 0; i < K; ++i) {
                c.it += 1;
                const float dt_old = c.dt;
                c.cnm1 = c.cn;
                c.t += dt_old;
            }
        done += K;
    }
    return DNS2D_OK;
}

extern "C" int dns2d_batch_sync(dns2d_batch *b)
{
    if (!b) return DNS2D_ERR_ARG;
    BATCH_CUDA(cudaStreamSynchronize(b->stream), "sync");
    return DNS2D_OK;
}

extern "C" int dns2d_batch_get_om2(dns2d_batch *b, int member, float *om2)
{
    if (!b || !om2 || member < 0 || member >= b->count) return DNS2D_ERR_ARG;
    const auto [gi, k] = b->where[(size_t)member];
    BatchGroup &g = b->groups[(size_t)gi];
    const size_t nom = (size_t)g.N * g.H;
    float2 *stage = nullptr;
    BATCH_CUDA(cudaMallocAsync((void **)&stage, nom * 8, b->stream), "staging");
    dim3 tb(32, 8), tg((g.N + 31) / 32, (g.H + 31) / 32);
    k_transpose_c64<<<tg, tb, 0, b->stream>>>(g.om2 + (size_t)k * nom, stage, g.H, g.N);
    BATCH_CUDA(cudaGetLastError(), "transpose");
    BATCH_CUDA(cudaMemcpyAsync(om2, stage, nom * 8, cudaMemcpyDeviceToHost, b->stream), "om2 copy");
    BATCH_CUDA(cudaFreeAsync(stage, b->stream), "staging free");
    BATCH_CUDA(cudaStreamSynchronize(b->stream), "om2 sync");
    return DNS2D_OK;
}

extern "C" int dns2d_batch_get_scalars(dns2d_batch *b, int member, dns2d_scalars *o)
{
    if (!b || !o || member < 0 || member >= b->count) return DNS2D_ERR_ARG;
    const auto [gi, k] = b->where[(size_t)member];
    (void)k;
    const BatchGroup &g = b->groups[(size_t)gi];
    const MemberScalars &c = b->sc[(size_t)member];
    o->N = g.N;
    o->NX_full = g.L;
    o->NK_full = 3 * g.N / 4 + 1;
    o->it = c.it;
    o->ifn = c.ifn;
    o->Re = c.Re;
    o->K0 = c.K0;
    o->visc = c.visc;
    o->t = c.t;
    o->dt = c.dt;
    o->cn = c.cn;
    o->cnm1 = c.cnm1;
    o->cflnum = c.cflnum;
    o->cflm = c.cflm;
    return DNS2D_OK;
}

// ============================================================================================
// Learned-closure network (cnn.cuh): parameters, activations, dataset and Adam state on the
// device; forward / backward / training driven from here.
// ============================================================================================
// Autotuner: times the kernel variants of one size on a scratch state (k^4 field) and keeps
// the fastest per (device, N).  The variants differ in rows per CTA (small grids), thread groups
// per column CTA and L2 prefetch distances (large grids) and compute the same arithmetic, so a
// tuned run gives the same results as an untuned one.  States and batches created afterwards on
// that device use the choice; DNS2D_AUTOTUNE=1 in the environment tunes at dns2d_create.
// ============================================================================================
namespace {
// mean ms of one launch of fn over reps launches (after 2 warm-up launches) on the state's stream
template <class F>
float time_launches(dns2d_state *s, int reps, F fn)
{
    for (int i = 0; i < 2; ++i) fn();
    cudaEventRecord(s->ev0, s->stream);
    for (int i = 0; i < reps; ++i) fn();
    cudaEventRecord(s->ev1, s->stream);
    cudaEventSynchronize(s->ev1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->ev0, s->ev1);
    return ms / (float)reps;
}
}  // namespace

extern "C" int dns2d_set_tuning(int N, int device, const int *config)
{
    const KernelSet *ks = kernel_set(N);
    if (!ks || !config) return DNS2D_ERR_ARG;
    if (!(config[0] == 0 || config[0] == 2 || config[0] == 4 || config[0] == 8) || config[1] < 0 || config[1] > 2 ||
        config[2] < 0 || config[3] < 0 || config[4] < 0 || config[4] >= ks->nplans || config[5] < 0 ||
        config[5] >= ks->nplans)
        return DNS2D_ERR_ARG;
    Tuning t;
    t.rows_tile = config[0];
    t.cols_groups = config[1];
    t.pf_rows = config[2];
    t.pf_cols = config[3];
    t.plan_rows = config[4];
    t.plan_cols = config[5];
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{device, N}] = t;
    return DNS2D_OK;
}

extern "C" int dns2d_autotune(int N, int device, int *config)
{
    const KernelSet *ks = kernel_set(N);
    if (!ks) return DNS2D_ERR_SIZE;
    Tuning best;
    if (!cluster_size(N)) {  // the cluster sizes have a single configuration
        t_in_autotune = true;
        dns2d_state *s = nullptr;
        int rc = dns2d_create(&s, N, 1.0e5f, 4.0f, 0.1f, device);
        if (!rc) rc = dns2d_init_k4(s, 1);
        if (!rc) rc = dns2d_next_dt(s, nullptr);
        if (!rc) rc = dns2d_step(s, 1, nullptr, nullptr);
        if (!rc) rc = dns2d_sync(s, 0);
        t_in_autotune = false;
        if (rc) {
            dns2d_destroy(s);
            return rc;
        }
        const int reps = N >= 2048 ? 20 : 100;
        const bool large = N >= 1024;
        float tb = 1e30f;
        if (large) {
            for (int pf : {0, 148, 296, 444, 592}) {
                s->tune = best;
                s->tune.pf_rows = pf;
                const Pointers p = s->ptrs();
                const float t = time_launches(s, reps, [&] { ks->rows_step(p, s->stream, 1); });
                if (t < tb) tb = t, best.pf_rows = pf;
            }
            tb = 1e30f;
            for (int g : {1, 2})
                for (int pf : {0, 37, 74, 148}) {
                    s->tune = best;
                    s->tune.cols_groups = g;
                    s->tune.pf_cols = pf;
                    const Pointers p = s->ptrs();
                    const float t = time_launches(s, reps, [&] { ks->cols_step(p, 0, 0, s->stream, 1); });
                    if (t < tb) tb = t, best.cols_groups = g, best.pf_cols = pf;
                }
        } else {
            best = tune_small(ks->nplans, best, [&](const Tuning &t, bool rows) {
                s->tune = t;
                const Pointers p = s->ptrs();
                if (rows) return time_launches(s, reps, [&] { ks->rows_step(p, s->stream, 1); });
                return time_launches(s, reps, [&] { ks->cols_step(p, 0, 0, s->stream, 1); });
            });
        }
        const cudaError_t e = cudaStreamSynchronize(s->stream);
        dns2d_destroy(s);
        if (e != cudaSuccess) return DNS2D_ERR_CUDA;
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[{device, N}] = best;
    }
    if (config) {
        config[0] = best.rows_tile;
        config[1] = best.cols_groups;
        config[2] = best.pf_rows;
        config[3] = best.pf_cols;
        config[4] = best.plan_rows;
        config[5] = best.plan_cols;
    }
    return DNS2D_OK;
}

// ============================================================================================
struct dns2d_cnn {
    int layers = 0, channels = 0, device = 0, nparams = 0;
    std::vector<int> ci, co;       // per layer
    std::vector<size_t> woff;      // weight offset per layer (bias follows the weights)
    cudaStream_t stream = nullptr;
    float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr, *wflip = nullptr, *zero = nullptr;
    std::vector<float *> z, a;     // pre-activations / activations per layer (capacity cap_elems each)
    float *xin = nullptr, *tgt = nullptr, *gout = nullptr, *gtmp = nullptr;
    size_t cap_elems = 0;          // per activation tensor: B * max(C, 3) * H * W
    int capB = 0, capH = 0, capW = 0;
    double *part = nullptr;
    long long step = 0;
    float *data_x = nullptr, *data_t = nullptr;  // device-resident training set
    int data_n = 0, data_H = 0, data_W = 0;
    // BF16 tensor-core inference path (cnn_tc.cuh, cnn_net.cuh): packed weights, padded
    // chunk-planar bf16 activations, error flag of the bounded waits; gen counts parameter
    // changes.  tc_mode 1 runs layers 1 .. L-1 as one persistent launch where their weights fit
    // in shared memory (net_sync: its ticket and row counters), 0 one launch per layer.
    __nv_bfloat16 *wtc = nullptr;
    __nv_bfloat16 *act_tc[2] = {nullptr, nullptr};
    size_t act_tc_cap = 0;  // bytes of each activation buffer
    int *tc_err = nullptr;
    unsigned int *net_sync = nullptr;
    size_t net_sync_cap = 0;  // words
    int tc_mode = 1, net_grid = 0;
    // optional per-tile timestamps of the persistent launch (8 per tile, the last launch's)
    unsigned long long *trace = nullptr;
    size_t trace_cap = 0;  // tiles
    int trace_on = 0, trace_tiles = 0;
    // training convolutions as tcgen05 GEMMs (cnn_gemm.cuh) when train_tc is set
    dns2d::cnngemm::Work gw;
    int train_tc = 0;
    long long gen = 0, tc_gen = -1;
    std::string err;
};

namespace {

int nfail(dns2d_cnn *n, int code, const char *what, cudaError_t e = cudaSuccess)
{
    if (n) n->err = std::string(what) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return code;
}

#define CNN_CUDA(call, what)                                                     \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) return nfail(n, DNS2D_ERR_CUDA, what, e_);        \
    } while (0)

uint64_t sm64(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int cnn_reserve(dns2d_cnn *n, int B, int H, int W)
{
    if (B <= n->capB && H == n->capH && W == n->capW) return DNS2D_OK;
    CNN_CUDA(cudaStreamSynchronize(n->stream), "sync");
    for (float *p : n->z) cudaFree(p);
    for (float *p : n->a) cudaFree(p);
    cudaFree(n->xin);
    cudaFree(n->tgt);
    cudaFree(n->gout);
    cudaFree(n->gtmp);
    n->z.assign(n->layers, nullptr);
    n->a.assign(n->layers, nullptr);
    const size_t cap = (size_t)B * std::max(n->channels, 3) * H * W;
    for (int l = 0; l < n->layers; ++l) {
        CNN_CUDA(cudaMalloc((void **)&n->z[l], cap * 4), "activation alloc");
        CNN_CUDA(cudaMalloc((void **)&n->a[l], cap * 4), "activation alloc");
    }
    CNN_CUDA(cudaMalloc((void **)&n->xin, (size_t)B * 3 * H * W * 4), "input alloc");
    CNN_CUDA(cudaMalloc((void **)&n->tgt, (size_t)B * H * W * 4), "target alloc");
    CNN_CUDA(cudaMalloc((void **)&n->gout, cap * 4), "grad alloc");
    CNN_CUDA(cudaMalloc((void **)&n->gtmp, cap * 4), "grad alloc");
    n->cap_elems = cap;
    n->capB = B;
    n->capH = H;
    n->capW = W;
    return DNS2D_OK;
}

void conv(dns2d_cnn *n, const float *x, const float *w, const float *b, float *y, int B, int Ci, int Co, int H, int W,
          cudaStream_t st)
{
    using namespace dns2d::cnn;
    dim3 grid((W + TILE - 1) / TILE, (H + TILE - 1) / TILE, B * ((Co + COT - 1) / COT));
    const size_t sm = ((size_t)Ci * (TILE + 2) * (TILE + 2) + (size_t)COT * Ci * 9) * 4;
    k_conv3x3<<<grid, dim3(TILE, TILE), sm, st>>>(x, w, b, y, B, Ci, Co, H, W);
}

// forward of B images in n->xin; output (layer L-1 pre-activation) in n->z[L-1]
int cnn_forward_dev(dns2d_cnn *n, int B, int H, int W, cudaStream_t st = nullptr)
{
    if (!st) st = n->stream;
    const float *in = n->xin;
    if (n->train_tc) {  // every layer as a tcgen05 GEMM (bf16 operands, FP32 accumulation)
        for (int l = 0; l < n->layers; ++l) {
            const float *w = n->params + n->woff[l], *bias = w + (size_t)n->co[l] * n->ci[l] * 9;
            CNN_CUDA(dns2d::cnngemm::conv_fwd(in, n->ci[l], w, bias, n->co[l], n->z[l],
                                              l + 1 < n->layers ? n->a[l] : nullptr, B, H, W, n->gw, st),
                     "tensor-core forward");
            in = n->a[l];
        }
        return DNS2D_OK;
    }
    for (int l = 0; l < n->layers; ++l) {
        conv(n, in, n->params + n->woff[l], n->params + n->woff[l] + (size_t)n->co[l] * n->ci[l] * 9, n->z[l], B,
             n->ci[l], n->co[l], H, W, st);
        if (l + 1 < n->layers) {
            const size_t cnt = (size_t)B * n->co[l] * H * W;
            dns2d::cnn::k_gelu<<<1024, 256, 0, st>>>(n->z[l], n->a[l], cnt);
            in = n->a[l];
        }
    }
    CNN_CUDA(cudaGetLastError(), "cnn forward");
    return DNS2D_OK;
}

// BF16 tensor-core forward: hidden layers 32 -> 32 on tcgen05 (W a multiple of 128)
bool cnn_tc_supported(const dns2d_cnn *n, int H, int W)
{
    return n->channels == dns2d::cnntc::C && n->layers >= 3 && W % dns2d::cnntc::TM == 0 && H % dns2d::cnntc::TR == 0;
}

int cnn_tc_reserve(dns2d_cnn *n, int B, int H, int W)
{
    const size_t need = dns2d::cnntc::act_bytes(B, H, W);
    CNN_CUDA(cudaFuncSetAttribute(dns2d::cnntc::k_conv_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  dns2d::cnntc::TcShape<32>::SMEM_BYTES),
             "tc smem attribute");
    CNN_CUDA(cudaFuncSetAttribute(dns2d::cnntc::k_conv_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  dns2d::cnntc::TcShape<16>::SMEM_BYTES),
             "tc smem attribute");
    // hidden layers [tap][chunk][32][8], the last layer [tap][chunk][16][8], the first [chunk][32][8]
    if (!n->wtc)
        CNN_CUDA(cudaMalloc((void **)&n->wtc,
                            ((size_t)(n->layers - 2) * 9 * 4 * 32 * 8 + 9 * 4 * 16 * 8 + 4 * 32 * 8) * 2),
                 "tc weights alloc");
    if (!n->tc_err) {
        CNN_CUDA(cudaMalloc((void **)&n->tc_err, 4), "tc flag alloc");
        CNN_CUDA(cudaMemset(n->tc_err, 0, 4), "tc flag clear");
    }
    if (need > n->act_tc_cap) {
        CNN_CUDA(cudaStreamSynchronize(n->stream), "sync");
        cudaFree(n->act_tc[0]);
        cudaFree(n->act_tc[1]);
        n->act_tc[0] = n->act_tc[1] = nullptr;
        CNN_CUDA(cudaMalloc((void **)&n->act_tc[0], need), "tc activation alloc");
        CNN_CUDA(cudaMalloc((void **)&n->act_tc[1], need), "tc activation alloc");
        n->act_tc_cap = need;
    }
    // counters of the persistent launch: zero once, then reset by each launch's last CTA
    const size_t words = dns2d::cnntc::net_sync_words(n->layers, B, H);
    if (words > n->net_sync_cap) {
        CNN_CUDA(cudaStreamSynchronize(n->stream), "sync");
        cudaFree(n->net_sync);
    cudaFree(n->trace);
    dns2d::cnngemm::work_free(n->gw);
        n->net_sync = nullptr;
        CNN_CUDA(cudaMalloc((void **)&n->net_sync, words * 4), "network counters alloc");
        CNN_CUDA(cudaMemset(n->net_sync, 0, words * 4), "network counters clear");
        n->net_sync_cap = words;
    }
    return DNS2D_OK;
}

// packed bf16 weights follow the parameters (repacked after set_params / train)
int cnn_tc_prepare(dns2d_cnn *n, cudaStream_t st)
{
    if (n->tc_gen == n->gen) return DNS2D_OK;
    for (int l = 1; l + 1 < n->layers; ++l)
        dns2d::cnntc::k_pack_weights<32><<<36, 256, 0, st>>>(n->params + n->woff[l], 32,
                                                             n->wtc + (size_t)(l - 1) * 9 * 32 * 32);
    dns2d::cnntc::k_pack_weights<16><<<18, 256, 0, st>>>(n->params + n->woff[n->layers - 1], 1,
                                                         n->wtc + (size_t)(n->layers - 2) * 9 * 32 * 32);
    dns2d::cnntc::k_pack_first<<<1, 256, 0, st>>>(n->params + n->woff[0],
                                                  n->wtc + (size_t)(n->layers - 2) * 9 * 32 * 32 + 9 * 4 * 16 * 8);
    CNN_CUDA(cudaGetLastError(), "tc weight pack");
    n->tc_gen = n->gen;
    return DNS2D_OK;
}

// inputs: three f32 planes times their scales; output: the last layer times out_scale in n->z[L-1]
int cnn_forward_tc_dev(dns2d_cnn *n, int B, int H, int W, const dns2d::cnntc::FirstIn &in, float out_scale,
                       cudaStream_t st)
{
    using namespace dns2d::cnntc;
    const int L = n->layers;
    const dim3 grid((W / TM) * (H / TR), B);
    const __nv_bfloat16 *w_last = n->wtc + (size_t)(L - 2) * 9 * 32 * 32;
    const __nv_bfloat16 *w_first = w_last + 9 * 4 * 16 * 8;
    k_conv_tc_first<<<grid, NT_FIRST, SMEM_FIRST, st>>>(in, w_first, n->params + n->woff[0] + (size_t)n->co[0] * n->ci[0] * 9,
                                                  n->act_tc[0], H, W, n->tc_err);
    const int stages = n->tc_mode == 1 ? net_stages_that_fit(L) : 0;
    if (stages >= 2) {
        NetLaunch q;
        q.wtc = n->wtc;
        for (int l = 1; l < L; ++l) q.bias[l] = n->params + n->woff[l] + (size_t)n->co[l] * n->ci[l] * 9;
        q.act[0] = n->act_tc[0];
        q.act[1] = n->act_tc[1];
        q.yf = n->z[L - 1];
        q.out_scale = out_scale;
        q.L = L;
        q.B = B;
        q.H = H;
        q.W = W;
        q.stages = stages;
        q.sync = n->net_sync;
        q.err = n->tc_err;
        if (n->trace_on) {
            const size_t tiles = (size_t)(L - 1) * B * (H / TR) * (W / TM);
            if (tiles > n->trace_cap) {
                CNN_CUDA(cudaStreamSynchronize(st), "sync");
                cudaFree(n->trace);
                n->trace = nullptr;
                CNN_CUDA(cudaMalloc((void **)&n->trace, tiles * kNetTraceSlots * sizeof(unsigned long long)),
                         "trace alloc");
                n->trace_cap = tiles;
            }
            q.trace = n->trace;
            n->trace_tiles = (int)tiles;
        }
        CNN_CUDA(net_launch(q, st, &n->net_grid), "persistent network launch");
        return DNS2D_OK;
    }
    int cur = 0;
    for (int l = 1; l + 1 < L; ++l) {
        const float *bias = n->params + n->woff[l] + (size_t)n->co[l] * n->ci[l] * 9;
        k_conv_tc<32><<<grid, NT, TcShape<32>::SMEM_BYTES, st>>>(n->act_tc[cur], n->wtc + (size_t)(l - 1) * 9 * 32 * 32,
                                                                 bias, n->act_tc[cur ^ 1], nullptr, 1.0f, H, W,
                                                                 n->tc_err);
        cur ^= 1;
    }
    k_conv_tc<16><<<grid, NT, TcShape<16>::SMEM_BYTES, st>>>(
        n->act_tc[cur], w_last, n->params + n->woff[L - 1] + (size_t)n->co[L - 1] * n->ci[L - 1] * 9, nullptr,
        n->z[L - 1], out_scale, H, W, n->tc_err);
    CNN_CUDA(cudaGetLastError(), "tc forward");
    return DNS2D_OK;
}

// backward from the loss gradient in n->gout (shape of the output); fills n->grad
int cnn_backward_dev(dns2d_cnn *n, int B, int H, int W)
{
    float *dz = n->gout, *other = n->gtmp;
    if (n->train_tc && ((size_t)B * H * W) % dns2d::cnngemm::BK == 0) {
        // weight and data gradients as tcgen05 GEMMs; GELU' is applied in the data-gradient epilogue
        for (int l = n->layers - 1; l >= 0; --l) {
            const float *xin = (l == 0) ? n->xin : n->a[l - 1];
            float *dw = n->grad + n->woff[l];
            float *db = dw + (size_t)n->co[l] * n->ci[l] * 9;
            CNN_CUDA(dns2d::cnngemm::conv_wgrad(xin, n->ci[l], dz, n->co[l], dw, db, B, H, W, n->gw, n->stream),
                     "tensor-core weight gradient");
            if (l > 0) {
                CNN_CUDA(dns2d::cnngemm::conv_dgrad(dz, n->co[l], n->params + n->woff[l], n->ci[l], n->z[l - 1], other,
                                                    B, H, W, n->gw, n->stream),
                         "tensor-core data gradient");
                std::swap(dz, other);
            }
        }
        return DNS2D_OK;
    }
    for (int l = n->layers - 1; l >= 0; --l) {
        const float *xin = (l == 0) ? n->xin : n->a[l - 1];
        float *dw = n->grad + n->woff[l];
        float *db = dw + (size_t)n->co[l] * n->ci[l] * 9;
        dns2d::cnn::k_conv3x3_wgrad<<<dim3(n->ci[l], n->co[l]), 256, 0, n->stream>>>(xin, dz, dw, db, B, n->ci[l],
                                                                                   n->co[l], H, W);
        if (l > 0) {
            dns2d::cnn::k_flip_weights<<<64, 256, 0, n->stream>>>(n->params + n->woff[l], n->wflip, n->ci[l], n->co[l]);
            conv(n, dz, n->wflip, n->zero, other, B, n->co[l], n->ci[l], H, W, n->stream);
            const size_t cnt = (size_t)B * n->ci[l] * H * W;
            dns2d::cnn::k_gelu_back<<<1024, 256, 0, n->stream>>>(n->z[l - 1], other, cnt);
            std::swap(dz, other);
        }
    }
    CNN_CUDA(cudaGetLastError(), "cnn backward");
    return DNS2D_OK;
}

int cnn_loss(dns2d_cnn *n, int B, int H, int W, double *loss)
{
    const size_t cnt = (size_t)B * H * W;
    dns2d::cnn::k_mse<<<256, 256, 0, n->stream>>>(n->z[n->layers - 1], n->tgt, n->gout, n->part, cnt);
    CNN_CUDA(cudaGetLastError(), "mse");
    if (loss) {
        double h[256];
        CNN_CUDA(cudaMemcpyAsync(h, n->part, sizeof(h), cudaMemcpyDeviceToHost, n->stream), "loss copy");
        CNN_CUDA(cudaStreamSynchronize(n->stream), "loss sync");
        double t = 0.0;
        for (double v : h) t += v;
        *loss = t / (double)cnt;
    }
    return DNS2D_OK;
}

}  // namespace

extern "C" void dns2d_cnn_destroy(dns2d_cnn *n)
{
    if (!n) return;
    if (n->stream) cudaStreamSynchronize(n->stream);
    for (float *p : n->z) cudaFree(p);
    for (float *p : n->a) cudaFree(p);
    cudaFree(n->params);
    cudaFree(n->grad);
    cudaFree(n->adam_m);
    cudaFree(n->adam_v);
    cudaFree(n->wflip);
    cudaFree(n->zero);
    cudaFree(n->xin);
    cudaFree(n->tgt);
    cudaFree(n->gout);
    cudaFree(n->gtmp);
    cudaFree(n->part);
    cudaFree(n->data_x);
    cudaFree(n->data_t);
    cudaFree(n->wtc);
    cudaFree(n->act_tc[0]);
    cudaFree(n->act_tc[1]);
    cudaFree(n->tc_err);
    cudaFree(n->net_sync);
    cudaFree(n->trace);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

extern "C" const char *dns2d_cnn_last_error(const dns2d_cnn *n) { return n ? n->err.c_str() : "null network"; }

extern "C" int dns2d_cnn_create(dns2d_cnn **out, int layers, int channels, uint64_t seed, int device)
{
    if (!out || layers < 2 || channels < 1 || channels > 256) return DNS2D_ERR_ARG;
    *out = nullptr;
    dns2d_cnn *n = new dns2d_cnn();
    n->layers = layers;
    n->channels = channels;
    n->device = device;
    auto bail = [&](int rc) {
        dns2d_cnn_destroy(n);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(DNS2D_ERR_CUDA);
    size_t off = 0;
    for (int l = 0; l < layers; ++l) {
        n->ci.push_back(l == 0 ? 3 : channels);
        n->co.push_back(l == layers - 1 ? 1 : channels);
        n->woff.push_back(off);
        off += (size_t)n->co[l] * n->ci[l] * 9 + n->co[l];
    }
    n->nparams = (int)off;
    // He-normal weights (Box-Muller on splitmix64), zero biases; last layer scaled by 0.1
    std::vector<float> p(off, 0.0f);
    uint64_t st = seed;
    for (int l = 0; l < layers; ++l) {
        const double sd = std::sqrt(2.0 / (9.0 * n->ci[l])) * (l == layers - 1 ? 0.1 : 1.0);
        const size_t nw = (size_t)n->co[l] * n->ci[l] * 9;
        for (size_t i = 0; i < nw; ++i) {
            const double u1 = ((sm64(st) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
            const double u2 = (sm64(st) >> 11) * (1.0 / 9007199254740992.0);
            p[n->woff[l] + i] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2));
        }
    }
    size_t maxw = 0;
    for (int l = 0; l < layers; ++l) maxw = std::max(maxw, (size_t)n->co[l] * n->ci[l] * 9);
    if (cudaMalloc((void **)&n->params, off * 4) != cudaSuccess || cudaMalloc((void **)&n->grad, off * 4) != cudaSuccess ||
        cudaMalloc((void **)&n->adam_m, off * 4) != cudaSuccess || cudaMalloc((void **)&n->adam_v, off * 4) != cudaSuccess ||
        cudaMalloc((void **)&n->wflip, maxw * 4) != cudaSuccess || cudaMalloc((void **)&n->zero, 256 * 4) != cudaSuccess ||
        cudaMalloc((void **)&n->part, 256 * 8) != cudaSuccess)
        return bail(DNS2D_ERR_NOMEM);
    if (cudaMemcpy(n->params, p.data(), off * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(n->adam_m, 0, off * 4) != cudaSuccess || cudaMemset(n->adam_v, 0, off * 4) != cudaSuccess ||
        cudaMemset(n->zero, 0, 256 * 4) != cudaSuccess)
        return bail(DNS2D_ERR_CUDA);
    const int smax = (int)(((size_t)channels * (dns2d::cnn::TILE + 2) * (dns2d::cnn::TILE + 2) +
                            (size_t)dns2d::cnn::COT * channels * 9) * 4);
    if (cudaFuncSetAttribute(dns2d::cnn::k_conv3x3, cudaFuncAttributeMaxDynamicSharedMemorySize, smax) != cudaSuccess)
        return bail(DNS2D_ERR_CUDA);
    *out = n;
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_num_params(const dns2d_cnn *n) { return n ? n->nparams : 0; }

extern "C" int dns2d_cnn_get_params(dns2d_cnn *n, float *p)
{
    if (!n || !p) return DNS2D_ERR_ARG;
    CNN_CUDA(cudaMemcpyAsync(p, n->params, (size_t)n->nparams * 4, cudaMemcpyDeviceToHost, n->stream), "params copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "params sync");
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_set_params(dns2d_cnn *n, const float *p)
{
    if (!n || !p) return DNS2D_ERR_ARG;
    CNN_CUDA(cudaMemcpyAsync(n->params, p, (size_t)n->nparams * 4, cudaMemcpyHostToDevice, n->stream), "params copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "params sync");
    n->gen += 1;
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_forward(dns2d_cnn *n, const float *x, int B, int H, int W, float *y)
{
    if (!n || !x || !y || B <= 0 || H <= 0 || W <= 0) return DNS2D_ERR_ARG;
    int rc = cnn_reserve(n, B, H, W);
    if (rc) return rc;
    CNN_CUDA(cudaMemcpyAsync(n->xin, x, (size_t)B * 3 * H * W * 4, cudaMemcpyHostToDevice, n->stream), "input copy");
    rc = cnn_forward_dev(n, B, H, W);
    if (rc) return rc;
    CNN_CUDA(cudaMemcpyAsync(y, n->z[n->layers - 1], (size_t)B * H * W * 4, cudaMemcpyDeviceToHost, n->stream), "out copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "forward sync");
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_set_tc_mode(dns2d_cnn *n, int mode)
{
    if (!n || mode < 0 || mode > 1) return DNS2D_ERR_ARG;
    n->tc_mode = mode;
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_set_trace(dns2d_cnn *n, int on)
{
    if (!n || on < 0 || on > 1) return DNS2D_ERR_ARG;
    n->trace_on = on;
    if (!on) n->trace_tiles = 0;
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_read_trace(dns2d_cnn *n, unsigned long long *out, int cap, int *tiles)
{
    if (!n || !out || cap < 0 || !tiles) return DNS2D_ERR_ARG;
    *tiles = n->trace_tiles;
    const int m = n->trace_tiles < cap ? n->trace_tiles : cap;
    if (m <= 0) return DNS2D_OK;
    CNN_CUDA(cudaStreamSynchronize(n->stream), "trace sync");
    CNN_CUDA(cudaMemcpy(out, n->trace, (size_t)m * dns2d::cnntc::kNetTraceSlots * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost),
             "trace copy");
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_set_train_tc(dns2d_cnn *n, int on)
{
    if (!n || on < 0 || on > 1) return DNS2D_ERR_ARG;
    if (on && n->channels > dns2d::cnngemm::BN)
        return nfail(n, DNS2D_ERR_SIZE, "tensor-core training needs at most 32 channels");
    n->train_tc = on;
    return DNS2D_OK;
}

// the tensor-core training GEMMs' wait flag (0 when no GEMM ran); the stream is synchronised
static int train_tc_status(dns2d_cnn *n)
{
    if (!n->gw.err) return DNS2D_OK;
    int flag = 0;
    CNN_CUDA(cudaMemcpyAsync(&flag, n->gw.err, 4, cudaMemcpyDeviceToHost, n->stream), "flag copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "flag sync");
    if (flag) return nfail(n, DNS2D_ERR_TIMEOUT, "tensor-core training GEMM wait timed out");
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_tc_info(const dns2d_cnn *n, int *mode, int *grid)
{
    if (!n) return DNS2D_ERR_ARG;
    if (mode) *mode = n->tc_mode;
    if (grid) *grid = n->net_grid;
    return DNS2D_OK;
}

// the same network on the BF16 tensor-core path (hidden layers on tcgen05); W % 128 == 0
extern "C" int dns2d_cnn_forward_tc(dns2d_cnn *n, const float *x, int B, int H, int W, float *y)
{
    if (!n || !x || !y || B <= 0 || H <= 0 || W <= 0) return DNS2D_ERR_ARG;
    if (!cnn_tc_supported(n, H, W))
        return nfail(n, DNS2D_ERR_SIZE, "tensor-core path needs 32 channels, >= 3 layers, W % 128 == 0 and even H");
    int rc = cnn_reserve(n, B, H, W);
    if (!rc) rc = cnn_tc_reserve(n, B, H, W);
    if (rc) return rc;
    CNN_CUDA(cudaMemcpyAsync(n->xin, x, (size_t)B * 3 * H * W * 4, cudaMemcpyHostToDevice, n->stream), "input copy");
    dns2d::cnntc::FirstIn in;
    const size_t plane = (size_t)H * W;
    for (int c = 0; c < 3; ++c) {
        in.p[c] = n->xin + c * plane;
        in.s[c] = 1.0f;
    }
    in.pstride = 3 * plane;
    if ((rc = cnn_tc_prepare(n, n->stream)) || (rc = cnn_forward_tc_dev(n, B, H, W, in, 1.0f, n->stream))) return rc;
    CNN_CUDA(cudaMemcpyAsync(y, n->z[n->layers - 1], (size_t)B * H * W * 4, cudaMemcpyDeviceToHost, n->stream), "out copy");
    int flag = 0;
    CNN_CUDA(cudaMemcpyAsync(&flag, n->tc_err, 4, cudaMemcpyDeviceToHost, n->stream), "flag copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "forward sync");
    if (flag) return nfail(n, DNS2D_ERR_TIMEOUT, "tensor-core MMA completion wait timed out");
    return DNS2D_OK;
}

extern "C" int dns2d_cnn_loss_grad(dns2d_cnn *n, const float *x, const float *t, int B, int H, int W, double *loss,
                                   float *grad)
{
    if (!n || !x || !t || B <= 0) return DNS2D_ERR_ARG;
    int rc = cnn_reserve(n, B, H, W);
    if (rc) return rc;
    CNN_CUDA(cudaMemcpyAsync(n->xin, x, (size_t)B * 3 * H * W * 4, cudaMemcpyHostToDevice, n->stream), "input copy");
    CNN_CUDA(cudaMemcpyAsync(n->tgt, t, (size_t)B * H * W * 4, cudaMemcpyHostToDevice, n->stream), "target copy");
    if ((rc = cnn_forward_dev(n, B, H, W)) || (rc = cnn_loss(n, B, H, W, loss)) || (rc = cnn_backward_dev(n, B, H, W)))
        return rc;
    if (grad) CNN_CUDA(cudaMemcpyAsync(grad, n->grad, (size_t)n->nparams * 4, cudaMemcpyDeviceToHost, n->stream), "grad copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "grad sync");
    return train_tc_status(n);
}

extern "C" int dns2d_cnn_set_dataset(dns2d_cnn *n, const float *x, const float *t, int count, int H, int W)
{
    if (!n || !x || !t || count <= 0) return DNS2D_ERR_ARG;
    cudaFree(n->data_x);
    cudaFree(n->data_t);
    n->data_x = n->data_t = nullptr;
    CNN_CUDA(cudaMalloc((void **)&n->data_x, (size_t)count * 3 * H * W * 4), "dataset alloc");
    CNN_CUDA(cudaMalloc((void **)&n->data_t, (size_t)count * H * W * 4), "dataset alloc");
    CNN_CUDA(cudaMemcpyAsync(n->data_x, x, (size_t)count * 3 * H * W * 4, cudaMemcpyHostToDevice, n->stream), "dataset copy");
    CNN_CUDA(cudaMemcpyAsync(n->data_t, t, (size_t)count * H * W * 4, cudaMemcpyHostToDevice, n->stream), "dataset copy");
    CNN_CUDA(cudaStreamSynchronize(n->stream), "dataset sync");
    n->data_n = count;
    n->data_H = H;
    n->data_W = W;
    return DNS2D_OK;
}

// Adam iterations on minibatches drawn (without replacement within a batch) from the resident
// dataset by splitmix64(seed); losses (nullable) receives the loss of every iteration
extern "C" int dns2d_cnn_train(dns2d_cnn *n, int iters, int batch, float lr, uint64_t seed, double *losses)
{
    if (!n || iters < 0 || batch <= 0 || !n->data_n) return DNS2D_ERR_ARG;
    const int H = n->data_H, W = n->data_W;
    int rc = cnn_reserve(n, batch, H, W);
    if (rc) return rc;
    uint64_t st = seed;
    std::vector<int> idx((size_t)n->data_n);
    const size_t xs = (size_t)3 * H * W, ts = (size_t)H * W;
    for (int it = 0; it < iters; ++it) {
        for (int i = 0; i < n->data_n; ++i) idx[(size_t)i] = i;
        for (int i = 0; i < batch && i < n->data_n; ++i) {
            const int j = i + (int)(sm64(st) % (uint64_t)(n->data_n - i));
            std::swap(idx[(size_t)i], idx[(size_t)j]);
        }
        for (int i = 0; i < batch; ++i) {
            const int k = idx[(size_t)(i % n->data_n)];
            CNN_CUDA(cudaMemcpyAsync(n->xin + i * xs, n->data_x + k * xs, xs * 4, cudaMemcpyDeviceToDevice, n->stream),
                     "batch gather");
            CNN_CUDA(cudaMemcpyAsync(n->tgt + i * ts, n->data_t + k * ts, ts * 4, cudaMemcpyDeviceToDevice, n->stream),
                     "batch gather");
        }
        double loss = 0.0;
        if ((rc = cnn_forward_dev(n, batch, H, W)) || (rc = cnn_loss(n, batch, H, W, losses ? &loss : nullptr)) ||
            (rc = cnn_backward_dev(n, batch, H, W)))
            return rc;
        n->step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.0f - (float)std::pow((double)b1, (double)n->step);
        const float c2 = 1.0f - (float)std::pow((double)b2, (double)n->step);
        dns2d::cnn::k_adam<<<64, 256, 0, n->stream>>>(n->params, n->grad, n->adam_m, n->adam_v, n->nparams, lr, b1, b2,
                                                      1e-8f, c1, c2);
        CNN_CUDA(cudaGetLastError(), "adam");
        if (losses) losses[it] = loss;
    }
    CNN_CUDA(cudaStreamSynchronize(n->stream), "train sync");
    n->gen += 1;
    return train_tc_status(n);
}

// ============================================================================================
// Learned closure coupled to a state.  Every step: the state's u, w and omega on the L x L grid
// (the CNN's inputs, divided by the input scales) -> CNN -> forcing field (times the output
// scale) -> its retained spectrum, added to FN in the column pass.  With the energy check on, a
// step whose energy rises (the viscous bound: unforced 2D flow can only lose energy) is redone
// as the plain step.
// ============================================================================================
namespace {

__global__ void k_closure_inputs(const float *phys, float *xin, size_t plane, float s_om, float s_u, float s_w)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x) {
        xin[i] = phys[2 * plane + i] / s_om;
        xin[plane + i] = phys[i] / s_u;
        xin[2 * plane + i] = phys[plane + i] / s_w;
    }
}

__global__ void k_scale_copy(const float *in, float *out, size_t n, float sc)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[i] * sc;
}

// forcing spectrum of the current state into s->force; with g.om2 set the forcing's column
// transform also decides the step's energy gate (GateArgs, dns2d_kernels.cuh)
int closure_forcing(dns2d_state *s, const GateArgs &g = GateArgs{})
{
    dns2d_cnn *n = s->cnn;
    const int L = s->L;
    const size_t plane = (size_t)L * L;
    Pointers p = s->ptrs();
    s->ks->rows_velocity(p, s->phys, nullptr, 1.0f, s->stream, 1);
    s->ks->cols_scalar(p, s->scratch, 0, s->stream);
    s->ks->rows_scalar(p, s->scratch, s->phys + 2 * plane, s->minmax, s->stream);
    const float *forcing_field = s->closure_in;
    if (s->closure_tc && cnn_tc_supported(n, L, L)) {
        // tensor-core path: the first layer reads (omega, u, w) / scales straight from the planes,
        // the last layer writes its output times the output scale
        dns2d::cnntc::FirstIn in;
        in.p[0] = s->phys + 2 * plane;
        in.p[1] = s->phys;
        in.p[2] = s->phys + plane;
        for (int c = 0; c < 3; ++c) in.s[c] = 1.0f / s->in_scale[c];
        in.pstride = 0;
        int rc = cnn_forward_tc_dev(n, 1, L, L, in, s->out_scale, s->stream);
        if (rc) return fail(s, rc, "closure network: %s", n->err.c_str());
        forcing_field = n->z[n->layers - 1];
    } else {
        k_closure_inputs<<<256, 256, 0, s->stream>>>(s->phys, n->xin, plane, s->in_scale[0], s->in_scale[1],
                                                     s->in_scale[2]);
        DNS2D_LAUNCHED("closure inputs");
        int rc = cnn_forward_dev(n, 1, L, L, s->stream);
        if (rc) return fail(s, rc, "closure network: %s", n->err.c_str());
        k_scale_copy<<<256, 256, 0, s->stream>>>(n->z[n->layers - 1], s->closure_in, plane, s->out_scale);
        DNS2D_LAUNCHED("closure output");
    }
    s->ks->rows_fwd_scalar(p, forcing_field, s->scratch, s->stream);
    s->ks->cols_fwd_scalar(p, s->scratch, s->force, g, s->stream);
    DNS2D_LAUNCHED("closure transform");
    return DNS2D_OK;
}

}  // namespace

// one closed step on the device: forcing, energy gate, row pass, column pass (capturable)
static int closure_device_step(dns2d_state *s, int first, int slot)
{
    s->mm_plane2 = 0;  // the closure's inputs are staged in the physical planes
    GateArgs g;
    const bool gated = s->closure_check == 1 || s->closure_check == 3;
    if (gated) {
        g.om2 = s->om2;
        g.visc = s->visc;
        g.scale = s->closure_check == 3 ? 1 : 0;
        g.gate = s->gate;
        g.off = s->gate_off;
        g.part = s->gate_part;
        g.counter = s->gate_counter;
    }
    int rc = closure_forcing(s, g);
    if (rc) return rc;
    Pointers p = s->ptrs();
    p.force = s->force;
    p.force_clamp = s->closure_clamp;
    if (gated) p.gate = s->gate;
    s->ks->rows_step(p, s->stream, 1);
    s->ks->cols_step(p, first, slot, s->stream, 1);
    DNS2D_LAUNCHED("closed step");
    return DNS2D_OK;
}

static int closure_run(dns2d_state *s, int nsteps, double *E_hist, double *Z_hist)
{
    const size_t nom = (size_t)s->N * s->H, nwork = 2 * (size_t)s->L * s->H;
    if (s->closure_check != 2) {
        // device-side energy gate; chunks of up to 128 closed steps are captured CUDA graphs
        int done = 0;
        while (done < nsteps) {
            const int K = std::min(kChunk, nsteps - done);
            const float cnm1_first = (done == 0) ? s->cnm1 : s->cn;
            k_set_params<<<1, 1, 0, s->stream>>>(s->prm, s->dt, cnm1_first, s->cn, s->visc);
            DNS2D_LAUNCHED("set params");
            const int key = (done == 0 ? 1 : 0) * 1000 + K;
            auto itg = s->closure_graphs.find(key);
            cudaGraphExec_t ex = nullptr;
            if (itg != s->closure_graphs.end()) {
                ex = itg->second;
            } else {
                cudaGraph_t g = nullptr;
                DNS2D_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
                for (int i = 0; i < K; ++i) {
                    int rc = closure_device_step(s, (done == 0 && i == 0) ? 1 : 0, i);
                    if (rc) {
                        cudaStreamEndCapture(s->stream, &g);
                        if (g) cudaGraphDestroy(g);
                        return rc;
                    }
                }
                DNS2D_CUDA(cudaStreamEndCapture(s->stream, &g), "end capture");
                cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return cuda_check(s, e, "graph instantiate");
                s->closure_graphs[key] = ex;
            }
            DNS2D_CUDA(cudaGraphLaunch(ex, s->stream), "graph launch");
            if (E_hist || Z_hist) {
                DNS2D_CUDA(cudaMemcpyAsync(s->hist_host, s->hist, (size_t)K * 16, cudaMemcpyDeviceToHost, s->stream),
                           "history copy");
                DNS2D_CUDA(cudaStreamSynchronize(s->stream), "history sync");
                for (int i = 0; i < K; ++i) {
                    if (E_hist) E_hist[done + i] = s->hist_host[i].x;
                    if (Z_hist) Z_hist[done + i] = s->hist_host[i].y;
                }
            }
            for (int i = 0; i < K; ++i) {
                s->it += 1;
                const float dt_old = s->dt;
                s->cnm1 = s->cn;
                s->t += dt_old;
            }
            s->closure_steps += K;
            done += K;
        }
        return DNS2D_OK;
    }
    if (s->closure_check && s->closure_E < 0.0) {
        double E0 = 0.0;
        int rc = dns2d_energy_enstrophy(s, &E0, nullptr);
        if (rc) return rc;
        s->closure_E = E0;
    }
    for (int i = 0; i < nsteps; ++i) {
        const float cnm1_eff = (i == 0) ? s->cnm1 : s->cn;
        k_set_params<<<1, 1, 0, s->stream>>>(s->prm, s->dt, cnm1_eff, s->cn, s->visc);
        if (s->closure_check) {
            DNS2D_CUDA(cudaMemcpyAsync(s->bk_om2, s->om2, nom * 8, cudaMemcpyDeviceToDevice, s->stream), "backup");
            DNS2D_CUDA(cudaMemcpyAsync(s->bk_fnm1, s->fnm1, nom * 8, cudaMemcpyDeviceToDevice, s->stream), "backup");
            DNS2D_CUDA(cudaMemcpyAsync(s->bk_work, s->work, nwork * 8, cudaMemcpyDeviceToDevice, s->stream), "backup");
        }
        int rc = closure_forcing(s);
        if (rc) return rc;
        Pointers p = s->ptrs();
        p.force = s->force;
        p.force_clamp = s->closure_clamp;
        s->ks->rows_step(p, s->stream, 1);
        s->ks->cols_step(p, 1, 0, s->stream, 1);
        DNS2D_LAUNCHED("closure step");
        s->closure_steps += 1;
        double2 ez = make_double2(0.0, 0.0);
        if (s->closure_check || E_hist || Z_hist) {
            DNS2D_CUDA(cudaMemcpyAsync(&ez, s->hist, 16, cudaMemcpyDeviceToHost, s->stream), "energy copy");
            DNS2D_CUDA(cudaStreamSynchronize(s->stream), "energy sync");
        }
        if (s->closure_check && ez.x > s->closure_E * (1.0 + 1.0e-7)) {
            // energy rose above the viscous bound: redo this step without the closure
            DNS2D_CUDA(cudaMemcpyAsync(s->om2, s->bk_om2, nom * 8, cudaMemcpyDeviceToDevice, s->stream), "restore");
            DNS2D_CUDA(cudaMemcpyAsync(s->fnm1, s->bk_fnm1, nom * 8, cudaMemcpyDeviceToDevice, s->stream), "restore");
            DNS2D_CUDA(cudaMemcpyAsync(s->work, s->bk_work, nwork * 8, cudaMemcpyDeviceToDevice, s->stream), "restore");
            Pointers q = s->ptrs();
            s->ks->rows_step(q, s->stream, 1);
            s->ks->cols_step(q, 1, 0, s->stream, 1);
            DNS2D_LAUNCHED("plain step");
            DNS2D_CUDA(cudaMemcpyAsync(&ez, s->hist, 16, cudaMemcpyDeviceToHost, s->stream), "energy copy");
            DNS2D_CUDA(cudaStreamSynchronize(s->stream), "energy sync");
            s->closure_fallbacks += 1;
        }
        if (s->closure_check) s->closure_E = ez.x;
        if (E_hist) E_hist[i] = ez.x;
        if (Z_hist) Z_hist[i] = ez.y;
        s->it += 1;
        const float dt_old = s->dt;
        s->cnm1 = s->cn;
        s->t += dt_old;
    }
    return DNS2D_OK;
}

extern "C" int dns2d_closure_attach(dns2d_state *s, dns2d_cnn *n, const float *scales4, int energy_check)
{
    if (!s) return DNS2D_ERR_ARG;
    if (!n) {  // detach
        s->cnn = nullptr;
        return DNS2D_OK;
    }
    if (!scales4) return DNS2D_ERR_ARG;
    if (!s->ks->rows_fwd_scalar || !s->ks->cols_fwd_scalar)
        return fail(s, DNS2D_ERR_SIZE, "no closure transforms at N=%d", s->N);
    const size_t nom = (size_t)s->N * s->H, nwork = 2 * (size_t)s->L * s->H, plane = (size_t)s->L * s->L;
    if (!s->force) {
        if (cudaMalloc((void **)&s->force, nom * 8) != cudaSuccess || cudaMalloc((void **)&s->bk_om2, nom * 8) != cudaSuccess ||
            cudaMalloc((void **)&s->bk_fnm1, nom * 8) != cudaSuccess ||
            cudaMalloc((void **)&s->bk_work, nwork * 8) != cudaSuccess ||
            cudaMalloc((void **)&s->closure_in, plane * 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(s, DNS2D_ERR_NOMEM, "closure buffers");
        }
    }
    if (!s->gate) {
        if (cudaMalloc((void **)&s->gate, 4) != cudaSuccess || cudaMalloc((void **)&s->gate_off, 8) != cudaSuccess ||
            cudaMalloc((void **)&s->gate_part, (size_t)s->H * 16) != cudaSuccess ||
            cudaMalloc((void **)&s->gate_counter, 4) != cudaSuccess ||
            cudaMemset(s->gate_counter, 0, 4) != cudaSuccess) {
            cudaGetLastError();
            return fail(s, DNS2D_ERR_NOMEM, "closure gate");
        }
    }
    DNS2D_CUDA(cudaMemsetAsync(s->gate_off, 0, 8, s->stream), "gate counter");
    for (auto &kv : s->closure_graphs) cudaGraphExecDestroy(kv.second);
    s->closure_graphs.clear();
    int rc = cnn_reserve(n, 1, s->L, s->L);
    if (!rc && cnn_tc_supported(n, s->L, s->L)) {
        rc = cnn_tc_reserve(n, 1, s->L, s->L);
        if (!rc) rc = cnn_tc_prepare(n, n->stream);
        if (!rc && cudaStreamSynchronize(n->stream) != cudaSuccess) rc = DNS2D_ERR_CUDA;
    }
    if (rc) return fail(s, rc, "closure network: %s", n->err.c_str());
    s->cnn = n;
    for (int c = 0; c < 3; ++c) s->in_scale[c] = scales4[c];
    s->out_scale = scales4[3];
    s->closure_check = (energy_check < 0 || energy_check > 3) ? 1 : energy_check;
    s->closure_E = -1.0;
    s->closure_steps = 0;
    s->closure_fallbacks = 0;
    return DNS2D_OK;
}

// forcing spectrum that the attached closure adds to FN for the current state (compact layout of
// dns2d_get_fnm1)
// forcing limiter of the attached closure: per mode |forcing| <= alpha |FN| (alpha <= 0: off)
extern "C" int dns2d_closure_clamp(dns2d_state *s, float alpha)
{
    if (!s) return DNS2D_ERR_ARG;
    s->closure_clamp = alpha > 0.0f ? alpha : 0.0f;
    for (auto &kv : s->closure_graphs) cudaGraphExecDestroy(kv.second);
    s->closure_graphs.clear();
    return DNS2D_OK;
}

// BF16 tensor-core inference of the attached closure network (default on where the grid allows
// it); 0 runs the FP32 SIMT network
extern "C" int dns2d_closure_tensor_cores(dns2d_state *s, int enable)
{
    if (!s) return DNS2D_ERR_ARG;
    s->closure_tc = enable ? 1 : 0;
    for (auto &kv : s->closure_graphs) cudaGraphExecDestroy(kv.second);
    s->closure_graphs.clear();
    return DNS2D_OK;
}

extern "C" int dns2d_closure_forcing(dns2d_state *s, float *force)
{
    if (!s || !force) return DNS2D_ERR_ARG;
    if (!s->cnn) return fail(s, DNS2D_ERR_STATE, "no closure attached");
    if (!s->initialised) return fail(s, DNS2D_ERR_STATE, "no initial condition");
    int rc = closure_forcing(s);
    if (rc) return rc;
    return download_compact(s, s->force, force);
}

extern "C" int dns2d_closure_stats(dns2d_state *s, long long *steps, long long *fallbacks)
{
    if (!s) return DNS2D_ERR_ARG;
    if (s->cnn && s->cnn->tc_err) {  // a tensor-core wait that ran out marks the closure unusable
        int flag = 0;
        DNS2D_CUDA(cudaMemcpyAsync(&flag, s->cnn->tc_err, 4, cudaMemcpyDeviceToHost, s->stream), "flag copy");
        DNS2D_CUDA(cudaStreamSynchronize(s->stream), "flag sync");
        if (flag) return fail(s, DNS2D_ERR_TIMEOUT, "tensor-core MMA completion wait timed out in the closure network");
    }
    if (steps) *steps = s->closure_steps;
    if (fallbacks) {
        unsigned long long gated = 0;
        if (s->gate_off) {
            DNS2D_CUDA(cudaMemcpyAsync(&gated, s->gate_off, 8, cudaMemcpyDeviceToHost, s->stream), "gate copy");
            DNS2D_CUDA(cudaStreamSynchronize(s->stream), "gate sync");
        }
        *fallbacks = s->closure_fallbacks + (long long)gated;
    }
    return DNS2D_OK;
}

// ============================================================================================
// Time step without device allocation.
//
// For callers that may not allocate device memory at all (an application that hands the solver
// fixed buffers from its own pool or arena, a process under a strict device-memory budget, or
// code running where cudaMalloc is forbidden).  The caller owns the vorticity state; everything
// else the step needs (the U,W / D,E work buffer, transposed copies of the state, twiddles,
// parameter block, reduction partials) lives in one static device array of this file.
// ============================================================================================
namespace {

// one array per device, allocated when the module loads and held until the process exits
static __device__ __align__(256) unsigned char g_noalloc_scratch[DNS2D_NOALLOC_SCRATCH_BYTES];

// Per-device address of g_noalloc_scratch.  In host code the array's name is only a host-side
// stand-in, so the device address is looked up with cudaGetSymbolAddress, with the device
// current.  Outside stream capture the lookup is repeated on every call (it is a host-side
// query), so a context that was reset and reloaded the module at another address is never
// handed a stale pointer; while `stream` is capturing, the address cached by the last call
// outside capture is used.
unsigned char *noalloc_scratch_address(cudaStream_t stream, int *err)
{
    static std::mutex mu;
    static unsigned char *addr[128] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) {
        *err = DNS2D_ERR_CUDA;
        return nullptr;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
        *err = DNS2D_ERR_CUDA;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (cs == cudaStreamCaptureStatusNone || !addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            *err = DNS2D_ERR_CUDA;
            return nullptr;
        }
        addr[dev] = static_cast<unsigned char *>(p);
    }
    return addr[dev];
}

// the per-stage twiddle tables of a catalog, built in FP64 on the device and rounded once
__global__ void k_noalloc_twiddles(float2 *tw, TwCatalog c)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < c.total; e += gridDim.x * blockDim.x) {
        int i = 0;
        while (i + 1 < c.n && c.off[i + 1] <= e) ++i;
        const int R = c.R[i], NS = c.NS[i], M = R * NS;
        const int loc = e - c.off[i];
        const int r = loc / NS + 1, k = loc % NS;
        const long long m = ((long long)r * k) % M;
        double sn, cs;
        sincospi(2.0 * (double)m / (double)M, &sn, &cs);
        tw[e] = make_float2((float)cs, (float)-sn);
    }
}

__global__ void k_noalloc_reset(unsigned int *counter) { *counter = 0u; }

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int dns2d_step_noalloc(int N, float visc, float dt, float cnm1, float cn, int nsteps,
                                  void *om2, void *fnm1, void *stream)
{
    if (N > DNS2D_NOALLOC_MAX_N) return DNS2D_ERR_SIZE;
    const KernelSet *ks = kernel_set(N);
    if (!ks) return DNS2D_ERR_SIZE;
    if (!om2 || !fnm1 || nsteps < 0) return DNS2D_ERR_ARG;
    const size_t H = N / 2, L = 3 * (size_t)N / 2, nom = (size_t)N * H;
    // scratch layout inside g_noalloc_scratch
    const size_t o_work = 0;
    const size_t o_om = o_work + align256(2 * L * H * sizeof(float2));
    const size_t o_fn = o_om + align256(nom * sizeof(float2));
    const size_t o_tw = o_fn + align256(nom * sizeof(float2));
    const size_t o_prm = o_tw + align256((size_t)std::max(ks->cat->total, 1) * sizeof(float2));
    const size_t o_part = o_prm + align256(sizeof(StepParams));
    const size_t o_cnt = o_part + align256(H * sizeof(double2));
    const size_t o_hist = o_cnt + align256(sizeof(unsigned int));
    const size_t total = o_hist + align256(sizeof(double2));
    if (total > DNS2D_NOALLOC_SCRATCH_BYTES) return DNS2D_ERR_SIZE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // an error left pending on this thread by earlier, unrelated launches is cleared here, so
    // the checks below report only this call's own launches
    (void)cudaGetLastError();
    int err = DNS2D_OK;
    unsigned char *base = noalloc_scratch_address(st, &err);
    if (!base) return err;
    if (ks->setup() != cudaSuccess) return DNS2D_ERR_CUDA;
    Pointers p;
    p.work = reinterpret_cast<float2 *>(base + o_work);
    p.om2 = reinterpret_cast<float2 *>(base + o_om);
    p.fnm1 = reinterpret_cast<float2 *>(base + o_fn);
    p.tw = reinterpret_cast<const float2 *>(base + o_tw);
    p.prm = reinterpret_cast<const StepParams *>(base + o_prm);
    p.part = reinterpret_cast<double2 *>(base + o_part);
    p.counter = reinterpret_cast<unsigned int *>(base + o_cnt);
    p.hist = reinterpret_cast<double2 *>(base + o_hist);
    p.force = nullptr;
    p.gate = nullptr;
    p.s_state = p.s_work = 0;
    p.s_part = p.s_hist = 0;
    // the array keeps the previous call's contents: rebuild twiddles, parameters and counter
    k_noalloc_twiddles<<<(unsigned)((ks->cat->total + 255) / 256), 256, 0, st>>>(reinterpret_cast<float2 *>(base + o_tw),
                                                                                *ks->cat);
    k_set_params<<<1, 1, 0, st>>>(reinterpret_cast<StepParams *>(base + o_prm), dt, cnm1, cn, visc);
    k_noalloc_reset<<<1, 1, 0, st>>>(p.counter);
    dim3 tb(32, 8);
    k_transpose_c64<<<dim3((unsigned)((H + 31) / 32), (unsigned)((N + 31) / 32)), tb, 0, st>>>(
        static_cast<const float2 *>(om2), p.om2, N, (int)H);
    k_transpose_c64<<<dim3((unsigned)((H + 31) / 32), (unsigned)((N + 31) / 32)), tb, 0, st>>>(
        static_cast<const float2 *>(fnm1), p.fnm1, N, (int)H);
    ks->cols_init(p, nullptr, 1, st, 1);  // velocity of the given vorticity
    if (cudaGetLastError() != cudaSuccess) return DNS2D_ERR_CUDA;  // set-up launches
    for (int i = 0; i < nsteps; ++i) {
        ks->rows_step(p, st, 1);
        ks->cols_step(p, i == 0 ? 1 : 0, 0, st, 1);
        if (cudaGetLastError() != cudaSuccess) return DNS2D_ERR_CUDA;  // step launches
    }
    k_transpose_c64<<<dim3((unsigned)((N + 31) / 32), (unsigned)((H + 31) / 32)), tb, 0, st>>>(
        p.om2, static_cast<float2 *>(om2), (int)H, N);
    k_transpose_c64<<<dim3((unsigned)((N + 31) / 32), (unsigned)((H + 31) / 32)), tb, 0, st>>>(
        p.fnm1, static_cast<float2 *>(fnm1), (int)H, N);
    return cudaGetLastError() == cudaSuccess ? DNS2D_OK : DNS2D_ERR_CUDA;
}
