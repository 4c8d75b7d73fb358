// fft.cuh — shared-memory Stockham FFT engine for the B200 (sm_100a) DNS kernels.
//
// A transform of compile-time length L runs as a sequence of radix-R stages
// (radix plan = template list).  Each stage reads its R inputs per butterfly from shared
// memory into registers, applies the inter-stage twiddles W_{Ns*R}^{r*k} (looked up in
// FP64-built, once-rounded per-stage tables held in global memory / L1), performs the R-point
// DFT fully unrolled in registers (generic Cooley-Tukey codelets whose constants are folded at
// compile time) and writes the R outputs back in Stockham auto-sort order.  Several arrays
// (rows or columns of the DNS fields) can be transformed together by one CTA.
//
// Conventions: forward = exp(-2 pi i jk/L), inverse = exp(+2 pi i jk/L), both unnormalised,
// the same as the reference's cuFFT R2C/C2R calls (cuda/vfft_cuda.cu:14-42).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace dns2d {

// ------------------------------------------------------------------------------------------
// compile-time trigonometry for codelet constants: cos/sin(2 pi k / R) by Taylor series on an
// angle reduced to [-pi, pi]; the results are rounded to float, so double accuracy suffices.
// ------------------------------------------------------------------------------------------
constexpr double kPi = 3.14159265358979323846264338327950288;

constexpr double ct_series_sin(double x)
{
    double x2 = x * x, term = x, sum = x;
    for (int n = 1; n < 20; ++n) {
        term *= -x2 / (double)((2 * n) * (2 * n + 1));
        sum += term;
    }
    return sum;
}

constexpr double ct_series_cos(double x)
{
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int n = 1; n < 20; ++n) {
        term *= -x2 / (double)((2 * n - 1) * (2 * n));
        sum += term;
    }
    return sum;
}

constexpr double ct_angle(int k, int R)
{
    int m = ((k % R) + R) % R;
    if (2 * m > R) m -= R;  // reduce to [-pi, pi]
    return 2.0 * kPi * (double)m / (double)R;
}

constexpr double ct_cos(int k, int R) { return ct_series_cos(ct_angle(k, R)); }
constexpr double ct_sin(int k, int R) { return ct_series_sin(ct_angle(k, R)); }

constexpr int ct_first_factor(int R)
{
    if (R % 4 == 0 && R != 4) return 4;
    for (int f = 2; f * f <= R; ++f)
        if (R % f == 0) return f;
    return R;
}

constexpr bool ct_is_prime(int R) { return R > 1 && ct_first_factor(R) == R; }

template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (B < E) {
        f(std::integral_constant<int, B>{});
        static_for<B + 1, E>(f);
    }
}

// ------------------------------------------------------------------------------------------
// complex helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 cmul_mi(float2 a)
{
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// a * W_R^K with W_R = exp(-+ 2 pi i / R); trivial angles become sign swaps
template <int R, int K, bool INV>
__device__ __forceinline__ float2 twid(float2 a)
{
    constexpr int k = ((K % R) + R) % R;
    if constexpr (k == 0) {
        return a;
    } else if constexpr (2 * k == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * k == R) {
        return cmul_mi<INV>(a);
    } else if constexpr (4 * k == 3 * R) {
        return cmul_mi<!INV>(a);
    } else {
        constexpr float c = (float)ct_cos(k, R);
        constexpr float s = INV ? (float)ct_sin(k, R) : -(float)ct_sin(k, R);
        return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

// ------------------------------------------------------------------------------------------
// R-point DFT in registers, in place, natural order in and out.
// ------------------------------------------------------------------------------------------
template <int R, bool INV>
struct DFT;

template <bool INV>
struct DFT<1, INV> {
    static __device__ __forceinline__ void run(float2 (&)[1]) {}
};

template <bool INV>
struct DFT<2, INV> {
    static __device__ __forceinline__ void run(float2 (&v)[2])
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV>
struct DFT<3, INV> {
    static __device__ __forceinline__ void run(float2 (&v)[3])
    {
        constexpr float h = 0.5f;
        constexpr float s3 = 0.86602540378443864676f;
        float2 t1 = cadd(v[1], v[2]);
        float2 t2 = csub(v[1], v[2]);
        float2 m1 = make_float2(v[0].x - h * t1.x, v[0].y - h * t1.y);
        float2 m2 = cmul_mi<INV>(cscale(t2, s3));
        v[0] = cadd(v[0], t1);
        v[1] = cadd(m1, m2);
        v[2] = csub(m1, m2);
    }
};

template <bool INV>
struct DFT<4, INV> {
    static __device__ __forceinline__ void run(float2 (&v)[4])
    {
        float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        float2 t2 = cadd(v[1], v[3]), t3 = cmul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

// odd prime R (5, 7, ...): symmetric pair form with folded constants
template <int R, bool INV, bool PRIME = ct_is_prime(R)>
struct DFTGeneric;

template <int R, bool INV>
struct DFTGeneric<R, INV, true> {
    static __device__ __forceinline__ void run(float2 (&v)[R])
    {
        constexpr int M = (R - 1) / 2;
        float2 s[M + 1], d[M + 1];
        float2 x0 = v[0];
        float2 sum = x0;
        static_for<1, M + 1>([&](auto nc) {
            constexpr int n = decltype(nc)::value;
            s[n] = cadd(v[n], v[R - n]);
            d[n] = csub(v[n], v[R - n]);
            sum = cadd(sum, s[n]);
        });
        static_for<1, M + 1>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            float2 A = x0;
            float2 B = make_float2(0.f, 0.f);
            static_for<1, M + 1>([&](auto nc) {
                constexpr int n = decltype(nc)::value;
                constexpr float c = (float)ct_cos(n * k, R);
                constexpr float sn = (float)ct_sin(n * k, R);
                A = make_float2(A.x + c * s[n].x, A.y + c * s[n].y);
                B = make_float2(B.x + sn * d[n].x, B.y + sn * d[n].y);
            });
            // forward: X[k] = A - iB, X[R-k] = A + iB (inverse swaps)
            float2 iB = make_float2(-B.y, B.x);
            if constexpr (INV) {
                v[k] = cadd(A, iB);
                v[R - k] = csub(A, iB);
            } else {
                v[k] = csub(A, iB);
                v[R - k] = cadd(A, iB);
            }
        });
        v[0] = sum;
    }
};

// composite R = P * Q, decimation in time:
// X[k1 + P k2] = sum_{n2} W_R^{n2 k1} W_Q^{n2 k2} sum_{n1} x[Q n1 + n2] W_P^{n1 k1}
template <int R, bool INV>
struct DFTGeneric<R, INV, false> {
    static __device__ __forceinline__ void run(float2 (&v)[R])
    {
        constexpr int P = ct_first_factor(R);
        constexpr int Q = R / P;
        float2 t[R];
        static_for<0, Q>([&](auto n2c) {
            constexpr int n2 = decltype(n2c)::value;
            float2 a[P];
            static_for<0, P>([&](auto n1c) {
                constexpr int n1 = decltype(n1c)::value;
                a[n1] = v[Q * n1 + n2];
            });
            DFT<P, INV>::run(a);
            static_for<0, P>([&](auto k1c) {
                constexpr int k1 = decltype(k1c)::value;
                t[k1 * Q + n2] = twid<R, n2 * k1, INV>(a[k1]);
            });
        });
        static_for<0, P>([&](auto k1c) {
            constexpr int k1 = decltype(k1c)::value;
            float2 b[Q];
            static_for<0, Q>([&](auto n2c) {
                constexpr int n2 = decltype(n2c)::value;
                b[n2] = t[k1 * Q + n2];
            });
            DFT<Q, INV>::run(b);
            static_for<0, Q>([&](auto k2c) {
                constexpr int k2 = decltype(k2c)::value;
                v[k1 + P * k2] = b[k2];
            });
        });
    }
};

template <int R, bool INV>
struct DFT {
    static __device__ __forceinline__ void run(float2 (&v)[R]) { DFTGeneric<R, INV>::run(v); }
};

// ------------------------------------------------------------------------------------------
// Shared-memory layout: one float2 of padding every 2^PS elements (PS = 5 by default: bank-
// conflict-free strided butterfly writes for radix 8/16; a plan whose first stage writes at
// stride 16 uses PS = 4), and a per-array stride that shifts consecutive arrays by 8 banks.
// A warp's 8-byte accesses are served per half-warp: conflict-free when the 16 padded indices of
// a half-warp are distinct modulo 16.
// ------------------------------------------------------------------------------------------
template <int PS = 5>
__device__ __forceinline__ int sidx(int i) { return i + (i >> PS); }

// array stride of L padded elements, rounded up to 16 float2 plus EX (EX = 4 by default: consecutive
// arrays 8 banks apart)
template <int L, int PS = 5, int EX = 4>
struct SmemLen {
    static constexpr int raw = L + (L >> PS) + 1;
    static constexpr int value = ((raw + 15) / 16) * 16 + EX;
};

template <int... Rs>
struct Radices {};

template <int... Rs>
constexpr int radix_product(Radices<Rs...>)
{
    return (1 * ... * Rs);
}

// ------------------------------------------------------------------------------------------
// Per-stage twiddle tables.  Stage (R, Ns) of a length-L transform multiplies input r of
// butterfly j by W_{Ns R}^{r k}, k = j mod Ns.  Its table holds those factors as [r-1][k]
// (FP64-built, rounded once), so for fixed r the threads of a warp read consecutive entries.
// A catalog lists the (R, Ns > 1) stages of every plan compiled for one L and their offsets in
// one contiguous table; kernels get the table base and find their stage's offset at compile
// time.
// ------------------------------------------------------------------------------------------
struct TwCatalog {
    int n = 0;
    int total = 0;
    int R[64] = {};
    int NS[64] = {};
    int off[64] = {};
    constexpr int find(int r, int ns) const
    {
        for (int i = 0; i < n; ++i)
            if (R[i] == r && NS[i] == ns) return off[i];
        return -1;
    }
    constexpr void add_plan(const int *rs, int nr)
    {
        int ns = 1;
        for (int i = 0; i < nr; ++i) {
            if (ns > 1 && find(rs[i], ns) < 0) {
                R[n] = rs[i];
                NS[n] = ns;
                off[n] = total;
                total += (rs[i] - 1) * ns;
                ++n;
            }
            ns *= rs[i];
        }
    }
    template <int... Rs>
    constexpr void add(Radices<Rs...>)
    {
        const int a[] = {Rs...};
        add_plan(a, (int)sizeof...(Rs));
    }
};

// The thread index read so that the compiler cannot treat it as loop-invariant: inside a
// persistent kernel's work loop, expressions of threadIdx.x would otherwise be hoisted out of
// the loop for every stage of every transform and kept live across it (register spills).
__device__ __forceinline__ int opaque_tid()
{
    int t;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(t));
    return t;
}

// One Stockham stage over B arrays of length L (array b at s + b*LP); OPQ: read the thread
// index with opaque_tid().
template <class Cat, int L, int LP, int R, int NS, bool INV, int B, int NT, int PS = 5, bool OPQ = false>
__device__ __forceinline__ void fft_stage(float2 *__restrict__ s, const float2 *__restrict__ tw)
{
    const int tid = OPQ ? opaque_tid() : (int)threadIdx.x;
    constexpr int LR = L / R;
    constexpr int TOT = B * LR;
    constexpr int NBF = (TOT + NT - 1) / NT;
    float2 v[NBF][R];
#pragma unroll
    for (int i = 0; i < NBF; ++i) {
        const int t = tid + i * NT;
        if ((NBF * NT == TOT) || t < TOT) {
            const int b = t / LR;
            const int j = t - b * LR;
            const float2 *x = s + b * LP;
#pragma unroll
            for (int r = 0; r < R; ++r) v[i][r] = x[sidx<PS>(j + r * LR)];
            if constexpr (NS > 1) {
                constexpr int OFF = Cat::off(R, NS);
                static_assert(OFF >= 0, "stage missing from the twiddle catalog");
                const float2 *t = tw + OFF + j % NS;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = __ldg(t + (r - 1) * NS);
                    if constexpr (INV) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            DFT<R, INV>::run(v[i]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NBF; ++i) {
        const int t = tid + i * NT;
        if ((NBF * NT == TOT) || t < TOT) {
            const int b = t / LR;
            const int j = t - b * LR;
            float2 *y = s + b * LP;
            const int k = j % NS;
            const int base = (j / NS) * NS * R + k;
#pragma unroll
            for (int q = 0; q < R; ++q) y[sidx<PS>(base + q * NS)] = v[i][q];
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------------------------------
// One-butterfly-per-thread building blocks (the large-grid kernels).  Butterfly j of a stage
// (radix R, Ns) reads x[j + r L/R] and writes y[(j/Ns) Ns R + j%Ns + q Ns]; with Ns = 1 the
// reads of the first stage can come straight from global memory, and the last stage's outputs
// (Ns = L/R: positions j + q L/R) can go straight back, skipping two shared-memory passes.
// ------------------------------------------------------------------------------------------
template <class Cat, int L, int R, int NS, bool INV>
__device__ __forceinline__ void bfly(float2 (&v)[R], int j, const float2 *__restrict__ tw)
{
    if constexpr (NS > 1) {
        constexpr int OFF = Cat::off(R, NS);
        static_assert(OFF >= 0, "stage missing from the twiddle catalog");
        const float2 *t = tw + OFF + j % NS;
#pragma unroll
        for (int r = 1; r < R; ++r) {
            float2 w = __ldg(t + (r - 1) * NS);
            if constexpr (INV) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
    }
    DFT<R, INV>::run(v);
}

// 1: shared-memory addresses of a butterfly as one base plus compile-time offsets where the
// padding allows it (N = 4096: rows 0.361 -> 0.348 ms, columns 0.375 -> 0.371 ms on B200)
#ifndef DNS2D_IDX
#define DNS2D_IDX 1
#endif

// Butterfly j reads x[j + r L/R].  When L/R is a multiple of G = 2^PS the padded index is
// sidx(j) + r (L/R + L/R/G): one address, the rest compile-time offsets.
template <int L, int R, int PS = 5>
__device__ __forceinline__ void sm_load(float2 (&v)[R], const float2 *__restrict__ x, int j)
{
    constexpr int LR = L / R, G = 1 << PS;
    if constexpr (DNS2D_IDX && LR % G == 0) {
        const float2 *__restrict__ b = x + sidx<PS>(j);
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = b[r * (LR + LR / G)];
    } else {
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = x[sidx<PS>(j + r * LR)];
    }
}

// Butterfly j writes y[A + k + q Ns], A = (j / Ns) Ns R, k = j % Ns.  Compile-time offsets from
// one address when the G-element padding groups (G = 2^PS) allow it:
//   Ns % G == 0:                  sidx(A + k) + q (Ns + Ns/G)
//   G % Ns == 0, (Ns R) % G == 0: A + A/G + k + q Ns + (q Ns)/G   (k + q Ns never crosses a group)
//   Ns == 1, G % R == 0:          sidx(A) + q                     (A .. A+R-1 in one group)
template <int L, int R, int NS, int PS = 5>
__device__ __forceinline__ void sm_store(float2 *__restrict__ y, const float2 (&v)[R], int j)
{
    constexpr int G = 1 << PS;
    const int k = j % NS;
    const int A = (j / NS) * NS * R;
    if constexpr (DNS2D_IDX && NS % G == 0) {
        float2 *__restrict__ b = y + sidx<PS>(A + k);
#pragma unroll
        for (int q = 0; q < R; ++q) b[q * (NS + NS / G)] = v[q];
    } else if constexpr (DNS2D_IDX && G % NS == 0 && (NS * R) % G == 0) {
        float2 *__restrict__ b = y + A + (A >> PS) + k;
#pragma unroll
        for (int q = 0; q < R; ++q) b[q * NS + ((q * NS) >> PS)] = v[q];
    } else if constexpr (DNS2D_IDX && NS == 1 && G % R == 0) {
        float2 *__restrict__ b = y + sidx<PS>(A);
#pragma unroll
        for (int q = 0; q < R; ++q) b[q] = v[q];
    } else {
        const int base = A + k;
#pragma unroll
        for (int q = 0; q < R; ++q) y[sidx<PS>(base + q * NS)] = v[q];
    }
}

// Bands known at compile time.  A first stage (Ns = 1) reads positions j + r L/R, a last stage
// (Ns = L/R) writes positions j + q L/R, j < L/R: slot r (q) covers [r L/R, r L/R + L/R - 1].
// When that whole range lies in [B0, B1] (the 3/2 padding band of a spectrum), the input is zero
// for every j, or the output is never read: loads become constants and stores are dropped, and
// the compiler removes the arithmetic that only fed them.
template <int L, int R, int B0, int B1>
__device__ __forceinline__ constexpr bool slot_in_band(int r)
{
    return r * (L / R) >= B0 && r * (L / R) + L / R - 1 <= B1;
}

// last stage (Ns = L/R) with outputs in [B0, B1] dropped
template <class Cat, int L, int R, bool INV, int B0, int B1, int PS = 5>
__device__ __forceinline__ void stage1_last_band(float2 *s, const float2 *tw)
{
    constexpr int LR = L / R;
    const int j = threadIdx.x;
    float2 v[R];
    __syncthreads();
    if (j < LR) {
        sm_load<L, R, PS>(v, s, j);
        bfly<Cat, L, R, LR, INV>(v, j, tw);
    }
    __syncthreads();
    if (j < LR) {
#pragma unroll
        for (int q = 0; q < R; ++q)
            if (!slot_in_band<L, R, B0, B1>(q)) s[sidx<PS>(j + q * LR)] = v[q];
    }
}

// smem -> smem stage, one butterfly per thread (threads >= L/R idle); in place, so reads and
// writes are separated by a barrier.  Leading barrier included; no trailing barrier.
template <class Cat, int L, int R, int NS, bool INV, int PS = 5>
__device__ __forceinline__ void stage1(float2 *s, const float2 *tw)
{
    constexpr int LR = L / R;
    const int j = threadIdx.x;
    float2 v[R];
    __syncthreads();
    if (j < LR) {
        sm_load<L, R, PS>(v, s, j);
        bfly<Cat, L, R, NS, INV>(v, j, tw);
    }
    __syncthreads();
    if (j < LR) sm_store<L, R, NS, PS>(s, v, j);
}

// asynchronous global -> shared copies (cp.async; 8-byte elements, L1-allocating)
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gmem_src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <class Cat, int L, int LP, bool INV, int B, int NT, int PS, bool OPQ, int NS, int R0, int... Rs>
__device__ __forceinline__ void fft_stages(float2 *s, const float2 *tw)
{
    fft_stage<Cat, L, LP, R0, NS, INV, B, NT, PS, OPQ>(s, tw);
    if constexpr (sizeof...(Rs) > 0) fft_stages<Cat, L, LP, INV, B, NT, PS, OPQ, NS * R0, Rs...>(s, tw);
}

// PS: the padding of sidx<PS>; OPQ: read the thread index with opaque_tid()
template <class Cat, int L, int LP, bool INV, int B, int NT, int PS = 5, bool OPQ = false, int... Rs>
__device__ __forceinline__ void fft_run(float2 *s, const float2 *tw, Radices<Rs...>)
{
    static_assert((1 * ... * Rs) == L, "radix plan does not multiply to L");
    fft_stages<Cat, L, LP, INV, B, NT, PS, OPQ, 1, Rs...>(s, tw);
}

}  // namespace dns2d
