// kernel_sets.cuh — the launch table of one compiled grid size: a KernelSet holds host functions
// that launch that size's kernels (row / column pass, set-up, diagnostics).  Launch<N> serves the
// single-CTA sizes, LaunchC<N> the 4-CTA cluster sizes.  The sets are instantiated in sets_*.cu,
// one translation unit per group of sizes, so the library compiles in parallel.
#pragma once
#include "dns2d_kernels.cuh"
#include "cluster.cuh"

namespace dns2d {

struct KernelSet {
    int N;
    int nplans;  // radix plans of the small-grid passes (AltPlans<N>::count)
    int rows_blocks;
    const TwCatalog *cat;
    cudaError_t (*setup)();
    void (*rows_step)(const Pointers &, cudaStream_t, int);
    void (*cols_step)(const Pointers &, int, int, cudaStream_t, int);
    void (*cols_init)(const Pointers &, const float2 *, int, cudaStream_t, int);
    void (*rows_velocity)(const Pointers &, float *, float *, float, cudaStream_t, int);
    void (*rows_from_phys)(const Pointers &, const float *, cudaStream_t);
    void (*cols_scalar)(const Pointers &, float2 *, int, cudaStream_t);
    void (*rows_scalar)(const Pointers &, const float2 *, float *, float2 *, cudaStream_t);
    void (*rows_fwd_scalar)(const Pointers &, const float *, float2 *, cudaStream_t);
    // forward column transform of the forcing; with GateArgs.om2 set it also decides the closure's
    // energy gate for the step
    void (*cols_fwd_scalar)(const Pointers &, const float2 *, float2 *, const GateArgs &, cudaStream_t);
    // full 2D R2C of the physical u, w planes (dump path; nullptr at the cluster sizes)
    void (*velocity_r2c_full)(const Pointers &, const float *, float2 *, cudaStream_t);
    // min / max partials rows_scalar leaves in its `mm` argument (0: none that cover its output)
    int scalar_parts;
};

template <int N>
struct Launch {
    using C = Cfg<N>;
    static constexpr size_t smB = (size_t)C::ROWS * C::LP * sizeof(float2);
    static constexpr size_t smA = (size_t)2 * C::LP * sizeof(float2);
    static constexpr size_t smA1 = (size_t)C::LP * sizeof(float2);
    static constexpr int GB = C::L / C::ROWS;

    static constexpr bool V2 = Cfg2<N>::enabled;
    static constexpr size_t sm2 = V2 ? (size_t)Cfg2<N>::LP * sizeof(float2) : 0;
    using P0 = typename C::Plan;
    using P1 = typename AltPlans<N>::P1;
    using P2 = typename AltPlans<N>::P2;

    template <class Plan>
    static cudaError_t setup_plan()
    {
        const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
        cudaError_t e;
        if ((e = cudaFuncSetAttribute(k_rows_step<N, 2, Plan>, a, (int)(2 * C::LP * sizeof(float2)))) != cudaSuccess)
            return e;
        if ((e = cudaFuncSetAttribute(k_rows_step<N, 4, Plan>, a, (int)(4 * C::LP * sizeof(float2)))) != cudaSuccess)
            return e;
        if ((e = cudaFuncSetAttribute(k_rows_step<N, 8, Plan>, a, (int)(8 * C::LP * sizeof(float2)))) != cudaSuccess)
            return e;
        return cudaFuncSetAttribute(k_cols_step<N, Plan>, a, (int)smA);
    }
    // rows per CTA (autotuned): 2, 4 or 8; the arithmetic per row is the same
    template <class Plan>
    static void rows_plan(const Pointers &p, cudaStream_t s, int ny)
    {
        const int rt = p.rows_tile ? p.rows_tile : C::ROWS;
        const size_t sm = (size_t)rt * C::LP * sizeof(float2);
        if (rt == 2) k_rows_step<N, 2, Plan><<<dim3(C::L / 2, ny), C::NTB, sm, s>>>(p);
        else if (rt == 8) k_rows_step<N, 8, Plan><<<dim3(C::L / 8, ny), C::NTB, sm, s>>>(p);
        else k_rows_step<N, 4, Plan><<<dim3(C::L / 4, ny), C::NTB, sm, s>>>(p);
    }

    static cudaError_t setup()
    {
        const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
        cudaError_t e;
        if constexpr (V2) {
            if ((e = cudaFuncSetAttribute(k_rows_step2<N>, a, (int)sm2)) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k_cols_step2<N>, a, (int)(2 * sm2))) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k_cols_step4<N>, a, (int)cols4_smem_bytes<N>())) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k_rows_velocity2<N>, a, (int)sm2)) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k_cols_scalar2<N>, a, (int)sm2)) != cudaSuccess) return e;
            if ((e = cudaFuncSetAttribute(k_rows_pair2<N>, a, (int)sm2)) != cudaSuccess) return e;
        }
        if constexpr (!V2) {  // rows per CTA x radix plan variants of the small-grid passes
            if ((e = setup_plan<P0>()) != cudaSuccess) return e;
            if ((e = setup_plan<P1>()) != cudaSuccess) return e;
            if ((e = setup_plan<P2>()) != cudaSuccess) return e;
        }
        if ((e = cudaFuncSetAttribute(k_cols_step<N>, a, (int)smA)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_init<N>, a, (int)smA)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_velocity<N>, a, (int)smB)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_from_phys<N>, a, (int)smB)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_scalar<N>, a, (int)smA1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_scalar<N>, a, (int)smB)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_fwd_scalar<N>, a, (int)smB)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_fwd_scalar<N>, a, (int)smA1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_r2c_full<N>, a, (int)smB)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_c2c_full<N>, a, (int)smA1)) != cudaSuccess) return e;
        return cudaSuccess;
    }
    static void rows_step(const Pointers &p, cudaStream_t s, int ny)
    {
        if constexpr (V2) {
            k_rows_step2<N><<<dim3(C::L, ny), Cfg2<N>::NT, sm2, s>>>(p);
        } else {
            if (p.plan_rows == 1) rows_plan<P1>(p, s, ny);
            else if (p.plan_rows == 2) rows_plan<P2>(p, s, ny);
            else rows_plan<P0>(p, s, ny);
        }
    }
    static void cols_step(const Pointers &p, int first, int slot, cudaStream_t s, int ny)
    {
        // one or two thread groups per column CTA (autotuned; the default, two, was the faster on
        // B200 at N = 1024, 2048 and 4096); both give the same arithmetic
        if constexpr (V2) {
            const int g = p.cols_groups ? p.cols_groups : 2;
            if (g == 2) k_cols_step4<N><<<dim3(C::H, ny), 2 * Cfg2<N>::NT, cols4_smem_bytes<N>(), s>>>(p, first, slot);
            else k_cols_step2<N><<<dim3(C::H, ny), Cfg2<N>::NT, 2 * sm2, s>>>(p, first, slot);
        }
        else if (p.plan_cols == 1) k_cols_step<N, P1><<<dim3(C::H, ny), C::NTA, smA, s>>>(p, first, slot);
        else if (p.plan_cols == 2) k_cols_step<N, P2><<<dim3(C::H, ny), C::NTA, smA, s>>>(p, first, slot);
        else k_cols_step<N, P0><<<dim3(C::H, ny), C::NTA, smA, s>>>(p, first, slot);
    }
    static void cols_init(const Pointers &p, const float2 *uw, int mode, cudaStream_t s, int ny)
    {
        k_cols_init<N><<<dim3(C::H, ny), C::NTA, smA, s>>>(p, uw, mode);
    }
    // the diagnostics of the large-grid sizes run on the step kernels' plan (Cfg2)
    static void rows_velocity(const Pointers &p, float *phys, float *cflm, float dx, cudaStream_t s, int ny)
    {
        if constexpr (V2) k_rows_velocity2<N><<<dim3(C::L, ny), Cfg2<N>::NT, sm2, s>>>(p, phys, cflm, dx);
        else k_rows_velocity<N><<<dim3(GB, ny), C::NTB, smB, s>>>(p, phys, cflm, dx);
    }
    static void rows_from_phys(const Pointers &p, const float *phys, cudaStream_t s)
    {
        k_rows_from_phys<N><<<GB, C::NTB, smB, s>>>(p, phys);
    }
    static void cols_scalar(const Pointers &p, float2 *scratch, int kind, cudaStream_t s)
    {
        if constexpr (V2) k_cols_scalar2<N><<<C::H, Cfg2<N>::NT, sm2, s>>>(p, scratch, kind);
        else k_cols_scalar<N><<<C::H, C::NTA, smA1, s>>>(p, scratch, kind);
    }
    // one min / max pair per CTA into mm: GB of them, or L / 2 on the large-grid plan
    static void rows_scalar(const Pointers &p, const float2 *scratch, float *out, float2 *mm, cudaStream_t s)
    {
        if constexpr (V2) k_rows_pair2<N><<<C::L / 2, Cfg2<N>::NT, sm2, s>>>(p, scratch, out, mm);
        else k_rows_scalar<N><<<GB, C::NTB, smB, s>>>(p, scratch, out, mm);
    }
    static void rows_fwd_scalar(const Pointers &p, const float *f, float2 *scratch, cudaStream_t s)
    {
        k_rows_fwd_scalar<N><<<GB, C::NTB, smB, s>>>(p, f, scratch);
    }
    static void cols_fwd_scalar(const Pointers &p, const float2 *scratch, float2 *out, const GateArgs &g,
                                cudaStream_t s)
    {
        k_cols_fwd_scalar<N><<<C::H, C::NTA, smA1, s>>>(p, scratch, out, g);
    }
    static void velocity_r2c_full(const Pointers &p, const float *phys, float2 *spec, cudaStream_t s)
    {
        k_rows_r2c_full<N><<<GB, C::NTB, smB, s>>>(p, phys, spec);
        k_cols_c2c_full<N><<<dim3(C::L / 2 + 1, 2), C::NTA, smA1, s>>>(p, spec);
    }
    static KernelSet make()
    {
        return KernelSet{N, AltPlans<N>::count, V2 ? std::max(GB, C::L / 2) : GB, &TwCat<N>::cat, setup, rows_step,
                         cols_step, cols_init,
                         rows_velocity,
                         rows_from_phys, cols_scalar, rows_scalar, rows_fwd_scalar, cols_fwd_scalar,
                         velocity_r2c_full, V2 ? C::L / 2 : GB};
    }
};

// Sizes whose rows exceed one CTA's shared memory: every transform runs on a cluster of 4 CTAs
// (cluster.cuh).  Grids are 4 CTAs per row / column; the closure's forward scalar transforms are
// not provided at these sizes.
template <int N>
struct LaunchC {
    using C = CfgC<N>;
    static constexpr size_t sm1 = (size_t)C::MP * sizeof(float2);
    static constexpr size_t sm2 = 2 * sm1;

    static cudaError_t setup()
    {
        const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
        cudaError_t e;
        if ((e = cudaFuncSetAttribute(k_rows_step_c<N>, a, (int)sm1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_step_c<N>, a, (int)sm2)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_init_c<N>, a, (int)sm2)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_velocity_c<N>, a, (int)sm1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_from_phys_c<N>, a, (int)sm1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_cols_scalar_c<N>, a, (int)sm1)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k_rows_scalar_c<N>, a, (int)sm1)) != cudaSuccess) return e;
        return cudaSuccess;
    }
    static void rows_step(const Pointers &p, cudaStream_t s, int ny)
    {
        k_rows_step_c<N><<<dim3(4 * C::L, ny), C::NT, sm1, s>>>(p);
    }
    static void cols_step(const Pointers &p, int first, int slot, cudaStream_t s, int ny)
    {
        k_cols_step_c<N><<<dim3(4 * C::H, ny), C::NT, sm2, s>>>(p, first, slot);
    }
    static void cols_init(const Pointers &p, const float2 *uw, int mode, cudaStream_t s, int ny)
    {
        k_cols_init_c<N><<<dim3(4 * C::H, ny), C::NT, sm2, s>>>(p, uw, mode);
    }
    static void rows_velocity(const Pointers &p, float *phys, float *cflm, float dx, cudaStream_t s, int ny)
    {
        k_rows_velocity_c<N><<<dim3(4 * C::L, ny), C::NT, sm1, s>>>(p, phys, cflm, dx);
    }
    static void rows_from_phys(const Pointers &p, const float *phys, cudaStream_t s)
    {
        k_rows_from_phys_c<N><<<4 * C::L, C::NT, sm1, s>>>(p, phys);
    }
    static void cols_scalar(const Pointers &p, float2 *scratch, int kind, cudaStream_t s)
    {
        k_cols_scalar_c<N><<<4 * C::H, C::NT, sm1, s>>>(p, scratch, kind);
    }
    static void rows_scalar(const Pointers &p, const float2 *scratch, float *out, float2 *mm, cudaStream_t s)
    {
        k_rows_scalar_c<N><<<4 * C::L, C::NT, sm1, s>>>(p, scratch, out, mm);
    }
    static KernelSet make()
    {
        return KernelSet{N, 1, 4 * C::L, &TwCatC<N>::cat, setup, rows_step, cols_step, cols_init, rows_velocity,
                         rows_from_phys, cols_scalar, rows_scalar, nullptr, nullptr, nullptr, 0};
    }
};


// the compiled sizes, by translation unit (nullptr: N is not in that unit)
const KernelSet *kernel_sets_small(int N);    // 16 ... 128 (sets_small.cu)
const KernelSet *kernel_sets_256(int N);      // 256, 512 (sets_256.cu)
const KernelSet *kernel_sets_mid(int N);      // 1024, 2048 (sets_mid.cu)
const KernelSet *kernel_sets_4096(int N);     // 4096 (sets_4096.cu)
const KernelSet *kernel_sets_cluster(int N);  // 840, 8192, 9216 (sets_cluster.cu)
const KernelSet *kernel_sets_16384(int N);    // 16384 (sets_16384.cu)
const KernelSet *kernel_sets_29400(int N);    // 29400 (sets_29400.cu)

}  // namespace dns2d
