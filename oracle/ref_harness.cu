// ref_harness.cu — TEST INFRASTRUCTURE ONLY.
//
// Drives the reference solver (cudaturbo's cuFFT path, linked from its own unmodified
// object files built by oracle/Makefile into oracle/_ref/) from a given initial vorticity field,
// so the CUDA product can be compared with the reference field by field.  Only the reference's
// public solver API of cuda/cuda_dns.h is called, in the order of its mem_cuda loop
// (cuda/mem_cuda.cu:1767-1897):
//   start-up : velocity recovery through dnsCudaStep3 with dt = 0 (om' = om, FN = 0 from a
//              zeroed UC), dnsCudaStep2A, next_dt_gpu (init branch)
//   each step: dnsCudaStep2B, dnsCudaStep3, dnsCudaStep2A, t += dt_old,
//              at it == 1, it % UPDATE == 0, it == STEPS: next_dt_gpu + dnsCudaOm2Phys
// Usage: ref_harness N Re K0 CFL STEPS UPDATE om2_in.bin out_prefix [TIMED_STEPS]
//   om2_in.bin: [N][N/2] complex64.  Writes out_prefix.om2 / .fnm1 ([N][N/2] complex64) and
//   prints one "STEP it E Z" line per step (FP64 energy/enstrophy of OM2 after the step) and a
//   "DIAG it t dt cn cflm sigma" line per diagnostic step.  With TIMED_STEPS > 0 it instead
//   runs that many steps after the STEPS warm-up and prints "TIMING steps seconds".
#include "cuda_dns.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <string>
#include <vector>

static double display_sigma(const std::vector<float> &h)
{
    float mn = h[0], mx = h[0];
    for (float v : h) {
        mn = std::min(mn, v);
        mx = std::max(mx, v);
    }
    const float rng = mx - mn;
    double s = 0, s2 = 0;
    for (float v : h) {
        int pix = 128;
        if (std::fabs(rng) > 1.0e-12f) {
            float pf = 1.0f + ((v - mn) / rng) * 254.0f;
            pf = std::min(255.0f, std::max(1.0f, pf));
            pix = (int)pf;
        }
        s += pix;
        s2 += (double)pix * pix;
    }
    const double n = (double)h.size(), mean = s / n;
    return std::sqrt(std::max(0.0, s2 / n - mean * mean));
}

static void energy(const DnsDeviceState &S, double &E, double &Z)
{
    const int N = S.Nbase, H = N / 2;
    std::vector<cplx> om((size_t)N * H);
    cudaMemcpy(om.data(), S.d_om2, om.size() * sizeof(cplx), cudaMemcpyDeviceToHost);
    E = Z = 0.0;
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const int kz = (iz < H) ? iz : iz - N;
            const double k2 = (double)ix * ix + (double)kz * kz;
            const cplx o = om[(size_t)iz * H + ix];
            const double p = (double)o.x * o.x + (double)o.y * o.y;
            const double w = (ix == 0) ? 0.5 : 1.0;
            Z += w * p;
            if (k2 > 0) E += w * p / k2;
        }
}

int main(int argc, char **argv)
{
    if (argc < 9) {
        std::fprintf(stderr, "usage: %s N Re K0 CFL STEPS UPDATE om2_in.bin out_prefix [TIMED_STEPS]\n", argv[0]);
        return 2;
    }
    const int N = std::atoi(argv[1]);
    const float Re = (float)std::atof(argv[2]), K0 = (float)std::atof(argv[3]), CFL = (float)std::atof(argv[4]);
    const int STEPS = std::atoi(argv[5]), UPDATE = std::atoi(argv[6]);
    const int TIMED = (argc > 9) ? std::atoi(argv[9]) : 0;
    const int H = N / 2;
    DnsDeviceState S{};
    if (!dnsCudaCreate(&S, N, Re, K0)) return 1;
    S.cflnum = CFL;
    S.ifn = 1;
    S.it = 0;
    S.dt = 0.0f;
    S.cn = 1.0f;
    S.cnm1 = 0.0f;
    S.visc = float(1.0 / S.Re);

    std::vector<cplx> om((size_t)N * H);
    FILE *fp = std::fopen(argv[7], "rb");
    if (!fp || std::fread(om.data(), sizeof(cplx), om.size(), fp) != om.size()) {
        std::fprintf(stderr, "cannot read %s\n", argv[7]);
        return 1;
    }
    std::fclose(fp);
    cudaMemcpy(S.d_om2, om.data(), om.size() * sizeof(cplx), cudaMemcpyHostToDevice);
    cudaMemset(S.d_fnm1, 0, om.size() * sizeof(cplx));
    cudaMemset(S.d_uc_full, 0, (size_t)S.NZ_full * S.NK_full * 3 * sizeof(cplx));
    // velocity recovery with the reference's own STEP3 at dt = 0
    dnsCudaStep3(&S);
    S.cnm1 = 0.0f;
    cudaMemset(S.d_fnm1, 0, om.size() * sizeof(cplx));
    dnsCudaStep2A(&S);
    next_dt_gpu(&S);

    const size_t plane = (size_t)S.NX_full * S.NZ_full;
    std::vector<float> w(plane);
    if (TIMED > 0) {
        for (int it = 1; it <= STEPS + TIMED; ++it) {
            if (it == STEPS + 1) {
                cudaDeviceSynchronize();
            }
            static std::chrono::steady_clock::time_point t0;
            if (it == STEPS + 1) t0 = std::chrono::steady_clock::now();
            S.it = it;
            const float dt_old = S.dt;
            dnsCudaStep2B(&S);
            dnsCudaStep3(&S);
            dnsCudaStep2A(&S);
            S.t += dt_old;
            if (it == 1 || it % UPDATE == 0) {
                next_dt_gpu(&S);
                dnsCudaOm2Phys(&S);
            }
            if (it == STEPS + TIMED) {
                cudaDeviceSynchronize();
                const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                std::printf("TIMING %d %.9f\n", TIMED, sec);
            }
        }
        dnsCudaDestroy(&S);
        return 0;
    }
    for (int it = 1; it <= STEPS; ++it) {
        S.it = it;
        const float dt_old = S.dt;
        dnsCudaStep2B(&S);
        dnsCudaStep3(&S);
        dnsCudaStep2A(&S);
        S.t += dt_old;
        double E, Z;
        energy(S, E, Z);
        std::printf("STEP %d %.17g %.17g\n", it, E, Z);
        if (it == 1 || it % UPDATE == 0 || it == STEPS) {
            next_dt_gpu(&S);
            dnsCudaOm2Phys(&S);
            cudaMemcpy(w.data(), S.d_ur_full + 2 * plane, plane * sizeof(float), cudaMemcpyDeviceToHost);
            std::printf("DIAG %d %.10g %.10g %.10g %.10g %.6f\n", it, (double)S.t, (double)S.dt, (double)S.cn,
                        (double)S.cflm, display_sigma(w));
        }
    }
    cudaMemcpy(om.data(), S.d_om2, om.size() * sizeof(cplx), cudaMemcpyDeviceToHost);
    std::string p = std::string(argv[8]) + ".om2";
    fp = std::fopen(p.c_str(), "wb");
    std::fwrite(om.data(), sizeof(cplx), om.size(), fp);
    std::fclose(fp);
    cudaMemcpy(om.data(), S.d_fnm1, om.size() * sizeof(cplx), cudaMemcpyDeviceToHost);
    p = std::string(argv[8]) + ".fnm1";
    fp = std::fopen(p.c_str(), "wb");
    std::fwrite(om.data(), sizeof(cplx), om.size(), fp);
    std::fclose(fp);
    const cudaError_t e = cudaDeviceSynchronize();
    dnsCudaDestroy(&S);
    return e == cudaSuccess ? 0 : 1;
}
