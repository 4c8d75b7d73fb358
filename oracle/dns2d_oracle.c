/*
 * dns2d_oracle.c — TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * FP64 CPU restatement of cudaturbo's 2D pseudo-spectral vorticity time step on the
 * periodic [0,2pi]^2 box.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load this library, as the checker; nothing in the product links or calls it.
 *
 * It follows the reference scheme step by step, in double precision for the fields:
 *   STEP2B  cuda/step2b_cuda.cu:137-173 (u^2, w^2, uw), :232-276 (forward 2D R2C, zero row N)
 *   STEP3   cuda/step3_cuda.cu:35-139 (FN, Crank-Nicolson/AB2 update, FNM1<-FN, velocity)
 *           and :172 (host CNM1 <- CN)
 *   STEP2A  cuda/step2a_cuda.cu:59-82 (dealias kx in [N/2,3N/4]), :135-161 (reshuffle),
 *           cuda/vfft_cuda.cu:14-26 (inverse 2D C2R, batch 2)
 *   NEXTDT  cuda/dns_cuda.cu:486-580 (CFLM max, init branch, cn/dt update; float scalars)
 *   CALCOM  cuda/calcom_cuda.cu:84-132
 *   PAO     cuda/pao_km3_cuda.cu:36-498 (host FP32/FP64 initial condition, printed stats)
 *   OM2PHYS cuda/om2phys_cuda.cu:153-205, display sigma cuda/mem_cuda.cu:652-818
 *   spectrum cuda/mem_cuda.cu:575-649 (energy_spectrum.csv binning)
 * The scalar bookkeeping (dt, cn, cnm1, t) stays in float exactly like the reference host code,
 * so printed T/DT/CN digits can be compared.  cuFFT is replaced by an own mixed-radix
 * (2,3,4,5,7, generic) Stockham FFT in FP64, validated against numpy.fft by the tests.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex zc;

/* ------------------------------------------------------------------------------------------ */
/* Mixed-radix Stockham FFT (FP64).                                                            */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int L;
    int nst;
    int radix[40];
    zc *tw; /* W_L^j = exp(-2 pi i j / L), j in [0, L) */
} orc_fft;

static const double TWO_PI = 6.283185307179586476925286766559;

static orc_fft *fft_plan(int L)
{
    orc_fft *p = (orc_fft *)calloc(1, sizeof(orc_fft));
    p->L = L;
    int m = L;
    /* Prefer radix 4, then 2, 3, 5, 7, then any remaining prime factor (generic DFT). */
    while (m % 4 == 0) { p->radix[p->nst++] = 4; m /= 4; }
    while (m % 2 == 0) { p->radix[p->nst++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->radix[p->nst++] = f; m /= f; }
    }
    p->tw = (zc *)malloc(sizeof(zc) * (size_t)L);
    for (int j = 0; j < L; ++j) {
        double a = TWO_PI * (double)j / (double)L;
        p->tw[j] = CMPLX(cos(a), -sin(a));
    }
    return p;
}

static void fft_free(orc_fft *p)
{
    if (!p) return;
    free(p->tw);
    free(p);
}

/* One Stockham pass: x -> y, radix R, Ns = product of earlier radices; sign -1 forward. */
static void fft_pass(const orc_fft *p, int R, int Ns, const zc *x, zc *y, int inverse)
{
    const int L = p->L;
    const int LR = L / R;
    const int tstep = L / (Ns * R);
    zc v[64], o[64];
    zc wr[64];
    for (int q = 0; q < R; ++q) {
        zc w = p->tw[(size_t)((long long)q * (L / R) % L)];
        wr[q] = inverse ? conj(w) : w;
    }
    for (int j = 0; j < LR; ++j) {
        const int k = j % Ns;
        for (int r = 0; r < R; ++r) {
            zc a = x[j + r * LR];
            if (r && k) {
                zc w = p->tw[r * k * tstep];
                a *= inverse ? conj(w) : w;
            }
            v[r] = a;
        }
        if (R == 2) {
            o[0] = v[0] + v[1];
            o[1] = v[0] - v[1];
        } else if (R == 4) {
            zc t0 = v[0] + v[2], t1 = v[0] - v[2];
            zc t2 = v[1] + v[3], t3 = v[1] - v[3];
            zc t3r = inverse ? (I * t3) : (-I * t3);
            o[0] = t0 + t2;
            o[2] = t0 - t2;
            o[1] = t1 + t3r;
            o[3] = t1 - t3r;
        } else if (R == 3) {
            const double s3 = 0.86602540378443864676372317075294;
            zc t1 = v[1] + v[2], t2 = v[1] - v[2];
            zc m1 = v[0] - 0.5 * t1;
            zc m2 = (inverse ? I : -I) * s3 * t2;
            o[0] = v[0] + t1;
            o[1] = m1 + m2;
            o[2] = m1 - m2;
        } else {
            for (int q = 0; q < R; ++q) {
                zc s = 0;
                for (int r = 0; r < R; ++r) s += v[r] * wr[(r * q) % R];
                o[q] = s;
            }
        }
        const int base = (j / Ns) * Ns * R + k;
        for (int q = 0; q < R; ++q) y[base + q * Ns] = o[q];
    }
}

/* In-place transform of data[0..L) using scratch[0..L).  Unnormalised in both directions. */
static void fft_exec(const orc_fft *p, zc *data, zc *scratch, int inverse)
{
    zc *a = data, *b = scratch;
    int Ns = 1;
    for (int s = 0; s < p->nst; ++s) {
        fft_pass(p, p->radix[s], Ns, a, b, inverse);
        Ns *= p->radix[s];
        zc *t = a; a = b; b = t;
    }
    if (a != data) memcpy(data, a, sizeof(zc) * (size_t)p->L);
}

/* Exported 1D C2C for the numpy cross-check (double interleaved re/im). */
void orc_fft_c2c(int L, const double *in, double *out, int inverse)
{
    orc_fft *p = fft_plan(L);
    zc *d = (zc *)malloc(sizeof(zc) * (size_t)L);
    zc *s = (zc *)malloc(sizeof(zc) * (size_t)L);
    for (int i = 0; i < L; ++i) d[i] = CMPLX(in[2 * i], in[2 * i + 1]);
    fft_exec(p, d, s, inverse);
    for (int i = 0; i < L; ++i) { out[2 * i] = creal(d[i]); out[2 * i + 1] = cimag(d[i]); }
    free(d); free(s); fft_free(p);
}

/* ------------------------------------------------------------------------------------------ */
/* 2D transforms on the 3/2 grid in the reference layouts (cuda/cuda_dns.h:27-34):             */
/*   UR[c][z][x] (x fastest, L x L real), UC[c][z][kx] (kx fastest, L x Nk complex).            */
/* ------------------------------------------------------------------------------------------ */

/* forward R2C 2D of one real plane -> one complex plane (unnormalised, e^{-ikx}) */
static void fwd2d(const orc_fft *p, int Nk, const double *ur, zc *uc)
{
    const int L = p->L;
    /* rows: two real rows packed per complex FFT */
#pragma omp parallel
    {
        zc *d = (zc *)malloc(sizeof(zc) * (size_t)L);
        zc *s = (zc *)malloc(sizeof(zc) * (size_t)L);
#pragma omp for schedule(static)
        for (int z0 = 0; z0 < L; z0 += 2) {
            const int z1 = (z0 + 1 < L) ? z0 + 1 : -1;
            for (int x = 0; x < L; ++x)
                d[x] = ur[(size_t)z0 * L + x] + I * (z1 >= 0 ? ur[(size_t)z1 * L + x] : 0.0);
            fft_exec(p, d, s, 0);
            for (int k = 0; k < Nk; ++k) {
                zc a = d[k], b = conj(d[(L - k) % L]);
                uc[(size_t)z0 * Nk + k] = 0.5 * (a + b);
                if (z1 >= 0) uc[(size_t)z1 * Nk + k] = -0.5 * I * (a - b);
            }
        }
        free(d); free(s);
    }
    /* columns */
#pragma omp parallel
    {
        zc *d = (zc *)malloc(sizeof(zc) * (size_t)L);
        zc *s = (zc *)malloc(sizeof(zc) * (size_t)L);
#pragma omp for schedule(static)
        for (int k = 0; k < Nk; ++k) {
            for (int z = 0; z < L; ++z) d[z] = uc[(size_t)z * Nk + k];
            fft_exec(p, d, s, 0);
            for (int z = 0; z < L; ++z) uc[(size_t)z * Nk + k] = d[z];
        }
        free(d); free(s);
    }
}

/* inverse C2R 2D of one complex plane -> one real plane (unnormalised, e^{+ikx}).
 * Like a C2R transform, the imaginary parts of the kx = 0 and kx = L/2 entries are dropped
 * after the column pass. The input plane is left unchanged. */
static void inv2d(const orc_fft *p, int Nk, const zc *uc_in, double *ur)
{
    const int L = p->L;
    zc *tmp = (zc *)malloc(sizeof(zc) * (size_t)L * Nk);
#pragma omp parallel
    {
        zc *d = (zc *)malloc(sizeof(zc) * (size_t)L);
        zc *s = (zc *)malloc(sizeof(zc) * (size_t)L);
#pragma omp for schedule(static)
        for (int k = 0; k < Nk; ++k) {
            for (int z = 0; z < L; ++z) d[z] = uc_in[(size_t)z * Nk + k];
            fft_exec(p, d, s, 1);
            for (int z = 0; z < L; ++z) tmp[(size_t)z * Nk + k] = d[z];
        }
        free(d); free(s);
    }
#pragma omp parallel
    {
        zc *d = (zc *)malloc(sizeof(zc) * (size_t)L);
        zc *s = (zc *)malloc(sizeof(zc) * (size_t)L);
#pragma omp for schedule(static)
        for (int z0 = 0; z0 < L; z0 += 2) {
            const int z1 = (z0 + 1 < L) ? z0 + 1 : -1;
            for (int x = 0; x < L; ++x) d[x] = 0;
            for (int k = 0; k < Nk; ++k) {
                zc a = tmp[(size_t)z0 * Nk + k];
                zc b = (z1 >= 0) ? tmp[(size_t)z1 * Nk + k] : 0;
                if (k == 0 || 2 * k == L) { a = creal(a); b = creal(b); }
                d[k] += a + I * b;
                if (k != 0 && 2 * k != L) d[L - k] += conj(a) + I * conj(b);
            }
            fft_exec(p, d, s, 1);
            for (int x = 0; x < L; ++x) {
                ur[(size_t)z0 * L + x] = creal(d[x]);
                if (z1 >= 0) ur[(size_t)z1 * L + x] = cimag(d[x]);
            }
        }
        free(d); free(s);
    }
    free(tmp);
}

/* ------------------------------------------------------------------------------------------ */
/* Solver state                                                                                */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
    int N, H, L, Nk;
    float Re, K0, visc, t, dt, cn, cnm1, cflnum, cflm;
    int it, ifn;
    int f32_cn; /* 1: Crank-Nicolson factors rounded in float as the reference's STEP3 forms them */
    double *ur;  /* [3][L][L] */
    zc *uc;      /* [3][L][Nk] */
    zc *om2;     /* [N][H] compact, ix fastest */
    zc *fnm1;    /* [N][H] */
    orc_fft *pl;
    double last_E, last_Z; /* energy/enstrophy of om2 after the latest STEP3 */
} orc_state;

#define UR(S, c, z, x) ((S)->ur[((size_t)(c) * (S)->L + (size_t)(z)) * (S)->L + (size_t)(x)])
#define UC(S, c, z, k) ((S)->uc[((size_t)(c) * (S)->L + (size_t)(z)) * (S)->Nk + (size_t)(k)])

orc_state *orc_create(int N, float Re, float K0, float cflnum)
{
    if (N < 4 || (N % 4) != 0) return NULL;
    orc_state *S = (orc_state *)calloc(1, sizeof(orc_state));
    S->N = N; S->H = N / 2; S->L = 3 * N / 2; S->Nk = 3 * N / 4 + 1;
    S->Re = Re; S->K0 = K0; S->visc = 1.0f / Re;
    S->t = 0.0f; S->dt = 0.0f; S->cn = 1.0f; S->cnm1 = 0.0f; S->cflnum = cflnum;
    S->it = 0; S->ifn = 1;
    const size_t L = (size_t)S->L;
    S->ur = (double *)calloc(3 * L * L, sizeof(double));
    S->uc = (zc *)calloc(3 * L * (size_t)S->Nk, sizeof(zc));
    S->om2 = (zc *)calloc((size_t)N * S->H, sizeof(zc));
    S->fnm1 = (zc *)calloc((size_t)N * S->H, sizeof(zc));
    S->pl = fft_plan(S->L);
    if (!S->ur || !S->uc || !S->om2 || !S->fnm1) return NULL;
    return S;
}

void orc_destroy(orc_state *S)
{
    if (!S) return;
    free(S->ur); free(S->uc); free(S->om2); free(S->fnm1);
    fft_free(S->pl);
    free(S);
}

/* wavenumbers of the compact grid (cuda/pao_km3_cuda.cu:84-92, cuda/step3_cuda.cu:57-58) */
static inline int kz_of(int iz, int N) { return (iz < N / 2) ? iz : iz - N; }

/* ---- STEP2B (cuda/step2b_cuda.cu:137-173, :232-276) ---- */
static void step2b(orc_state *S)
{
    const size_t plane = (size_t)S->L * S->L;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < plane; ++i) {
        const double u = S->ur[i], w = S->ur[plane + i];
        S->ur[2 * plane + i] = u * w;
        S->ur[i] = u * u;
        S->ur[plane + i] = w * w;
    }
    for (int c = 0; c < 3; ++c)
        fwd2d(S->pl, S->Nk, S->ur + c * plane, S->uc + (size_t)c * S->L * S->Nk);
    for (int c = 0; c < 3; ++c)
        for (int kx = 0; kx < S->H; ++kx) UC(S, c, S->N, kx) = 0;
}

/* ---- STEP3 (cuda/step3_cuda.cu:35-139, host CNM1 <- CN at :172) ---- */
static void step3(orc_state *S)
{
    const int N = S->N, H = S->H;
    const double divxz = 1.0 / ((double)S->L * (double)S->L);
    const double visc = S->visc, dt = S->dt, cnm1 = S->cnm1;
    double E = 0.0, Z = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : E, Z)
    for (int iz = 0; iz < N; ++iz) {
        for (int ix = 0; ix < H; ++ix) {
            const size_t io = (size_t)iz * H + ix;
            const double ax = ix, gz = kz_of(iz, N);
            const double K2 = ax * ax + gz * gz;
            const int zspec = (iz < N / 2) ? iz : iz + N / 2;
            const zc u1 = UC(S, 0, zspec, ix), u2 = UC(S, 1, zspec, ix), u3 = UC(S, 2, zspec, ix);
            const zc FN = (gz * ax * (u1 - u2) + (gz * gz - ax * ax) * u3) * divxz;
            zc om;
            if (S->f32_cn) {
                /* the reference's float factors (cuda/step3_cuda.cu:82-91): VT, ARG, DEN, c1, c2, c3
                 * each rounded to float in its operation order; the update itself in double */
                const float VT = 0.5f * S->visc * S->dt;
                const float ARG = VT * ((float)ix * (float)ix + (float)gz * (float)gz);
                const float DEN = 1.0f + ARG, c1 = 1.0f - ARG;
                const float c2 = 0.5f * S->dt * (2.0f + S->cnm1), c3 = -0.5f * S->dt * S->cnm1;
                om = ((double)c1 * S->om2[io] + (double)c2 * FN + (double)c3 * S->fnm1[io]) / (double)DEN;
            } else {
                const double ARG = 0.5 * visc * dt * K2;
                const double DEN = 1.0 + ARG;
                om = ((1.0 - ARG) * S->om2[io] + 0.5 * dt * (2.0 + cnm1) * FN - 0.5 * dt * cnm1 * S->fnm1[io]) / DEN;
            }
            S->om2[io] = om;
            S->fnm1[io] = FN;
            zc o1 = 0, o2 = 0;
            if (ix >= 1) {
                const zc v = om / (K2 + 1.0e-30);
                o1 = -I * gz * v;
                o2 = I * ax * v;
            } else if (iz >= 1 && gz != 0.0) {
                o1 = -I * om / gz;
            }
            UC(S, 0, iz, ix) = o1;
            UC(S, 1, iz, ix) = o2;
            const double wgt = (ix == 0) ? 1.0 : 2.0;
            const double p = creal(om) * creal(om) + cimag(om) * cimag(om);
            Z += 0.5 * wgt * p;
            if (K2 > 0.0) E += 0.5 * wgt * p / K2;
        }
    }
    S->last_E = E;
    S->last_Z = Z;
    S->cnm1 = S->cn;
}

/* ---- STEP2A (cuda/step2a_cuda.cu:59-82, :135-161, cuda/vfft_cuda.cu:14-26) ---- */
static void step2a(orc_state *S)
{
    const int N = S->N;
    for (int c = 0; c < 2; ++c) {
        for (int z = 0; z < S->L; ++z)
            for (int kx = N / 2; kx <= 3 * N / 4 && kx < S->Nk; ++kx) UC(S, c, z, kx) = 0;
        for (int tz = 0; tz < N / 2; ++tz)
            for (int x = 0; x < N / 2; ++x) {
                UC(S, c, tz + N, x) = UC(S, c, tz + N / 2, x);
                UC(S, c, tz + N / 2, x) = 0;
            }
    }
    const size_t plane = (size_t)S->L * S->L;
    for (int c = 0; c < 2; ++c)
        inv2d(S->pl, S->Nk, S->uc + (size_t)c * S->L * S->Nk, S->ur + c * plane);
}

/* ---- NEXTDT (cuda/dns_cuda.cu:486-580) ---- */
static float cflm_of(const orc_state *S)
{
    const float PI = 3.14159265358979323846f;
    const double DX = (double)(2.0f * PI / (float)S->N);
    const size_t plane = (size_t)S->L * S->L;
    double m = 0.0;
#pragma omp parallel for schedule(static) reduction(max : m)
    for (size_t i = 0; i < plane; ++i) {
        const double a = fabs(S->ur[i]) / DX + fabs(S->ur[plane + i]) / DX;
        if (a > m) m = a;
    }
    return (float)m;
}

static void next_dt(orc_state *S)
{
    const float PI = 3.14159265358979323846f;
    if (S->it == 0 && S->dt == 0.0f) {
        const float CFLM = cflm_of(S);
        S->dt = S->cflnum / CFLM / PI;
        S->cflm = CFLM;
        return;
    }
    if (S->ifn > 0 && (S->it % S->ifn) == 0) {
        const float CFLM = cflm_of(S);
        const float CFL = CFLM * S->dt * PI;
        S->cn = 0.8f + 0.2f * (S->cflnum / CFL);
        S->dt = S->dt * S->cn;
        S->cflm = CFLM;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Initial conditions                                                                          */
/* ------------------------------------------------------------------------------------------ */

/* PAO-k^-3 host initialiser, transcribed from cuda/pao_km3_cuda.cu:36-424 with the same
 * float/double types.  out_uw: compact spectral velocity [z][x][2] complex float (u1,u3),
 * stats: the 19 printed values (Re, Energy, WiWi, Epsilon, a11, e11, Time scale,
 * Kolmogorov, Viscosity, dx/Kol, 2Pi/Nlamda, 2Pi/Lux, 2Pi/Luz, 2Pi/Lwx, 2Pi/Lwz,
 * Deps, Ceps2, E1, E3); seed_out: the final LCG seed ("PAO seed"). */
static float pao_frand(int *seed)
{
    const int IMM = 420029, IT = 2017, ID = 5011;
    *seed = (*seed * IMM + IT) % ID;
    return (float)(*seed) / (float)ID;
}

static double pao_hash01(int x, int z, int seed, int salt)
{
    const double a = ((double)x + 1.0) * 12.9898 + ((double)z + 1.0) * 78.233 +
                     ((double)seed + 1.0) * 0.010001 + ((double)salt + 1.0) * 37.719;
    const double s = sin(a) * 43758.5453123;
    return s - floor(s);
}

int orc_pao_spectrum(int N, float K0, float Re, float *out_uw, double *stats, int *seed_out)
{
    const int NE = N, ND2 = N / 2, NED2 = NE / 2;
    const float PI = 3.14159265358979f;
    const float DXZ = 2.0f * PI / (float)N;
    const float NORM = PI * K0 * K0;
    const float AMP2_FLOOR = 1.0e-40f;
    float *alfa = (float *)malloc(sizeof(float) * ND2);
    float *gamma = (float *)malloc(sizeof(float) * NE);
    const float E1 = 1.0f, E3 = 1.0f / E1;
    const float DALFA = 1.0f / E1, DGAMMA = 1.0f / E3;
    for (int x = 0; x < NED2; ++x) alfa[x] = (float)x * DALFA;
    gamma[0] = 0.0f;
    for (int z = 1; z <= NED2; ++z) {
        gamma[z] = (float)z * DGAMMA;
        gamma[NE - z] = -gamma[z];
    }
    /* UR(x,z,c) complex float, index c + 2*(x + ND2*z) */
    float complex *U = (float complex *)calloc((size_t)ND2 * NE * 2, sizeof(float complex));
#define URAT(x, z, c) U[(size_t)(c) + 2 * ((size_t)(x) + (size_t)ND2 * (size_t)(z))]
    const int seed_init = 1;
    int seed = seed_init;
    float RANVEC[97];
    for (int i = 0; i < 97; ++i) pao_frand(&seed);
    for (int i = 0; i < 97; ++i) RANVEC[i] = pao_frand(&seed);

    for (int z = 0; z < NE; ++z) {
        for (int x = 0; x < NED2; ++x) {
            float r = pao_frand(&seed);
            int idx = (int)(r * 97.0f);
            if (idx < 0) idx = 0;
            if (idx > 96) idx = 96;
            float rv = RANVEC[idx];
            RANVEC[idx] = r;
            float th = 2.0f * PI * rv;
            float cr = cosf(th), ci = sinf(th);
            float ax = alfa[x], gz = gamma[z];
            float K = sqrtf(ax * ax + gz * gz);
            if (ax == 0.0f) {
                URAT(x, z, 1) = 0.0f;
                float ABSU2 = expf(-(K / K0) * (K / K0)) / NORM;
                if (ABSU2 < AMP2_FLOOR) ABSU2 = AMP2_FLOOR;
                float amp = sqrtf(ABSU2);
                URAT(x, z, 0) = CMPLXF(amp * cr, amp * ci);
            } else {
                float denom = 1.0f + (gz * gz) / (ax * ax);
                float ABSW2 = expf(-(K / K0) * (K / K0)) / (denom * NORM);
                if (ABSW2 < AMP2_FLOOR) ABSW2 = AMP2_FLOOR;
                float ampw = sqrtf(ABSW2);
                float wr = ampw * cr, wi = ampw * ci;
                float f = -(gz / ax);
                URAT(x, z, 1) = CMPLXF(wr, wi);
                URAT(x, z, 0) = CMPLXF(f * wr, f * wi);
            }
        }
    }
    URAT(0, 0, 0) = 0.0f;
    URAT(0, 0, 1) = 0.0f;
    for (int z = 1; z < NED2; ++z) {
        URAT(0, NE - z, 0) = conjf(URAT(0, z, 0));
        URAT(0, NE - z, 1) = conjf(URAT(0, z, 1));
    }
    for (int x = 0; x < ND2; ++x) {
        URAT(x, NED2, 0) = 0.0f;
        URAT(x, NED2, 1) = 0.0f;
    }
    /* k^-3 reshaping (cuda/pao_km3_cuda.cu:176-335) */
    {
        const double k_nyquist = (double)ND2;
        const int kmax_shell = ND2;
        double *shell_energy = (double *)calloc((size_t)kmax_shell + 1, sizeof(double));
        double *shell_weight = (double *)calloc((size_t)kmax_shell + 1, sizeof(double));
        double *target_shell = (double *)calloc((size_t)kmax_shell + 1, sizeof(double));
        for (int x = 0; x < ND2; ++x) {
            const double m = (x == 0) ? 1.0 : 2.0;
            const double ax2 = (double)alfa[x] * (double)alfa[x];
            for (int z = 0; z < NE; ++z) {
                const double gz = (double)gamma[z];
                const double k = sqrt(ax2 + gz * gz);
                const int shell = (int)(k + 0.5);
                const float complex U1 = URAT(x, z, 0), U3 = URAT(x, z, 1);
                const double u1u1 = (double)crealf(U1) * (double)crealf(U1) +
                                    (double)cimagf(U1) * (double)cimagf(U1);
                const double u3u3 = (double)crealf(U3) * (double)crealf(U3) +
                                    (double)cimagf(U3) * (double)cimagf(U3);
                if (k > 0.0 && k <= k_nyquist && shell <= kmax_shell) {
                    int z_hash = z;
                    if (x == 0 && z > NED2) z_hash = NE - z;
                    const double jit = 0.75 + 0.50 * pao_hash01(x, z_hash, seed_init, 17);
                    shell_energy[shell] += m * (u1u1 + u3u3);
                    shell_weight[shell] += m * jit;
                }
            }
        }
        const double k0 = (double)K0 > 1.0 ? (double)K0 : 1.0;
        for (int shell = 1; shell <= kmax_shell; ++shell) {
            const double k = (double)shell;
            double shape;
            if (k < k0) {
                const double low = k / k0;
                shape = (low * low * low * low) / (k0 * k0 * k0);
            } else {
                shape = 1.0 / (k * k * k);
            }
            target_shell[shell] = shape;
        }
        double original_energy = 0.0, target_energy = 0.0;
        for (int shell = 1; shell <= kmax_shell; ++shell) {
            original_energy += shell_energy[shell];
            target_energy += target_shell[shell];
        }
        if (original_energy > 0.0 && target_energy > 0.0) {
            const double norm = original_energy / target_energy;
            for (int x = 0; x < ND2; ++x) {
                const double ax = (double)alfa[x];
                const double ax2 = ax * ax;
                for (int z = 0; z < NE; ++z) {
                    const double gz = (double)gamma[z];
                    const double gz2 = gz * gz;
                    const double k = sqrt(ax2 + gz2);
                    const int shell = (int)(k + 0.5);
                    if (k > 0.0 && k <= k_nyquist && shell <= kmax_shell && shell_weight[shell] > 0.0) {
                        int z_hash = z;
                        double phase_sign = 1.0;
                        if (x == 0 && z > NED2) { z_hash = NE - z; phase_sign = -1.0; }
                        const double jit = 0.75 + 0.50 * pao_hash01(x, z_hash, seed_init, 17);
                        const double mode_energy = (norm * target_shell[shell]) * jit / shell_weight[shell];
                        const double th = phase_sign * 2.0 * 3.14159265358979323846 *
                                          pao_hash01(x, z_hash, seed_init, 53);
                        const float pr = (float)cos(th), pi_ = (float)sin(th);
                        if (ax == 0.0) {
                            const float a = (float)sqrt(mode_energy);
                            URAT(x, z, 0) = CMPLXF(a * pr, a * pi_);
                            URAT(x, z, 1) = 0.0f;
                        } else {
                            const double denom = 1.0 + gz2 / ax2;
                            const float a = (float)sqrt(mode_energy / denom);
                            const float wr = a * pr, wi = a * pi_;
                            const float f = (float)(-gz / ax);
                            URAT(x, z, 0) = CMPLXF(f * wr, f * wi);
                            URAT(x, z, 1) = CMPLXF(wr, wi);
                        }
                    } else {
                        URAT(x, z, 0) = 0.0f;
                        URAT(x, z, 1) = 0.0f;
                    }
                }
            }
        }
        free(shell_energy); free(shell_weight); free(target_shell);
    }
    /* averages (cuda/pao_km3_cuda.cu:345-424) */
    double A1 = 0, A2 = 0, A3 = 0, A4 = 0, A5 = 0, A6 = 0, A7 = 0, E110 = 0;
    for (int x = 0; x < ND2; ++x) {
        const int x1 = (x == 0);
        for (int z = 0; z < N; ++z) {
            const float complex U1 = URAT(x, z, 0), U3 = URAT(x, z, 1);
            /* std::norm(complex<float>) evaluates re*re + im*im in float */
            const float n1 = crealf(U1) * crealf(U1) + cimagf(U1) * cimagf(U1);
            const float n3 = crealf(U3) * crealf(U3) + cimagf(U3) * cimagf(U3);
            const double u1u1 = n1, u3u3 = n3;
            const double ax2 = (double)alfa[x] * (double)alfa[x];
            const double gz2 = (double)gamma[z] * (double)gamma[z];
            const double K2 = ax2 + gz2;
            const double m = x1 ? 1.0 : 2.0;
            A1 += m * u1u1;
            A2 += m * u3u3;
            A3 += m * u1u1 * ax2;
            A4 += m * u1u1 * gz2;
            A5 += m * u3u3 * ax2;
            A6 += m * u3u3 * gz2;
            A7 += m * (u1u1 + u3u3) * K2 * K2;
            if (x1) E110 += u1u1;
        }
    }
    const double Q2 = A1 + A2, W2 = A3 + A4 + A5 + A6;
    const double visc = 1.0 / (double)Re;
    const double EP = visc * W2;
    const double De = 2.0 * visc * visc * A7;
    const double KOL = pow(visc * visc * visc / EP, 0.25);
    const double NLAM = (E110 != 0.0) ? 2.0 * A1 / E110 : 0.0;
    if (stats) {
        stats[0] = (double)Re;
        stats[1] = Q2;
        stats[2] = W2;
        stats[3] = EP;
        stats[4] = 2.0 * A1 / Q2 - 1.0;
        stats[5] = 2.0 * (A3 + A4) / W2 - 1.0;
        stats[6] = 0.5 * Q2 / EP;
        stats[7] = KOL;
        stats[8] = visc;
        stats[9] = DXZ / KOL;
        stats[10] = NLAM;
        stats[11] = 2.0 * PI / sqrt(2.0 * A1 / A3);
        stats[12] = 2.0 * PI / sqrt(2.0 * A1 / A4);
        stats[13] = 2.0 * PI / sqrt(2.0 * A2 / A5);
        stats[14] = 2.0 * PI / sqrt(2.0 * A2 / A6);
        stats[15] = De;
        stats[16] = 0.5 * Q2 * De / (EP * EP);
        stats[17] = (double)E1;
        stats[18] = (double)E3;
    }
    if (seed_out) *seed_out = seed;
    /* reshuffle loop (cuda/pao_km3_cuda.cu:429-442) is the identity for NE == N */
    if (out_uw) memcpy(out_uw, U, sizeof(float complex) * (size_t)ND2 * NE * 2);
#undef URAT
    free(U); free(alfa); free(gamma);
    return 0;
}

/* k^4 exp(-2 (k/K0)^2) random-phase vorticity spectrum, normalised to E = 1/2.
 * Written for the benchmark configurations; it has no counterpart in the reference code.
 * Phases: splitmix64(seed) drawn once per compact mode in [iz][ix] order, theta = 2 pi u,
 * u = (next >> 11) * 2^-53.  |w(k)|^2 = k (k/K0)^4 exp(-2 (k/K0)^2), then scaled so that
 * 1/2 sum_w |w|^2/K^2 = 1/2 (w = 1 at kx = 0, else 2).  Mode (0,0) and the kz = -N/2 row are
 * zero; the kx = 0 column is made Hermitian (w(0,-kz) = conj w(0,kz)). Output [iz][ix] c64. */
static uint64_t sm64_next(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int orc_k4_spectrum(int N, double K0, uint64_t seed, float *om2_out)
{
    const int H = N / 2;
    double *re = (double *)malloc(sizeof(double) * (size_t)N * H);
    double *im = (double *)malloc(sizeof(double) * (size_t)N * H);
    uint64_t s = seed;
    double Esum = 0.0;
    for (int iz = 0; iz < N; ++iz) {
        for (int ix = 0; ix < H; ++ix) {
            const double u = (double)(sm64_next(&s) >> 11) * (1.0 / 9007199254740992.0);
            const double th = 2.0 * 3.14159265358979323846 * u;
            const int kz = kz_of(iz, N);
            const double k2 = (double)ix * ix + (double)kz * kz;
            const size_t i = (size_t)iz * H + ix;
            if (k2 == 0.0 || kz == -H) { re[i] = 0.0; im[i] = 0.0; continue; }
            const double k = sqrt(k2), q = k / K0;
            const double a = sqrt(k * q * q * q * q * exp(-2.0 * q * q));
            re[i] = a * cos(th);
            im[i] = a * sin(th);
        }
    }
    for (int iz = N / 2 + 1; iz < N; ++iz) { /* kz < 0 on kx = 0: conjugate of kz > 0 */
        const size_t i = (size_t)iz * H, j = (size_t)(N - iz) * H;
        re[i] = re[j];
        im[i] = -im[j];
    }
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const int kz = kz_of(iz, N);
            const double k2 = (double)ix * ix + (double)kz * kz;
            if (k2 == 0.0) continue;
            const size_t i = (size_t)iz * H + ix;
            Esum += 0.5 * (ix == 0 ? 1.0 : 2.0) * (re[i] * re[i] + im[i] * im[i]) / k2;
        }
    const double sc = (Esum > 0.0) ? sqrt(0.5 / Esum) : 0.0;
    for (size_t i = 0; i < (size_t)N * H; ++i) {
        om2_out[2 * i] = (float)(re[i] * sc);
        om2_out[2 * i + 1] = (float)(im[i] * sc);
    }
    free(re); free(im);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Set-up paths                                                                                */
/* ------------------------------------------------------------------------------------------ */

/* mem_cuda start-up without restart (cuda/mem_cuda.cu:1767-1789): PAO -> CALCOM ->
 * STEP2A -> NEXTDT(init).  Returns the PAO seed. */
int orc_init_pao(orc_state *S, double *stats)
{
    const int N = S->N, H = S->H;
    float *uw = (float *)malloc(sizeof(float) * 4 * (size_t)N * H);
    int seed = 0;
    orc_pao_spectrum(N, S->K0, S->Re, uw, stats, &seed);
    S->visc = (float)(1.0 / (double)S->Re);
    memset(S->uc, 0, sizeof(zc) * 3 * (size_t)S->L * S->Nk);
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const size_t b = 4 * ((size_t)ix + (size_t)H * iz);
            UC(S, 0, iz, ix) = CMPLX((double)uw[b], (double)uw[b + 1]);
            UC(S, 1, iz, ix) = CMPLX((double)uw[b + 2], (double)uw[b + 3]);
        }
    /* CALCOM (cuda/calcom_cuda.cu:84-132): om = i (gamma u1 - alfa u2), rows taken directly */
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const double ax = ix, gz = kz_of(iz, N);
            S->om2[(size_t)iz * H + ix] = I * (gz * UC(S, 0, iz, ix) - ax * UC(S, 1, iz, ix));
        }
    memset(S->fnm1, 0, sizeof(zc) * (size_t)N * H);
    free(uw);
    step2a(S);
    next_dt(S);
    return seed;
}

/* Start from a given vorticity field om2 [iz][ix] c64 (FNM1 = 0): velocity recovery as in
 * STEP3 phase 2 (cuda/mem_cuda.cu:1138-1188), STEP2A, NEXTDT(init). */
void orc_init_om2(orc_state *S, const float *om2)
{
    const int N = S->N, H = S->H;
    memset(S->uc, 0, sizeof(zc) * 3 * (size_t)S->L * S->Nk);
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const size_t i = (size_t)iz * H + ix;
            const zc om = CMPLX((double)om2[2 * i], (double)om2[2 * i + 1]);
            S->om2[i] = om;
            S->fnm1[i] = 0;
            const double ax = ix, gz = kz_of(iz, N), K2 = ax * ax + gz * gz;
            zc o1 = 0, o2 = 0;
            if (ix >= 1) {
                const zc v = om / (K2 + 1.0e-30);
                o1 = -I * gz * v;
                o2 = I * ax * v;
            } else if (iz >= 1 && gz != 0.0) {
                o1 = -I * om / gz;
            }
            UC(S, 0, iz, ix) = o1;
            UC(S, 1, iz, ix) = o2;
        }
    S->it = 0; S->dt = 0.0f; S->cn = 1.0f; S->cnm1 = 0.0f; S->t = 0.0f;
    step2a(S);
    next_dt(S);
}

/* ------------------------------------------------------------------------------------------ */
/* Time loop (cuda/mem_cuda.cu:1848-1897)                                                      */
/* ------------------------------------------------------------------------------------------ */

/* OM2PHYS in FP64 (cuda/om2phys_cuda.cu:153-205): omega on the L x L grid -> out (may be NULL) */
static void om2phys(orc_state *S, double *out)
{
    const int N = S->N, H = S->H, L = S->L, Nk = S->Nk;
    zc *tmp = (zc *)calloc((size_t)L * Nk, sizeof(zc));
    for (int iz = 0; iz < N / 2; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            tmp[(size_t)iz * Nk + ix] = S->om2[(size_t)iz * H + ix];
            tmp[(size_t)(iz + N) * Nk + ix] = S->om2[(size_t)(iz + N / 2) * H + ix];
        }
    inv2d(S->pl, Nk, tmp, out);
    free(tmp);
}

/* display sigma of the 8-bit quantised field (cuda/mem_cuda.cu:742-818), in double */
static double display_sigma(const double *f, size_t n)
{
    double mn = f[0], mx = f[0];
    for (size_t i = 1; i < n; ++i) { if (f[i] < mn) mn = f[i]; if (f[i] > mx) mx = f[i]; }
    const double rng = mx - mn;
    double s = 0, s2 = 0;
    for (size_t i = 0; i < n; ++i) {
        int pix = 128;
        if (fabs(rng) > 1.0e-12) {
            double pf = 1.0 + ((f[i] - mn) / rng) * 254.0;
            if (pf < 1.0) pf = 1.0;
            if (pf > 255.0) pf = 255.0;
            pix = (int)pf;
        }
        s += pix;
        s2 += (double)pix * pix;
    }
    const double mean = s / (double)n;
    double var = s2 / (double)n - mean * mean;
    if (var < 0) var = 0;
    return sqrt(var);
}

/* Run steps it+1 .. it+nsteps of the reference loop with diagnostics every `update` steps and
 * at step `steps_total` (the loop's STEPS).  Per-step energy/enstrophy (after STEP3) go to
 * E_hist/Z_hist when non-NULL.  diag_out (when non-NULL) receives, for the last diagnostic
 * step, {it, t, dt, cn, cflm, sigma}. */
int orc_run(orc_state *S, int nsteps, int update, int steps_total, double *E_hist, double *Z_hist,
            double *diag_out)
{
    for (int n = 0; n < nsteps; ++n) {
        const int it = S->it + 1;
        S->it = it;
        const float dt_old = S->dt;
        step2b(S);
        step3(S);
        step2a(S);
        S->t += dt_old;
        if (E_hist) E_hist[n] = S->last_E;
        if (Z_hist) Z_hist[n] = S->last_Z;
        if (it == 1 || (update > 0 && it % update == 0) || it == steps_total) {
            next_dt(S);
            if (diag_out) {
                const size_t plane = (size_t)S->L * S->L;
                double *w = (double *)malloc(sizeof(double) * plane);
                om2phys(S, w);
                diag_out[0] = it;
                diag_out[1] = S->t;
                diag_out[2] = S->dt;
                diag_out[3] = S->cn;
                diag_out[4] = S->cflm;
                diag_out[5] = display_sigma(w, plane);
                free(w);
            }
        }
    }
    return 0;
}

/* Run steps with a prescribed dt for every step (no NEXTDT): the "fixed dt sequence" mode.
 * cnm1 bookkeeping follows the reference (cnm1 <- cn after every STEP3). */
int orc_run_fixed(orc_state *S, int nsteps, const float *dts, const float *cns, double *E_hist,
                  double *Z_hist)
{
    for (int n = 0; n < nsteps; ++n) {
        S->it += 1;
        S->dt = dts[n];
        S->cn = cns[n];
        step2b(S);
        step3(S);
        step2a(S);
        S->t += dts[n];
        if (E_hist) E_hist[n] = S->last_E;
        if (Z_hist) Z_hist[n] = S->last_Z;
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Accessors                                                                                   */
/* ------------------------------------------------------------------------------------------ */
/* 1: form the Crank-Nicolson factors in float as the reference does (for attributing the
 * reference's own distance from the FP64 scheme); 0 (default): FP64 */
void orc_set_f32_cn(orc_state *S, int on) { S->f32_cn = on; }

void orc_get_scalars(const orc_state *S, double *out)
{
    out[0] = S->it; out[1] = S->t; out[2] = S->dt; out[3] = S->cn; out[4] = S->cnm1;
    out[5] = S->cflm; out[6] = S->visc; out[7] = S->cflnum;
}

void orc_set_scalars(orc_state *S, const double *in)
{
    S->it = (int)in[0]; S->t = (float)in[1]; S->dt = (float)in[2]; S->cn = (float)in[3];
    S->cnm1 = (float)in[4]; S->cflm = (float)in[5]; S->visc = (float)in[6]; S->cflnum = (float)in[7];
}

/* om2 / fnm1 as [iz][ix] complex double interleaved */
void orc_get_om2(const orc_state *S, double *out)
{
    const size_t n = (size_t)S->N * S->H;
    for (size_t i = 0; i < n; ++i) { out[2 * i] = creal(S->om2[i]); out[2 * i + 1] = cimag(S->om2[i]); }
}

void orc_get_fnm1(const orc_state *S, double *out)
{
    const size_t n = (size_t)S->N * S->H;
    for (size_t i = 0; i < n; ++i) { out[2 * i] = creal(S->fnm1[i]); out[2 * i + 1] = cimag(S->fnm1[i]); }
}

/* physical u (c=0) / w (c=1) on the L x L grid, [z][x] */
void orc_get_ur(const orc_state *S, int c, double *out)
{
    memcpy(out, S->ur + (size_t)c * S->L * S->L, sizeof(double) * (size_t)S->L * S->L);
}

void orc_om2phys(orc_state *S, double *out) { om2phys(S, out); }

double orc_display_sigma(const double *f, size_t n) { return display_sigma(f, n); }

/* FP64 energy and enstrophy of a compact vorticity field [iz][ix] (double interleaved) */
void orc_energy_enstrophy(int N, const double *om2, double *E, double *Z)
{
    const int H = N / 2;
    double e = 0, z = 0;
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const size_t i = (size_t)iz * H + ix;
            const int kz = kz_of(iz, N);
            const double k2 = (double)ix * ix + (double)kz * kz;
            const double w = (ix == 0) ? 1.0 : 2.0;
            const double p = om2[2 * i] * om2[2 * i] + om2[2 * i + 1] * om2[2 * i + 1];
            z += 0.5 * w * p;
            if (k2 > 0) e += 0.5 * w * p / k2;
        }
    *E = e;
    *Z = z;
}

/* Shell spectrum E(k) = 1/2 sum_{round(|k|) = k} w |om|^2 / K^2, k = 0..nb-1 */
void orc_shell_spectrum(int N, const double *om2, double *Ek, int nb)
{
    const int H = N / 2;
    for (int k = 0; k < nb; ++k) Ek[k] = 0;
    for (int iz = 0; iz < N; ++iz)
        for (int ix = 0; ix < H; ++ix) {
            const size_t i = (size_t)iz * H + ix;
            const int kz = kz_of(iz, N);
            const double k2 = (double)ix * ix + (double)kz * kz;
            if (k2 == 0) continue;
            const int sh = (int)(sqrt(k2) + 0.5);
            if (sh >= nb) continue;
            const double w = (ix == 0) ? 1.0 : 2.0;
            Ek[sh] += 0.5 * w * (om2[2 * i] * om2[2 * i] + om2[2 * i + 1] * om2[2 * i + 1]) / k2;
        }
}

/* 2D forward transform of a real L x L plane, as cuFFT R2C: out [L][Nk] complex double */
void orc_fwd2d(int L, const double *in, double *out)
{
    orc_fft *p = fft_plan(L);
    const int Nk = L / 2 + 1;
    fwd2d(p, Nk, in, (zc *)out);
    fft_free(p);
}

/* 2D inverse (C2R) of an [L][Nk] complex plane -> real L x L */
void orc_inv2d(int L, const double *in, double *out)
{
    orc_fft *p = fft_plan(L);
    const int Nk = L / 2 + 1;
    inv2d(p, Nk, (const zc *)in, out);
    fft_free(p);
}

int orc_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
