/*
 * dns2d.h — C ABI of the B200 (sm_100a) 2D pseudo-spectral vorticity solver.
 *
 * Drop-in replacement for the in-process solver API of cudaturbo's mem_cuda
 * (cuda/cuda_dns.h:108-202).  Plain C types only: every array argument is a host pointer
 * with an explicit layout, every function returns DNS2D_OK or a DNS2D_ERR_* code (nothing
 * aborts), and dns2d_last_error() gives the message of the latest failure on a state.
 *
 * Grid conventions (the reference's, cuda/cuda_dns.h:27-34, cuda/step3_cuda.cu:57-65):
 *   N      base resolution (multiple of 8), retained modes |kx| < N/2, -N/2 <= kz < N/2
 *   L      = 3N/2, the dealiased physical grid (NX_full = NZ_full)
 *   om2    vorticity spectrum, [iz][ix] complex64 (N rows of N/2), kz = iz < N/2 ? iz : iz-N
 *   fnm1   previous nonlinear term, same layout
 *   phys   physical planes [L][L] float32, x fastest: comp 0 = u, 1 = w, 2 = scalar (omega,
 *          stream function or |u| after the matching call)
 * A state owns one CUDA stream; calls on one state must come from one host thread.
 */
#ifndef DNS2D_H
#define DNS2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DNS2D_OK = 0,
    DNS2D_ERR_ARG = 1,      /* bad argument (NULL pointer, wrong size, bad component) */
    DNS2D_ERR_SIZE = 2,     /* N not supported by the compiled kernels */
    DNS2D_ERR_CUDA = 3,     /* CUDA runtime error (message in dns2d_last_error) */
    DNS2D_ERR_NOMEM = 4,    /* device allocation failed */
    DNS2D_ERR_IO = 5,       /* file could not be opened / read / written */
    DNS2D_ERR_FORMAT = 6,   /* restart file header or sizes do not match */
    DNS2D_ERR_STATE = 7,    /* call out of order (e.g. step before an initial condition) */
    DNS2D_ERR_TIMEOUT = 8   /* host watchdog expired waiting for the device */
};

typedef struct dns2d_state dns2d_state;

/* Scalars of the run; the float fields follow the reference's float host arithmetic. */
typedef struct {
    int32_t N, NX_full, NK_full, it, ifn;
    float Re, K0, visc, t, dt, cn, cnm1, cflnum, cflm;
} dns2d_scalars;

/* ---- life cycle: replaces dnsCudaCreate / dnsCudaDestroy (cuda/cuda_dns.h:108-109) ---- */
int dns2d_create(dns2d_state **out, int N, float Re, float K0, float cflnum, int device);
void dns2d_destroy(dns2d_state *s);
const char *dns2d_strerror(int code);
const char *dns2d_last_error(const dns2d_state *s);
/* 1 when N has compiled kernels in this library, else 0 */
int dns2d_supported(int N);
/* device bytes held by a state of size N */
size_t dns2d_device_bytes(int N);

/* ---- initial conditions: replace dnsCudaInit = PAO + CALCOM (cuda/cuda_dns.h:118-127) ----
 * All set it = 0, t = 0, dt = 0, cn = 1, cnm1 = 0, and leave the velocity ready, so the next
 * call is dns2d_next_dt() (the reference's initial STEP2A + NEXTDT init branch). */
/* PAO-k^-3 field of cuda/pao_km3_cuda.cu:59-498; stats19 (nullable) receives the 19 printed
 * statistics (Reynolds n., Energy, WiWi, Epsilon, a11, e11, Time scale, Kolmogorov,
 * Viscosity, dx/Kol., 2Pi/Nlamda, 2Pi/Lux, 2Pi/Luz, 2Pi/Lwx, 2Pi/Lwz, Deps., Ceps2, E1, E3),
 * pao_seed (nullable) the final generator state ("PAO seed"). */
int dns2d_init_pao(dns2d_state *s, double *stats19, int *pao_seed);
/* given vorticity (and optional previous nonlinear term, NULL = 0), [iz][ix] complex64 */
int dns2d_init_vorticity(dns2d_state *s, const float *om2, const float *fnm1);
/* seeded random-phase spectrum E(k) ~ (k/K0)^4 exp(-2 (k/K0)^2), total energy 1/2 (no
 * counterpart in the reference; written for the benchmark configurations) */
int dns2d_init_k4(dns2d_state *s, uint64_t seed);
/* the same field on the host without a state: om2 [N][N/2] complex64 */
int dns2d_k4_spectrum(int N, float K0, uint64_t seed, float *om2);

/* ---- time stepping: replaces dnsCudaStep2B + dnsCudaStep3 + dnsCudaStep2A and the host
 * bookkeeping of the mem_cuda loop (cuda/mem_cuda.cu:1848-1857).  Advances nsteps steps with
 * the current dt; per step it += 1, t += dt (float), cnm1 <- cn.  E_hist / Z_hist (nullable,
 * nsteps entries) receive the FP64 energy 1/2 sum w|om|^2/K^2 and enstrophy 1/2 sum w|om|^2
 * (w = 1 on kx = 0, else 2) after each step.  Asynchronous unless a history is requested. */
int dns2d_step(dns2d_state *s, int nsteps, double *E_hist, double *Z_hist);
/* NEXTDT of cuda/dns_cuda.cu:553-580 on the current velocity; writes CFLM (nullable) */
int dns2d_next_dt(dns2d_state *s, float *cflm);
/* Build the CUDA graphs dns2d_step(s, nsteps) will launch, without running them (no counterpart
 * in the reference): keeps the one-time graph capture out of a timed dns2d_step.  Nothing to do
 * with a closure attached. */
int dns2d_prepare(dns2d_state *s, int nsteps);
/* the state's CUDA stream (a cudaStream_t), for callers that order their own work after it */
void *dns2d_stream(dns2d_state *s);
/* wait for the state's stream; watchdog: DNS2D_ERR_TIMEOUT after timeout_ms (<= 0: none) */
int dns2d_sync(dns2d_state *s, int timeout_ms);

/* ---- diagnostics ---- */
/* omega to physical space into phys[2] (dnsCudaOm2Phys, cuda/om2phys_cuda.cu:153-205) */
int dns2d_om2phys(dns2d_state *s);
/* stream function psi = om/K^2 into phys[2] (dnsCudaStreamFunc, cuda/om2phys_cuda.cu:258) */
int dns2d_stream_func(dns2d_state *s);
/* u, w into phys[0], phys[1] (the reference's UR_full after STEP2A) */
int dns2d_velocity_phys(dns2d_state *s);
/* |u| into phys[2] from phys[0..1] (dnsCudaKinetic, cuda/om2phys_cuda.cu:358) */
int dns2d_kinetic(dns2d_state *s);
/* std-dev of the 8-bit quantised phys[comp] image (computeDisplaySigma, cuda/mem_cuda.cu:820) */
int dns2d_display_sigma(dns2d_state *s, int comp, double *sigma);
/* FP64 energy and enstrophy of the current vorticity */
int dns2d_energy_enstrophy(dns2d_state *s, double *E, double *Z);
/* FP64 shell spectrum E(k) = 1/2 sum_{round|k| = k} w |om|^2 / K^2, k = 0..nbins-1 */
int dns2d_shell_spectrum(dns2d_state *s, double *Ek, int nbins);
/* palinstrophy ratio of cuda/mem_cuda.cu:872-940 (FP64 on the device) */
int dns2d_palin(dns2d_state *s, double *pal_over_ens_kmax2);
/* energy_spectrum.csv bins of cuda/mem_cuda.cu:575-649 (nbins = 3N): the forward R2C of the
 * physical velocity over every mode, binned on the host in the reference's loop order, so the
 * bins beyond the retained radius hold the transform's rounding noise as in the reference; at the
 * cluster sizes (N >= 8192, rows beyond one CTA) only the retained modes, exactly */
int dns2d_velocity_spectrum_bins(dns2d_state *s, double *esum, int *count, int nbins);

/* ---- state transfer ---- */
int dns2d_get_scalars(const dns2d_state *s, dns2d_scalars *out);
int dns2d_set_scalars(dns2d_state *s, const dns2d_scalars *in);
int dns2d_get_om2(dns2d_state *s, float *om2);
int dns2d_get_fnm1(dns2d_state *s, float *fnm1);
int dns2d_get_phys(dns2d_state *s, int comp, float *plane);
/* load u, w physical planes (e.g. a restart file's UR_full) as the current velocity */
int dns2d_set_velocity_phys(dns2d_state *s, const float *u, const float *w);
/* restart.bin v2 writer / v1+v2 reader (cuda/mem_cuda.cu:1019-1394 byte layout).  The file moves
 * through three pinned staging buffers of up to 64 MiB each (allocated at the first save or load,
 * freed by dns2d_destroy), with device<->host copies overlapping the file writes / reads.  A load
 * checks the header and the file size before it touches the state. */
int dns2d_save_restart(dns2d_state *s, const char *path);
int dns2d_load_restart(dns2d_state *s, const char *path);

/* ---- movie frames (cuda/color_cuda.cu:491-597, dnsCudaMovieScaleF / dnsCudaSaveFieldInfernoPng
 * without the PNG file: the CLI writes it) ----
 * dns2d_movie_scale: the downsampling factor F the reference uses for size N.
 * dns2d_movie_frame: inferno RGB image (rows of width * 3 bytes) of physical plane comp (0..2; 2 is
 * the vorticity after dns2d_om2phys), every F-th point of the 3N/2 x 3N/2 grid (F <= 0 means 1).
 * With rgb NULL only width/height are returned; sigma_out (nullable) receives the plane's pixel
 * sigma that sets the contrast stretch. */
int dns2d_movie_scale(int N);
int dns2d_movie_frame(dns2d_state *s, int comp, int scale_f, unsigned char *rgb, int *width, int *height,
                      double *sigma_out);

/* ---- time step without device allocation (no counterpart in the reference) ----
 * For callers that cannot allocate device memory: an application that hands out only its own
 * pooled or arena buffers, a process under a fixed device-memory budget, or code where
 * cudaMalloc is not allowed.  The caller passes the state in its own device buffers:
 *   om2, fnm1  device arrays [iz][ix] complex64 (N rows of N/2), advanced nsteps steps in place
 *   visc, dt   viscosity and time step; cnm1 is used by the first step, cn by the later ones
 *              (the reference's CNM1 <- CN rule); stream is a cudaStream_t (NULL = default)
 * Nothing is allocated: all scratch (about 20 N^2 bytes) lives in one static device array of
 * DNS2D_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the process exits,
 * which limits N to DNS2D_NOALLOC_MAX_N; larger N returns DNS2D_ERR_SIZE.  A call looks up that
 * array's device address with the device current; while the stream is capturing it reuses the
 * address found by the last call outside capture, so make the first call on a device before any
 * stream capture.  Every call shares the array: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.  An error already pending on the
 * calling thread is cleared on entry and not reported.  The call is asynchronous on the stream;
 * the host scalars (t, it, cnm1) are the caller's to advance. */
#define DNS2D_NOALLOC_MAX_N 512
#define DNS2D_NOALLOC_SCRATCH_BYTES (6u << 20)
int dns2d_step_noalloc(int N, float visc, float dt, float cnm1, float cn, int nsteps,
                       void *om2, void *fnm1, void *stream);

/* ---- batched ensembles (no counterpart in the reference: written for its ensemble
 * configuration).  Independent runs, each with its own N (any supported size), Re, K0, CFL
 * and initial-field seed, advanced together: members of one N share each kernel launch, and a
 * chunk of up to 128 ensemble steps is one captured CUDA graph.  Every member keeps the
 * reference's float scalar bookkeeping; results equal those of one dns2d_state per member. */
typedef struct {
    int32_t N;
    float Re, K0, cflnum;
    uint64_t seed; /* seed of the k^4 exp(-2 (k/K0)^2) initial field (dns2d_batch_init_k4) */
} dns2d_member;
typedef struct dns2d_batch dns2d_batch;
int dns2d_batch_create(dns2d_batch **out, const dns2d_member *members, int count, int device);
void dns2d_batch_destroy(dns2d_batch *b);
const char *dns2d_batch_last_error(const dns2d_batch *b);
void *dns2d_batch_stream(dns2d_batch *b);
/* every member from its own seeded k^4 field (then call dns2d_batch_next_dt) */
/* Autotuner for a batch (no counterpart in the reference): times each size group's kernel
 * variants at the group's member count on the batch's buffers and keeps the fastest; call before
 * dns2d_batch_init_k4 (DNS2D_ERR_STATE after it).  Variants compute the same arithmetic. */
int dns2d_batch_autotune(dns2d_batch *b);
int dns2d_batch_init_k4(dns2d_batch *b);
/* NEXTDT for every member; cflm (nullable) receives count values */
int dns2d_batch_next_dt(dns2d_batch *b, float *cflm);
/* nsteps steps of every member; E_hist / Z_hist (nullable) are [count][nsteps] */
int dns2d_batch_step(dns2d_batch *b, int nsteps, double *E_hist, double *Z_hist);
/* build the graphs a later dns2d_batch_step(b, nsteps) launches, without running them */
int dns2d_batch_prepare(dns2d_batch *b, int nsteps);
/* Stepping mode of a batch (no counterpart in the reference): 0 = one CUDA graph per chunk of up
 * to 128 steps, each size group's row and column kernels a parallel branch (default); 1 = one
 * persistent launch per chunk: every member of every size advances inside one cooperative kernel
 * whose CTAs take row and column work items in dependency order and wait on per-member
 * completion counters (sizes 64, 128, 256, 512, each on its default radix plan; the fields equal
 * mode 0's on those plans bit for bit).  DNS2D_ERR_SIZE when the batch holds another size. */
int dns2d_batch_set_mode(dns2d_batch *b, int mode);
/* The persistent launch's dependency waits: polls of a counter before a wait gives up, which
 * makes dns2d_batch_step return DNS2D_ERR_TIMEOUT with the context still usable (default 4 M,
 * about a second), and a member whose column items wait for a count that nothing reaches (-1:
 * none), with which a test makes a wait run out. */
int dns2d_batch_set_waits(dns2d_batch *b, long long spin_limit, int stall_member);
/* Work-item size of the persistent launch (powers of two up to 64, reduced per size group to a
 * divisor of its count): row tiles of 4 physical rows per row item (default 8) and column groups
 * per column item (default 4).  Scheduling only: the results do not change. */
int dns2d_batch_set_items(dns2d_batch *b, int tiles_per_item, int groups_per_item);
int dns2d_batch_sync(dns2d_batch *b);
int dns2d_batch_get_om2(dns2d_batch *b, int member, float *om2);
int dns2d_batch_get_scalars(dns2d_batch *b, int member, dns2d_scalars *out);

/* ---- learned subgrid closure network (no counterpart in the reference) ----
 * Periodic 3x3 CNN: `layers` convolutions, inputs (filtered vorticity, u, w), `channels` hidden
 * channels with GELU, one output channel (the subgrid forcing).  Arrays are [B][C][H][W] float32
 * host buffers; parameters are one flat vector (per layer: weights [Co][Ci][3][3], bias [Co]).
 * Training runs on the device with the library's own forward, backward and Adam kernels. */
typedef struct dns2d_cnn dns2d_cnn;
int dns2d_cnn_create(dns2d_cnn **out, int layers, int channels, uint64_t seed, int device);
void dns2d_cnn_destroy(dns2d_cnn *n);
const char *dns2d_cnn_last_error(const dns2d_cnn *n);
int dns2d_cnn_num_params(const dns2d_cnn *n);
int dns2d_cnn_get_params(dns2d_cnn *n, float *params);
int dns2d_cnn_set_params(dns2d_cnn *n, const float *params);
int dns2d_cnn_forward(dns2d_cnn *n, const float *x, int B, int H, int W, float *y);
/* mean squared error against t and its gradient with respect to every parameter */
int dns2d_cnn_loss_grad(dns2d_cnn *n, const float *x, const float *t, int B, int H, int W, double *loss,
                        float *grad);
/* keep a training set of count samples on the device; then Adam on random minibatches */
int dns2d_cnn_set_dataset(dns2d_cnn *n, const float *x, const float *t, int count, int H, int W);
int dns2d_cnn_train(dns2d_cnn *n, int iters, int batch, float lr, uint64_t seed, double *losses);
/* Training convolutions on the tensor cores (off by default; channels <= 32): forward, data and
 * weight gradients as tcgen05 GEMMs over bf16 im2col expansions with FP32 accumulation (the
 * weight gradient split over the pixels, partials summed in fixed order in FP64); loss, GELU and
 * Adam stay FP32.  Applies to dns2d_cnn_forward, dns2d_cnn_loss_grad and dns2d_cnn_train; the
 * gradients then agree with the FP32 ones to bf16 rounding of the operands. */
int dns2d_cnn_set_train_tc(dns2d_cnn *n, int on);
/* The same forward on the BF16 tensor-core path: every layer runs as an implicit GEMM on tcgen05
 * (bf16 inputs, weights and activations, FP32 accumulation, GELU in its tanh form).  Needs channels == 32, layers >= 3 and W % 128 == 0 (DNS2D_ERR_SIZE otherwise). */
int dns2d_cnn_forward_tc(dns2d_cnn *n, const float *x, int B, int H, int W, float *y);
/* How the tensor-core path launches layers 1 .. L-1: mode 1 (default) one persistent,
 * warp-specialised launch (one CTA per SM; tiles handed out in layer order, each waiting for its
 * three input tile rows of the previous layer) wherever the weights of those layers fit in shared
 * memory (layers <= 8), else one launch per layer; mode 0 always one launch per layer.  Both give
 * the same values bit for bit.  tc_info reports the mode and the grid of the last persistent
 * launch (0 before any).  The mode (and the trace below) applies to launches made after the
 * call; a state's already captured closed-step graphs keep theirs until the closure is attached
 * again. */
int dns2d_cnn_set_tc_mode(dns2d_cnn *n, int mode);
int dns2d_cnn_tc_info(const dns2d_cnn *n, int *mode, int *grid);
/* Per-tile timestamps of the persistent launch (globaltimer ns; off by default): with tracing on,
 * each persistent launch records for every tile (layer-major order, tile rows rotated by one per
 * layer) 8 times: the producer took the tile, found its input rows complete, found its halo stage
 * free, issued its halo copy; the MMA issuer found the copy landed, then (once the accumulator
 * buffer was free) had issued and committed the MMAs; the epilogue started, and its first warp
 * released the tile (or wrote the output).  read_trace copies up to cap tiles x 8 values of the last launch and sets *tiles
 * to its tile count. */
int dns2d_cnn_set_trace(dns2d_cnn *n, int on);
int dns2d_cnn_read_trace(dns2d_cnn *n, unsigned long long *out, int cap, int *tiles);

/* Couple a trained network to a state as its subgrid closure (NULL network detaches): every
 * dns2d_step evaluates it on (omega/s0, u/s1, w/s2) of the current field on the L x L grid and
 * adds s3 * its output, transformed to the retained modes, to the nonlinear term.  The plain
 * coarse step is the fallback whenever the closure would make the resolved energy rise beyond
 * the viscous bound (unforced 2D flow only loses energy):
 *   energy_check 0  no check;
 *   energy_check 1  on the device, before each step: the closure is dropped for the step when its
 *                   energy input sum w Re(conj(om/K^2) F) exceeds the viscous loss 2 nu Z
 *                   (steps stay in captured CUDA graphs);
 *   energy_check 2  after each step on the host: a step whose energy rose is rolled back and
 *                   redone without the closure (one host sync per step);
 *   energy_check 3  as 1, but the forcing of such a step is scaled by 2 nu Z / P (its energy input
 *                   then equals the viscous loss) instead of dropped.
 * dns2d_closure_stats counts closed steps and fallbacks (dropped or scaled steps).  The network
 * must not be used by another state or trained while attached. */
int dns2d_closure_attach(dns2d_state *s, dns2d_cnn *n, const float *scales4, int energy_check);
/* The spectral forcing the attached closure adds to FN for the current state, in the compact
 * layout of dns2d_get_fnm1 (N x N/2 complex float, [kz][kx]); a diagnostic, the state is not
 * advanced. */
int dns2d_closure_forcing(dns2d_state *s, float *force);
/* Closed steps and fallbacks so far; DNS2D_ERR_TIMEOUT if a tensor-core wait of the closure
 * network ran out (its bounded mbarrier wait sets a device flag instead of hanging). */
int dns2d_closure_stats(dns2d_state *s, long long *steps, long long *fallbacks);
/* 1 (default): the closure network runs on the BF16 tensor-core path where the grid allows it
 * (L % 128 == 0, 32 channels); 0: FP32 on the SIMT pipes everywhere. */
int dns2d_closure_tensor_cores(dns2d_state *s, int enable);
/* Forcing limiter (default off): each mode's closure forcing is limited in magnitude to alpha
 * times the resolved nonlinear term FN of the same mode, so the closure cannot act where the
 * resolved transfer vanishes (e.g. shells the cascade has not reached yet). */
int dns2d_closure_clamp(dns2d_state *s, float alpha);

/* Autotuner (no counterpart in the reference): times the kernel variants of size N on a scratch
 * state on `device` -- rows per CTA and the radix plans of the small-grid (N <= 512) row and
 * column passes, one or two thread groups per column CTA and the L2 prefetch distances of the
 * large-grid passes -- and keeps the fastest for states and batches created afterwards on that
 * device.  Rows per CTA, thread groups and prefetch distances do not change the arithmetic; a
 * radix plan changes the FP32 rounding (every plan meets the oracle tolerances), and an
 * alternative plan is kept only when it is at least 3 % faster than the default one.  config
 * (nullable, 6 ints) receives {rows_tile, cols_groups, pf_rows, pf_cols, plan_rows, plan_cols}
 * (0 = the size's default).  DNS2D_AUTOTUNE=1 in the environment makes dns2d_create tune its
 * size once per process. */
int dns2d_autotune(int N, int device, int *config);
/* Pin a configuration {rows_tile (0, 2, 4, 8), cols_groups (0, 1, 2), pf_rows, pf_cols,
 * plan_rows, plan_cols (0 .. plans of N - 1; 3 plans at N = 64 ... 512, else 1)} for size N on
 * `device` (no counterpart in the reference); used by states created afterwards. */
int dns2d_set_tuning(int N, int device, const int *config);

/* ---- phase timing: PHASE_TIMING of cuda/dns_cuda.cu:26-150 on the fused kernels ---- */
int dns2d_phase_timing(dns2d_state *s, int enable);
/* ms[0..3], counts[0..3]: row pass, column pass, NEXTDT/CFLM, OM2PHYS+sigma */
int dns2d_phase_report(dns2d_state *s, double *ms, long long *counts);

#ifdef __cplusplus
}
#endif
#endif /* DNS2D_H */
