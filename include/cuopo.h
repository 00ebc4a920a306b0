/*
 * cuopo.h -- C ABI of cuopo_b200, a B200 (sm_100a) split-step Fourier
 * coupled-wave solver for optical parametric oscillators.
 *
 * The library is a drop-in for the crystal pass and the cavity round-trip
 * loop of the reference simulator cuOPO.  Each entry point below names the
 * reference interface it replaces (paths relative to the reference's
 * repository root).  All functions return a cuopo_status and never exit
 * the process.  Device pointers are plain CUDA device addresses; "stream"
 * is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *
 * Field layout: one contiguous array of n_t interleaved complex values per
 * field (re, im), float pairs for CUOPO_F32 plans and double pairs for
 * CUOPO_F64 plans -- the layout of the reference's cufftComplex arrays.
 */
#ifndef CUOPO_H
#define CUOPO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum {
    CUOPO_OK = 0,
    CUOPO_EINVAL = 1,       /* bad argument (sizes, pointers, ranges) */
    CUOPO_ENOMEM = 2,       /* host or device allocation failed */
    CUOPO_ECUDA = 3,        /* a CUDA runtime call failed */
    CUOPO_ETIMEOUT = 4,     /* a bounded device-side wait gave up */
    CUOPO_ENONFINITE = 5,   /* a field became NaN/Inf */
    CUOPO_EUNSUPPORTED = 6, /* configuration not built into this library */
    CUOPO_EIO = 7           /* file I/O failed */
} cuopo_status;

enum { CUOPO_PPLN = 0, CUOPO_SPPLT = 1 };   /* -DPPLN / -DSPPLT */
enum { CUOPO_CW = 0, CUOPO_NS = 1 };        /* -DCW_OPO / -DNS_OPO */
/* Field precision.  CUOPO_F32: complex64 fields, every phase factor formed
 * in FP64 and rounded once; CUOPO_F64: complex128 fields and FP64
 * arithmetic; CUOPO_F32_PHASE32 (plans only): complex64 fields with the
 * phase factors (dispersion, RK4 stage phases, modulator, AddPhase) formed
 * by FP32 sin/cos after FP64 reduction of the argument to [-pi, pi] -- the
 * third variant of the precision study (the GDD/TOD factor formed inside
 * the kernel stays FP64). */
enum { CUOPO_F32 = 0, CUOPO_F64 = 1, CUOPO_F32_PHASE32 = 2 };

/*
 * Solver parameters: the arguments of EvolutionInCrystal
 * (src/headers/cwes2.cuh:132, src/headers/cwes3.cuh:139) plus the values the
 * round-trip loop src/cuOPO.cu:474-610 reads.  Units are the reference's:
 * um, ps, V.  All values are doubles; the reference's own float values are
 * represented exactly.
 */
typedef struct {
    int n_eqs;          /* 2 or 3 (-DTHREE_EQS) */
    int n_t;            /* grid points per round trip (SIZE), power of 2 */
    int n_z;            /* slices per crystal pass (NZ) */
    int regime;         /* CUOPO_CW or CUOPO_NS */
    double vp, vs, vi;              /* group velocities [um/ps] */
    double b2p, b2s, b2i;           /* GVD [ps^2/um] */
    double b3p, b3s, b3i;           /* TOD [ps^3/um] */
    double dk;                      /* phase mismatch [1/um] */
    double kp, ks, ki;              /* coupling kappa [1/V] */
    double dz;                      /* slice length [um] */
    double alpha_crp, alpha_crs, alpha_cri;  /* absorption [1/um] */
    double Rs, Ri;                  /* mirror reflectivities (fractions) */
    double delta;                   /* detuning in units of pi */
    double gdd;                     /* intracavity GDD [ps^2] */
    double tod_s, tod_i;            /* TOD compensation [ps^3] */
    int use_eom;                    /* intracavity phase modulator */
    int eom_idler;                  /* modulator also acts on the idler */
    double mod_depth;               /* modulation depth [rad] */
    double fpm;                     /* modulation frequency [THz] */
    double t_rt;                    /* round-trip time [ps] */
    double ap0;                     /* CW pump amplitude [V/um] */
} cuopo_params;

/*
 * Physical inputs: the reference's positional argv (src/cuOPO.sh:159,
 * parsed at src/cuOPO.cu:92-267) plus the values it hard-codes, made
 * run-time fields.  cuopo_inputs_default() fills the hard-coded values.
 */
typedef struct {
    int crystal;            /* CUOPO_PPLN / CUOPO_SPPLT */
    int n_eqs;              /* 2 or 3 */
    int regime;             /* CUOPO_CW / CUOPO_NS */
    int n_t;                /* SIZE (cuOPO.cu:28) */
    int n_z;                /* NZ (cuOPO.cu:29) */
    int n_rt;               /* NRT (cuOPO.cu:30) */
    double lp_nm;           /* argv[1] pump wavelength [nm] */
    double temp_c;          /* argv[2] (unused by the reference: T is scanned) */
    double lambda_um;       /* argv[3] grating period [um] */
    double n_thr;           /* argv[4] pump power / threshold */
    double r_percent;       /* argv[5] signal reflectivity [%] */
    double delta;           /* argv[6] detuning [units of pi] */
    double gdd_percent;     /* argv[7] GDD compensation [% of crystal GDD] */
    double tod_percent;     /* argv[8] TOD compensation [%] */
    int use_eom;            /* argv[9] */
    double mod_depth_pi;    /* argv[10] modulation depth [units of pi] */
    double freq_det_mhz;    /* argv[11] EOM frequency detuning [MHz] */
    double lcr_mm;          /* argv[12] crystal length [mm] */
    double ls_nm;           /* signal wavelength; 0 = 2*lp (cuOPO.cu:93) */
    int temp_from_scan;     /* 1 = scan 10..150 C like cuOPO.cu:100 */
    double lcav_um;         /* cavity length (cuOPO.cu:129: 100e3) */
    double ri;              /* idler reflectivity (cuOPO.cu:133: 0.98) */
    double waist_um;        /* pump waist (cuOPO.cu:202: 55) */
    double fwhm_ps;         /* NS pump FWHM (cuOPO.cu:244: 10000) */
} cuopo_inputs;

/* Derived quantities that the reference prints but the solver does not read. */
typedef struct {
    double temp_c, np, ns, ni, li, dkp, t_rt, fsr, finesse, ith, pth, power,
        gamma_l, alphas, alphai, sigmap, dT, dF;
} cuopo_info;

/* ------------------------------------------------------------ host set-up */

/* Fills the reference's hard-coded defaults (cuOPO.cu:28-30,93,129,133,202,244). */
void cuopo_inputs_default(cuopo_inputs *in);

/* Parameter derivation of src/cuOPO.cu:92-234 (Sellmeier: src/headers/ppln.cuh:33-189,
 * src/headers/spplt.cuh:31-153; temperature scan: src/headers/functions.cuh:23-54),
 * evaluated in float exactly as the reference does. */
cuopo_status cuopo_derive_params(const cuopo_inputs *in, cuopo_params *out, cuopo_info *info);

/* The same derivation for `count` instances at once on the device (the
 * batched set-up of a sweep): one warp per instance runs the temperature
 * scan, then the derivation, from the same source as cuopo_derive_params.
 * in_dev, out_dev and status_dev (CUOPO_OK or CUOPO_EINVAL per instance)
 * are device arrays; no cuopo_info.  Float operations round as on the host;
 * CUDA's powf/pow may differ from glibc's in the last bits, so the result
 * can differ from the host's (which is bit-exact with the reference's) by a
 * few float ulps.  Asynchronous on stream. */
cuopo_status cuopo_derive_params_device(const cuopo_inputs *in_dev, int count, cuopo_params *out_dev,
                                        int *status_dev, void *stream);

/* Sellmeier model of the crystal: which = 0 n, 1 dn/dl, 2 d2n/dl2, 3 d3n/dl3,
 * 4 group velocity, 5 GVD, 6 TOD.  L in um, T in C.  (ppln.cuh:33-189) */
float cuopo_sellmeier(int crystal, int which, float L, float T);

/* findPhaseMatchingTemp, src/headers/functions.cuh:23-54. */
float cuopo_phase_matching_temp(int crystal, float lp, float ls, float lambda_um,
                                float t_min, float t_max);

/* Grids of src/cuOPO.cu:169-189: T (n_t time points of one round trip) and
 * w (angular frequency, fftshifted, with the reference's (n-1) linspace
 * spacing).  Either output may be NULL. */
cuopo_status cuopo_make_grids(int n_t, double t_rt, float *T, float *w);

/* linspace (src/headers/functions.cuh:12-18) of length n into out. */
void cuopo_linspace(float *out, long n, float xmin, float xmax);

/* Pump inputs: CW constant (functions.cuh:91-100) and the NS Gaussian window
 * over n_t*n_rt points (cuOPO.cu:164-175,243-248, functions.cuh:77-85). */
cuopo_status cuopo_pump_cw(float *out_c32, int n_t, double ap0);
cuopo_status cuopo_pump_ns(float *out_c32, int n_t, int n_rt, double t_rt,
                           double ap0, double fwhm_ps);

/* Seeded complex Gaussian noise (re and im each N(0, sigma^2)), replacing
 * the clock-seeded NoiseGeneratorCPU (functions.cuh:58-71).  Philox4x32-10
 * counter-based generator + Box-Muller; the host and device versions give
 * identical bits.  out_c32 is float pairs (host or device pointer). */
cuopo_status cuopo_noise_host(float *out_c32, long n, double sigma, uint64_t seed,
                              uint64_t stream_id);
cuopo_status cuopo_noise_device(void *out_c32, long n, double sigma, uint64_t seed,
                                uint64_t stream_id, void *stream);

/* .dat writers of src/headers/files.cuh:21-62: one value per line,
 * 20 significant digits; complex vectors go to <name>_r.dat/<name>_i.dat. */
cuopo_status cuopo_write_dat_real(const char *path, const float *v, long n);
cuopo_status cuopo_write_dat_complex(const char *prefix, const float *v_c32, long n);
/* Reader for the same format (n values expected). */
cuopo_status cuopo_read_dat_complex(const char *prefix, float *v_c32, long n);

/* ------------------------------------------------------------- GPU solver */

typedef struct cuopo_plan cuopo_plan;

/*
 * Creates a plan: device-resident dispersion, GDD and RK4 tables for one
 * parameter set, and the kernel configuration (cluster size, threads).
 * w_host: the n_t angular frequencies the reference passes to
 * EvolutionInCrystal as w_ext_gpu (cuOPO.cu:183-189); NULL = build them
 * with cuopo_make_grids.  T_host likewise (used by the modulator).
 * Replaces the set-up of cuOPO.cu:379-454 (buffers, cufftPlan1d).
 * Grids (n_t, powers of 2): F32 512..2^16 with 2 equations, 512..2^17 with
 * 3; F64 512..2^16 with 2, 512..2^17 with 3.  Other sizes: CUOPO_EUNSUPPORTED.
 */
cuopo_status cuopo_plan_create(cuopo_plan **plan, const cuopo_params *p,
                               const float *w_host, const float *T_host,
                               int precision);
cuopo_status cuopo_plan_destroy(cuopo_plan *plan);

/* Cluster size and threads per CTA the plan launches with. */
cuopo_status cuopo_plan_config(const cuopo_plan *plan, int *cluster, int *threads,
                               int *smem_bytes);

/*
 * One crystal pass on device fields in place: EvolutionInCrystal,
 * src/headers/cwes2.cuh:132-215 (n_eqs 2; Ai ignored) and
 * src/headers/cwes3.cuh:139-225 (n_eqs 3).  One kernel launch.
 */
cuopo_status cuopo_crystal_pass(cuopo_plan *plan, void *Ap, void *As, void *Ai,
                                void *stream);

/*
 * Round trips nn = rt_begin .. rt_begin+rt_count-1 of the loop body
 * src/cuOPO.cu:474-610 on device fields in place, in one kernel launch:
 * pump injection (CW copy of pump[0..n_t), :480; NS ReadPump of the
 * n_t*n_rt window with its last-rt offset, :484), crystal pass, modulator
 * (:509-518), GDD/TOD compensation (:521-553), AddPhase (:557-566),
 * SaveRoundTrip (:570-608) of rts in [save_first, save_first+save_count)
 * to slot nn-save_first of save_p/save_s/save_i (each n_t*save_count
 * values; any may be NULL).  ps_hist (device, doubles, may be NULL) gets
 * (1/n_t) sum|As|^2 after each rt.  If tol > 0 the launch stops after the
 * first rt from the second on whose relative change of that power is
 * below tol; *rt_done_dev (device int, may be NULL) gets the number of rts
 * run.
 */
cuopo_status cuopo_round_trips(cuopo_plan *plan, void *Ap, void *As, void *Ai,
                               const void *pump, int n_rt, int rt_begin, int rt_count,
                               void *save_p, void *save_s, void *save_i,
                               int save_first, int save_count,
                               double *ps_hist, double tol, int *rt_done_dev,
                               void *stream);

/* Reads (and with reset != 0 clears) the plan's device-side status word:
 * CUOPO_OK, or CUOPO_ENONFINITE if a launch met a NaN/Inf signal power
 * (that instance stops at the round trip where it happened).  Synchronous. */
cuopo_status cuopo_plan_status(cuopo_plan *plan, int *status, int reset);

/*
 * The library's FFT alone: `batch` unnormalised C2C transforms of n points
 * (in place when in == out), exponent sign +1 = CUFFT_INVERSE, -1 =
 * CUFFT_FORWARD.  Replaces cufftPlan1d/cufftExecC2C of the reference
 * (src/headers/cwes2.cuh:139-140,170-182; src/cuOPO.cu:453-454,522-550).
 * n: power of 2 in [512, 8192] (F32) or [512, 4096] (F64).
 */
cuopo_status cuopo_fft_c2c(const void *in, void *out, int n, int batch, int sign,
                           int precision, void *stream);

/* ------------------------------------------------------- batched sweeps */

/*
 * One point of a CW 2-equation parameter sweep.  The reference runs every
 * sweep point as its own process (the nested loops of src/cuOPO.sh:91-174
 * around ./cuOPO); a batch runs them all in one persistent launch per
 * distinct grid size, every instance in its own CTA with its fields in
 * shared memory, until it converges or reaches the round-trip limit.
 */
typedef struct {
    int n_t;            /* grid points of this instance (power of 2) */
    double ap0;         /* CW pump amplitude [V/um] (cuOPO.cu:229) */
    double Rs;          /* signal mirror reflectivity, fraction (cuOPO.cu:130) */
    double delta;       /* detuning in units of pi (cuOPO.cu:140) */
    double gdd;         /* intracavity GDD [ps^2] (cuOPO.cu:142) */
    uint64_t seed;      /* seed of the initial signal noise */
} cuopo_instance;

typedef struct cuopo_batch cuopo_batch;

/* base supplies the crystal and everything not in cuopo_instance (CW,
 * 2 or 3 equations). */
cuopo_status cuopo_batch_create(cuopo_batch **batch, const cuopo_params *base,
                                const cuopo_instance *inst, int count, int precision);
/* A sweep of points of the reference's shell script (src/cuOPO.sh:91-174):
 * every instance has its own argv-level inputs -- pump wavelength, grating
 * period, crystal length, pump ratio, reflectivity, detuning, GDD and TOD
 * compensation, modulator, grid size, slices, 2 or 3 equations, CW or
 * nanosecond regime -- derived as cuopo_derive_params does.  A nanosecond
 * instance gets its own Gaussian pump window of n_t * n_rt points
 * (cuOPO.cu:164-175,243-248) and runs at most its n_rt round trips.
 * Instances with equal physics share one set of tables; all instances of a
 * grid size run in one persistent launch.  seeds: per-instance noise
 * seeds, or NULL for 0..count-1. */
cuopo_status cuopo_batch_create_inputs(cuopo_batch **batch, const cuopo_inputs *in, const uint64_t *seeds,
                                       int count, int precision);
/* Signal power (1/n_t) sum |As|^2 after each round trip of nanosecond
 * instance i (its n_rt values; the first n are copied).  Synchronous. */
cuopo_status cuopo_batch_history(cuopo_batch *batch, int i, double *ps, int n, void *stream);
cuopo_status cuopo_batch_destroy(cuopo_batch *batch);
/* Number of signal values of all instances (sum of n_t). */
cuopo_status cuopo_batch_total_elements(const cuopo_batch *batch, long *n);
/* Signal of every instance := seeded noise (cuopo_noise_device with the
 * instance's seed, stream id 0); idler of 3-equation instances likewise
 * with stream id 1. */
cuopo_status cuopo_batch_seed_noise(cuopo_batch *batch, double sigma, void *stream);
/* Copies all signals in/out: instances concatenated in creation order. */
cuopo_status cuopo_batch_set_signal(cuopo_batch *batch, const void *src, int src_on_device, void *stream);
cuopo_status cuopo_batch_get_signal(cuopo_batch *batch, void *dst, int dst_on_device, void *stream);
/* Runs every instance from round trip 0 until the relative change of its
 * signal power per round trip stays below tol for `patience` consecutive
 * round trips, or max_rt round trips have run.  Asynchronous on stream.
 * Equivalent to cuopo_batch_reset + cuopo_batch_step(chunk = max_rt). */
cuopo_status cuopo_batch_run(cuopo_batch *batch, int max_rt, double tol, int patience, void *stream);
/* Resumable form: reset every instance to round trip 0 (fields are kept),
 * then continue every still-running instance by up to `chunk` round trips
 * per call.  Instance state (round trips run, last power, flag) stays on the
 * device between calls. */
cuopo_status cuopo_batch_reset(cuopo_batch *batch, void *stream);
cuopo_status cuopo_batch_step(cuopo_batch *batch, int chunk, int max_rt, double tol, int patience,
                              void *stream);
/* A step returns once its launches are queued; each grid size runs on the
 * batch's own stream and goes on to its next step without waiting for the
 * others (all calls below that read or write the batch's state wait for
 * every grid size first).  cuopo_batch_wait makes `stream` wait for the
 * work queued so far, e.g. before recording a timing event. */
cuopo_status cuopo_batch_wait(cuopo_batch *batch, void *stream);
/* Number of instances still running (synchronous). */
cuopo_status cuopo_batch_pending(cuopo_batch *batch, int *running, void *stream);
/* Per-instance last signal power, round trips run and flag (0 running,
 * 1 converged, 2 round-trip limit reached, 5 non-finite) into host arrays
 * (any may be NULL).  Waits for stream. */
cuopo_status cuopo_batch_results(cuopo_batch *batch, double *ps, int *rts, int *flags, void *stream);

/*
 * Kernel autotuner (no counterpart in the reference, which has one cuFFT plan
 * and fixed launch shapes).  Grids that more than one built kernel
 * configuration can run (e.g. 2^15 points as 8 CTAs of 4096 or 4 CTAs of
 * 8192) are timed on `count` copies of the CW 2-equation instance `base`
 * (its n_t, ap0, Rs, delta, gdd) for n_rt round trips each (best of two
 * runs); the built-in choice stays unless another configuration is more
 * than 3 % faster, and the result becomes the one every plan and batch
 * created afterwards in this process uses for (precision, n_eqs, n_t).
 * The timing runs one grid size alone: in a sweep that runs several grid
 * sizes at once, configurations with one CTA per SM pack worse next to the
 * others than this timing shows.  Reports the chosen points per CTA,
 * cluster size and its time (ms; -1 when there was one candidate).
 * Synchronous; allocates device memory while it runs.
 */
cuopo_status cuopo_autotune(const cuopo_params *base, int precision, int count, int n_rt, int *points_per_cta,
                            int *cluster, double *ms);
/* Records a built configuration as the choice for (precision, n_eqs, n_t)
 * without timing (CUOPO_EUNSUPPORTED if it was not built). */
cuopo_status cuopo_kernel_select(int precision, int n_eqs, int n_t, int points_per_cta, int cluster);
/* Forgets every autotuned or selected choice (the built-in preference order applies). */
cuopo_status cuopo_autotune_reset(void);
/* The configuration a plan created now would use. */
cuopo_status cuopo_kernel_config(int precision, int n_eqs, int n_t, int *points_per_cta, int *cluster);

/*
 * One crystal pass that allocates no device memory, for callers that cannot
 * call cudaMalloc: a plugin in a process whose device memory belongs to
 * another allocator (a framework's caching allocator or a fixed memory
 * budget, where a cudaMalloc behind its back can fail or fragment its
 * pool).  It has no counterpart in the reference (whose caller allocates
 * every buffer, src/cuOPO.cu:384-442).  Same computation as
 * cuopo_crystal_pass on an FP32 plan built from (p, w_host); fields are
 * float pairs (device).  Its tables are built on the host and copied with
 * cudaMemcpyAsync from a static host buffer into a fixed 384 KiB device
 * array inside this library (held by every GPU that loads it until exit),
 * so n_t must be a power of 2 in [512, 8192] and n_z in [1, 1024]; larger
 * sizes return CUOPO_EINVAL.  What is tested: calls ordered on one stream,
 * each matching cuopo_crystal_pass.  The first call on a device looks up
 * that array's address and keeps it for the life of the process (so the
 * library must not be used across a cudaDeviceReset of that device).  The
 * array is shared by all calls and keeps the last call's tables, so calls
 * that overlap on the GPU race -- order them on one stream.  The pass does
 * not report non-finite fields (there is no status to read back; check the
 * fields).  w_host: the n_t angular frequencies, or NULL to build them from
 * p->t_rt.
 */
cuopo_status cuopo_crystal_pass_noalloc(const cuopo_params *p, const float *w_host, void *Ap, void *As,
                                        void *Ai, void *stream);

/* ---------------------------------------------- learned warm start (MLP) */

/*
 * A multilayer perceptron n_in -> width (GELU) x depth -> n_out that maps a
 * cavity's parameters to the low-order Fourier modes of its steady-state
 * signal; the solver starts from its prediction instead of noise.  No
 * counterpart in the reference, which always starts from noise
 * (src/headers/functions.cuh:58-71).  Weights and activations are BF16 on
 * the tensor cores (tcgen05) with FP32 accumulation; FP32 master weights,
 * Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the mean squared error over
 * all outputs.  Limits: 1 <= n_in <= 64, width and n_out multiples of 128
 * (n_out <= 1024), 1 <= depth <= 10.  Device buffers are sized for
 * max_batch rows (rounded up to 128).  Weights start uniform in
 * +-sqrt(6 / fan_in) from `seed`, biases at zero.  A network object is
 * not thread-safe: use it from one host thread (one stream at a time).
 */
typedef struct cuopo_mlp cuopo_mlp;

cuopo_status cuopo_mlp_create(cuopo_mlp **mlp, int n_in, int width, int depth, int n_out, int max_batch,
                              uint64_t seed);
cuopo_status cuopo_mlp_destroy(cuopo_mlp *mlp);
/* Number of parameters in the flat layout below. */
cuopo_status cuopo_mlp_param_count(const cuopo_mlp *mlp, long *n);
/* Flat FP32 host arrays, per layer l = 0..depth: W_l [n_out_l][n_in_l]
 * (row-major) then b_l [n_out_l].  set_params also clears the Adam state.
 * Synchronous. */
cuopo_status cuopo_mlp_set_params(cuopo_mlp *mlp, const float *host);
cuopo_status cuopo_mlp_get_params(cuopo_mlp *mlp, float *host);
/* Inference: x [batch][n_in] -> y [batch][n_out], FP32 device arrays. */
cuopo_status cuopo_mlp_forward(cuopo_mlp *mlp, const float *x, float *y, int batch, void *stream);
/* Loss (mean squared error over batch x n_out) and its gradient with
 * respect to every parameter (host array, flat layout) without an update.
 * x, t: device.  Synchronous. */
cuopo_status cuopo_mlp_gradients(cuopo_mlp *mlp, const float *x, const float *t, int batch, float *grad_host,
                                 float *loss_host, void *stream);
/* One Adam step on the batch (x, t device); the first call for a batch
 * size and stream captures forward, loss, backward and update in a CUDA
 * graph that later calls replay.  loss: device float of the batch's loss
 * before the update, or NULL.  Asynchronous. */
cuopo_status cuopo_mlp_train_step(cuopo_mlp *mlp, const float *x, const float *t, int batch, float lr, float *loss,
                                  void *stream);
/* Data-parallel training over ranks (one network copy per GPU):
 * grad_step runs forward, loss and backward on the rank's batch (one CUDA
 * graph per batch size and stream) and leaves the gradient in the network's
 * own device buffer, which grad_buffer exposes (FP32, `count` values, an
 * internal layout that an element-wise sum over ranks -- an NCCL
 * all-reduce -- keeps valid); apply_adam then takes one Adam step from that
 * buffer multiplied by grad_scale (1 / ranks after a sum).  With the same
 * parameters on every rank and equal batches, the ranks stay identical. */
cuopo_status cuopo_mlp_grad_step(cuopo_mlp *mlp, const float *x, const float *t, int batch, float *loss,
                                 void *stream);
cuopo_status cuopo_mlp_grad_buffer(cuopo_mlp *mlp, float **grad_dev, long *count);
cuopo_status cuopo_mlp_apply_adam(cuopo_mlp *mlp, float lr, float grad_scale, void *stream);
/* Waits for the device and reports CUOPO_ETIMEOUT if a GEMM's bounded wait
 * gave up since the last check. */
cuopo_status cuopo_mlp_status(cuopo_mlp *mlp);
/* The tensor-core GEMM alone: C[M][N] (FP32) = A[M][K] B[N][K]^T with A and
 * B row-major BF16 on the device; M a multiple of 128, N of 64, K of 64;
 * K split over `split` CTAs per tile (dividing K/64; C accumulated with
 * atomics when split > 1).  err_dev: device int that gets bit 0 if a
 * bounded wait (about 1 s) gave up, or NULL.  flags bit 0 is a test hook:
 * the tile's completion barrier is never signalled, so every CTA's wait
 * runs out, sets bit 0 and the CTA returns without storing (C is left
 * as it was). */
cuopo_status cuopo_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int split, int flags,
                             int *err_dev, void *stream);

/* Warm-start fields: `modes` holds per instance n_modes complex values
 * (re, im pairs) of the Fourier modes q = -n_modes/2 .. n_modes/2-1 (cycles
 * per round trip).  fields_from_modes writes each instance's n_t-point
 * time-domain field scale * sum_q c_q exp(+2 pi i q n / n_t) (the same
 * continuous field on any grid; n_modes a multiple of 16, <= 1024);
 * modes_from_spectrum reads the modes back from the cuopo_fft_c2c sign -1
 * transform of a field (divided by n_t * scale) with the sign that makes
 * the largest mode's real part >= 0 (the 2-wave equations are invariant
 * under As -> -As).  Device arrays; fields are float pairs;
 * fields_from_modes takes at most 65535 instances per call. */
cuopo_status cuopo_fields_from_modes(const float *modes, int count, int n_modes, int n_t, double scale, void *fields,
                                     void *stream);
cuopo_status cuopo_modes_from_spectrum(const void *spec, int count, int n_t, int n_modes, double scale, float *modes,
                                       void *stream);
/* Warm-start fields from the band representation: each row of `pred` (512
 * floats, an MLP output) holds the magnitudes of the 128 modes around +q0
 * ([0,128): q0-64 .. q0+63) and around -q0 ([128,256): -q0-64 .. -q0+63),
 * then 64 copies each of cos(Phi), sin(Phi), 2 (q0 / (n_t/2))^2 - 1 and
 * log10(P).  The field is scale * sum_q c_q exp(+2 pi i q n / n_t) with
 * |c_q| proportional to max(magnitude, 0), total power P (the means of the
 * copies; q0 rounded and clamped to [64, n_t/2 - 64]) and every mode of
 * phase Phi/2, so that each signal-idler pair c_q c_-q has the phase Phi.
 * centres (device, may be NULL) gets each instance's q0.  At most 65535
 * instances per call. */
cuopo_status cuopo_fields_from_bands(const float *pred, int count, int n_t, double scale, void *fields, int *centres,
                                     void *stream);

/* Measured FP32 FMA throughput of the current device in TFLOP/s (best of 3
 * launches each of a scalar and a packed FP32x2 FMA-chain kernel over every
 * SM); the denominator of the solver's roofline.  Synchronous. */
cuopo_status cuopo_probe_fp32_peak(double *tflops, void *stream);

/* The same for FP64 (best of 3 launches of an fma.rn.f64-chain kernel over
 * every SM): the denominator of the FP64 plans' roofline.  Synchronous. */
cuopo_status cuopo_probe_fp64_peak(double *tflops, void *stream);

/* Blocks until the plan's work on stream has finished; returns the first
 * asynchronous error. */
cuopo_status cuopo_sync(void *stream);

/* Text of the last error recorded by this thread (never NULL). */
const char *cuopo_last_error(void);

/* Library version string. */
const char *cuopo_version(void);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* CUOPO_H */
