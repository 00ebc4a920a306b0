/*
 * ssfm_oracle.c -- CPU oracle for the cuOPO split-step Fourier (SSFM) solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * load it.  The product path (cuopo_b200/) never links or calls it.
 *
 * It restates, step by step and in the order the reference executes them,
 * the reference's crystal pass and cavity round trip:
 *
 *   dAdz (2 eqs)            src/headers/cwes2.cuh:30-42
 *   LinealCombination       src/headers/cwes2.cuh:54-65   (no step h: quirk Q1)
 *   rk4                     src/headers/cwes2.cuh:76-87
 *   LinearOperator          src/headers/cwes2.cuh:103-121
 *   EvolutionInCrystal      src/headers/cwes2.cuh:132-215 (2nd half-step at the
 *                                                          same z: quirk Q2)
 *   dAdz (3 eqs)            src/headers/cwes3.cuh:30-43   (k2..k4 on the
 *                                                          unperturbed fields: Q3)
 *   LinearOperator (3 eqs)  src/headers/cwes3.cuh:107-128 (GVM terms: Q4)
 *   EvolutionInCrystal (3)  src/headers/cwes3.cuh:139-225
 *   CUFFTscale              src/headers/functions.cuh:126-135
 *   AddPhase                src/headers/functions.cuh:139-152
 *   AddGDD / AddGDDTOD      src/headers/functions.cuh:156-186
 *   ReadPump                src/headers/functions.cuh:191-213 (last-rt offset: Q6)
 *   SaveRoundTrip           src/headers/functions.cuh:217-238
 *   PhaseModulatorIntraCavity src/headers/functions.cuh:242-253
 *   round-trip loop body    src/cuOPO.cu:474-610
 *
 * cufftExecC2C is replaced by an unnormalised radix-2 FFT written here
 * (CUFFT_INVERSE = exponent sign +1, CUFFT_FORWARD = sign -1), with
 * twiddles from double-precision cos/sin.
 *
 * The scalar type is ORACLE_REAL (double by default; the float build is
 * only used as a CPU timing baseline).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif

typedef ORACLE_REAL real;
typedef ORACLE_REAL _Complex cplx;

#define ORACLE_PI 3.14159265358979323846

/* Parameter block.  Field order is part of the ctypes binding in
 * oracle/binding.py (which passes the library's cuopo_params struct, whose
 * leading fields are these); keep them in step. */
typedef struct {
    int n_eqs;          /* 2 or 3 coupled-wave equations (THREE_EQS) */
    int n_t;            /* grid points per round trip (SIZE, a power of 2) */
    int n_z;            /* slices per crystal pass (NZ) */
    int regime;         /* 0 = CW_OPO (pump copied every rt), 1 = NS_OPO */
    double vp, vs, vi;        /* group velocities [um/ps] */
    double b2p, b2s, b2i;     /* GVD [ps^2/um] */
    double b3p, b3s, b3i;     /* TOD [ps^3/um] */
    double dk;                /* phase mismatch [1/um] */
    double kp, ks, ki;        /* coupling constants kappa [1/V] */
    double dz;                /* slice length [um] */
    double alpha_crp, alpha_crs, alpha_cri; /* linear absorption [1/um] */
    double Rs, Ri;            /* mirror reflectivities (fractions) */
    double delta;             /* detuning, in units of pi (functions.cuh:145) */
    double gdd;               /* intracavity GDD [ps^2] (cuOPO.cu:142) */
    double tod_s, tod_i;      /* TOD compensation [ps^3] (cuOPO.cu:143,145) */
    int use_eom;              /* intracavity phase modulator on/off */
    int eom_idler;            /* modulator also on the idler (cuOPO.cu:441) */
    double mod_depth;         /* modulation depth m [rad] */
    double fpm;               /* modulation frequency [THz] */
} oracle_params;

/* ------------------------------------------------------------------ FFT */

typedef struct {
    int n;
    int log2n;
    cplx *tw;       /* tw[k] = exp(-2 pi i k / n), k < n/2 */
    int *rev;
} fft_plan;

static int ilog2(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return ((1 << l) == n) ? l : -1;
}

static int fft_plan_init(fft_plan *p, int n)
{
    p->n = n;
    p->log2n = ilog2(n);
    if (p->log2n < 1) return -1;
    p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)(n / 2));
    p->rev = (int *)malloc(sizeof(int) * (size_t)n);
    if (!p->tw || !p->rev) return -1;
    for (int k = 0; k < n / 2; k++) {
        double a = -2.0 * ORACLE_PI * (double)k / (double)n;
        p->tw[k] = (real)cos(a) + I * (real)sin(a);
    }
    for (int i = 0; i < n; i++) {
        int r = 0;
        for (int b = 0; b < p->log2n; b++)
            if (i & (1 << b)) r |= 1 << (p->log2n - 1 - b);
        p->rev[i] = r;
    }
    return 0;
}

static void fft_plan_free(fft_plan *p)
{
    free(p->tw);
    free(p->rev);
}

/* Unnormalised out-of-place DFT: out[k] = sum_n in[n] exp(sign 2 pi i n k / N).
 * sign = +1 is cuFFT's CUFFT_INVERSE, sign = -1 is CUFFT_FORWARD. */
static void fft_exec(const fft_plan *p, const cplx *in, cplx *out, int sign)
{
    const int n = p->n;
    for (int i = 0; i < n; i++) out[p->rev[i]] = in[i];
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1;
        const int step = n / len;
        for (int i = 0; i < n; i += len) {
            for (int j = 0; j < half; j++) {
                cplx w = p->tw[j * step];
                if (sign > 0) w = conj(w);
                cplx u = out[i + j];
                cplx v = out[i + j + half] * w;
                out[i + j] = u + v;
                out[i + j + half] = u - v;
            }
        }
    }
}

void oracle_fft(int n, const cplx *in, cplx *out, int sign)
{
    fft_plan p;
    if (fft_plan_init(&p, n) != 0) return;
    fft_exec(&p, in, out, sign);
    fft_plan_free(&p);
}

/* --------------------------------------------------------- solver state */

typedef struct {
    int n;
    fft_plan plan;
    cplx *k1p, *k2p, *k3p, *k4p, *k1s, *k2s, *k3s, *k4s, *k1i, *k2i, *k3i, *k4i;
    cplx *auxp, *auxs, *auxi, *Apw, *Asw, *Aiw;
} work;

static int work_init(work *W, int n)
{
    memset(W, 0, sizeof(*W));
    W->n = n;
    if (fft_plan_init(&W->plan, n) != 0) return -1;
    cplx **bufs[] = {&W->k1p, &W->k2p, &W->k3p, &W->k4p, &W->k1s, &W->k2s,
                     &W->k3s, &W->k4s, &W->k1i, &W->k2i, &W->k3i, &W->k4i,
                     &W->auxp, &W->auxs, &W->auxi, &W->Apw, &W->Asw, &W->Aiw};
    for (size_t b = 0; b < sizeof(bufs) / sizeof(bufs[0]); b++) {
        *bufs[b] = (cplx *)calloc((size_t)n, sizeof(cplx));
        if (!*bufs[b]) return -1;
    }
    return 0;
}

static void work_free(work *W)
{
    fft_plan_free(&W->plan);
    cplx *bufs[] = {W->k1p, W->k2p, W->k3p, W->k4p, W->k1s, W->k2s, W->k3s,
                    W->k4s, W->k1i, W->k2i, W->k3i, W->k4i, W->auxp, W->auxs,
                    W->auxi, W->Apw, W->Asw, W->Aiw};
    for (size_t b = 0; b < sizeof(bufs) / sizeof(bufs[0]); b++) free(bufs[b]);
}

static inline cplx cpx_exp(real a) { return (real)cos(a) + I * (real)sin(a); }

/* ------------------------------------------------------ 2 equations */

/* cwes2.cuh:30-42 */
static void dAdz2(int n, cplx *dAp, cplx *dAs, const cplx *Ap, const cplx *As,
                  real kp, real ks, real dk, real z)
{
    const cplx ep = cpx_exp(+dk * z), es = cpx_exp(-dk * z);
    for (int i = 0; i < n; i++) {
        dAp[i] = I * kp * As[i] * As[i] * ep;
        dAs[i] = I * ks * Ap[i] * conj(As[i]) * es;
    }
}

/* cwes2.cuh:54-65 */
static void lin_comb2(int n, cplx *auxp, cplx *auxs, const cplx *Ap,
                      const cplx *As, const cplx *kp, const cplx *ks, real s)
{
    for (int i = 0; i < n; i++) {
        auxp[i] = Ap[i] + kp[i] * s;
        auxs[i] = As[i] + ks[i] * s;
    }
}

/* cwes2.cuh:76-87 */
static void rk4_2(int n, cplx *Ap, cplx *As, work *W, real h)
{
    for (int i = 0; i < n; i++) {
        Ap[i] = Ap[i] + (W->k1p[i] + 2 * W->k2p[i] + 2 * W->k3p[i] + W->k4p[i]) * h / 6;
        As[i] = As[i] + (W->k1s[i] + 2 * W->k2s[i] + 2 * W->k3s[i] + W->k4s[i]) * h / 6;
    }
}

/* The RK4 half step, cwes2.cuh:147-166 (and again at :188-207). */
static void rk4_half2(const oracle_params *P, cplx *Ap, cplx *As, work *W, real z)
{
    const int n = W->n;
    const real kp = (real)P->kp, ks = (real)P->ks, dk = (real)P->dk, dz = (real)P->dz;
    dAdz2(n, W->k1p, W->k1s, Ap, As, kp, ks, dk, z);
    lin_comb2(n, W->auxp, W->auxs, Ap, As, W->k1p, W->k1s, (real)0.5);
    dAdz2(n, W->k2p, W->k2s, W->auxp, W->auxs, kp, ks, dk, z + dz / 4);
    lin_comb2(n, W->auxp, W->auxs, Ap, As, W->k2p, W->k2s, (real)0.5);
    dAdz2(n, W->k3p, W->k3s, W->auxp, W->auxs, kp, ks, dk, z + dz / 4);
    lin_comb2(n, W->auxp, W->auxs, Ap, As, W->k3p, W->k3s, (real)1.0);
    dAdz2(n, W->k4p, W->k4s, W->auxp, W->auxs, kp, ks, dk, z + dz / 2);
    rk4_2(n, Ap, As, W, dz / 2);
}

/* cwes2.cuh:103-121, called with z = dz (cwes2.cuh:178). */
static void linear_op2(const oracle_params *P, const real *w, work *W, real z)
{
    const int n = W->n;
    const real vp = (real)P->vp, vs = (real)P->vs;
    const real b2p = (real)P->b2p, b2s = (real)P->b2s;
    const real b3p = (real)P->b3p, b3s = (real)P->b3s;
    const real attenp = (real)exp(-0.5 * P->alpha_crp * (double)z);
    const real attens = (real)exp(-0.5 * P->alpha_crs * (double)z);
    for (int i = 0; i < n; i++) {
        const real wi = w[i];
        cplx auxp = W->Apw[i] * cpx_exp(z * wi * ((1 / vp - 1 / vs) + (real)0.5 * wi * b2p + wi * wi * b3p / 6));
        cplx auxs = W->Asw[i] * cpx_exp(z * wi * ((1 / vs - 1 / vs) + (real)0.5 * wi * b2s + wi * wi * b3s / 6));
        W->Apw[i] = auxp * attenp;
        W->Asw[i] = auxs * attens;
    }
}

static void scale_inv(int n, cplx *A)
{
    const real s = (real)n;
    for (int i = 0; i < n; i++) A[i] = A[i] / s;
}

/* EvolutionInCrystal, cwes2.cuh:132-215. */
void oracle_crystal_pass2(const oracle_params *P, const real *w, cplx *Ap, cplx *As, work *W)
{
    const int n = W->n;
    const real dz = (real)P->dz;
    real z = 0;
    for (int s = 0; s < P->n_z; s++) {
        rk4_half2(P, Ap, As, W, z);
        fft_exec(&W->plan, As, W->Asw, +1);
        scale_inv(n, W->Asw);
        fft_exec(&W->plan, Ap, W->Apw, +1);
        scale_inv(n, W->Apw);
        linear_op2(P, w, W, dz);
        fft_exec(&W->plan, W->Asw, As, -1);
        fft_exec(&W->plan, W->Apw, Ap, -1);
        rk4_half2(P, Ap, As, W, z);
        z += dz;
    }
}

/* ------------------------------------------------------ 3 equations */

/* cwes3.cuh:30-43 */
static void dAdz3(int n, cplx *dAp, cplx *dAs, cplx *dAi, const cplx *Ap,
                  const cplx *As, const cplx *Ai, real kp, real ks, real ki,
                  real dk, real z)
{
    const cplx em = cpx_exp(-dk * z), ep = cpx_exp(+dk * z);
    for (int i = 0; i < n; i++) {
        dAp[i] = I * kp * As[i] * Ai[i] * em;
        dAs[i] = I * ks * Ap[i] * conj(Ai[i]) * ep;
        dAi[i] = I * ki * Ap[i] * conj(As[i]) * ep;
    }
}

/* cwes3.cuh:55-67 */
static void lin_comb3(int n, cplx *auxp, cplx *auxs, cplx *auxi, const cplx *Ap,
                      const cplx *As, const cplx *Ai, const cplx *kp,
                      const cplx *ks, const cplx *ki, real s)
{
    for (int i = 0; i < n; i++) {
        auxp[i] = Ap[i] + kp[i] * s;
        auxs[i] = As[i] + ks[i] * s;
        auxi[i] = Ai[i] + ki[i] * s;
    }
}

/* cwes3.cuh:78-90 */
static void rk4_3(int n, cplx *Ap, cplx *As, cplx *Ai, work *W, real h)
{
    for (int i = 0; i < n; i++) {
        Ap[i] = Ap[i] + (W->k1p[i] + 2 * W->k2p[i] + 2 * W->k3p[i] + W->k4p[i]) * h / 6;
        As[i] = As[i] + (W->k1s[i] + 2 * W->k2s[i] + 2 * W->k3s[i] + W->k4s[i]) * h / 6;
        Ai[i] = Ai[i] + (W->k1i[i] + 2 * W->k2i[i] + 2 * W->k3i[i] + W->k4i[i]) * h / 6;
    }
}

/* cwes3.cuh:154-170: every stage is evaluated on (Ap, As, Ai); the aux
 * vectors are formed but not read (quirk Q3). */
static void rk4_half3(const oracle_params *P, cplx *Ap, cplx *As, cplx *Ai, work *W, real z)
{
    const int n = W->n;
    const real kp = (real)P->kp, ks = (real)P->ks, ki = (real)P->ki;
    const real dk = (real)P->dk, dz = (real)P->dz;
    dAdz3(n, W->k1p, W->k1s, W->k1i, Ap, As, Ai, kp, ks, ki, dk, z);
    lin_comb3(n, W->auxp, W->auxs, W->auxi, Ap, As, Ai, W->k1p, W->k1s, W->k1i, (real)0.5);
    dAdz3(n, W->k2p, W->k2s, W->k2i, Ap, As, Ai, kp, ks, ki, dk, z + dz / 4);
    lin_comb3(n, W->auxp, W->auxs, W->auxi, Ap, As, Ai, W->k2p, W->k2s, W->k2i, (real)0.5);
    dAdz3(n, W->k3p, W->k3s, W->k3i, Ap, As, Ai, kp, ks, ki, dk, z + dz / 4);
    lin_comb3(n, W->auxp, W->auxs, W->auxi, Ap, As, Ai, W->k3p, W->k3s, W->k3i, (real)1.0);
    dAdz3(n, W->k4p, W->k4s, W->k4i, Ap, As, Ai, kp, ks, ki, dk, z + dz / 2);
    rk4_3(n, Ap, As, Ai, W, dz / 2);
}

/* cwes3.cuh:107-128: GVM terms (1/vp-1/vi), 0, (1/vi-1/vs) (quirk Q4). */
static void linear_op3(const oracle_params *P, const real *w, work *W, real z)
{
    const int n = W->n;
    const real vp = (real)P->vp, vs = (real)P->vs, vi = (real)P->vi;
    const real b2p = (real)P->b2p, b2s = (real)P->b2s, b2i = (real)P->b2i;
    const real b3p = (real)P->b3p, b3s = (real)P->b3s, b3i = (real)P->b3i;
    const real attenp = (real)exp(-0.5 * P->alpha_crp * (double)z);
    const real attens = (real)exp(-0.5 * P->alpha_crs * (double)z);
    const real atteni = (real)exp(-0.5 * P->alpha_cri * (double)z);
    for (int i = 0; i < n; i++) {
        const real wi = w[i];
        cplx auxp = W->Apw[i] * cpx_exp(z * wi * ((1 / vp - 1 / vi) + (real)0.5 * wi * b2p + wi * wi * b3p / 6));
        cplx auxs = W->Asw[i] * cpx_exp(z * wi * ((1 / vs - 1 / vs) + (real)0.5 * wi * b2s + wi * wi * b3s / 6));
        cplx auxi = W->Aiw[i] * cpx_exp(z * wi * ((1 / vi - 1 / vs) + (real)0.5 * wi * b2i + wi * wi * b3i / 6));
        W->Apw[i] = auxp * attenp;
        W->Asw[i] = auxs * attens;
        W->Aiw[i] = auxi * atteni;
    }
}

/* EvolutionInCrystal (3 eqs), cwes3.cuh:139-225. */
void oracle_crystal_pass3(const oracle_params *P, const real *w, cplx *Ap, cplx *As, cplx *Ai, work *W)
{
    const int n = W->n;
    const real dz = (real)P->dz;
    real z = 0;
    for (int s = 0; s < P->n_z; s++) {
        rk4_half3(P, Ap, As, Ai, W, z);
        fft_exec(&W->plan, As, W->Asw, +1);
        scale_inv(n, W->Asw);
        fft_exec(&W->plan, Ai, W->Aiw, +1);
        scale_inv(n, W->Aiw);
        fft_exec(&W->plan, Ap, W->Apw, +1);
        scale_inv(n, W->Apw);
        linear_op3(P, w, W, dz);
        fft_exec(&W->plan, W->Asw, As, -1);
        fft_exec(&W->plan, W->Aiw, Ai, -1);
        fft_exec(&W->plan, W->Apw, Ap, -1);
        rk4_half3(P, Ap, As, Ai, W, z);
        z += dz;
    }
}

/* ----------------------------------------------------------- cavity map */

/* PhaseModulatorIntraCavity, functions.cuh:242-253 */
static void eom(int n, cplx *A, real m, real fpm, const real *T)
{
    for (int i = 0; i < n; i++)
        A[i] = A[i] * cpx_exp(m * (real)sin(2 * ORACLE_PI * (double)fpm * (double)T[i]));
}

/* cuOPO.cu:521-553: IFFT, CUFFTscale, AddGDD (functions.cuh:156-169) or
 * AddGDDTOD (functions.cuh:173-186), FFT. */
static void gdd_comp(cplx *A, cplx *Aw, const real *w, real gdd, real tod,
                     int use_tod, work *W)
{
    const int n = W->n;
    fft_exec(&W->plan, A, Aw, +1);
    scale_inv(n, Aw);
    for (int i = 0; i < n; i++) {
        const real wi = w[i];
        if (use_tod)
            Aw[i] = Aw[i] * cpx_exp((real)0.5 * wi * (wi * gdd + wi * wi * tod / (real)3.0));
        else
            Aw[i] = Aw[i] * cpx_exp((real)0.5 * wi * wi * gdd);
    }
    fft_exec(&W->plan, Aw, A, -1);
}

/* AddPhase, functions.cuh:139-152 */
static void add_phase(int n, cplx *A, real R, real delta)
{
    const cplx f = (real)sqrt((double)R) * cpx_exp((real)ORACLE_PI * delta);
    for (int i = 0; i < n; i++) A[i] = A[i] * f;
}

/* ReadPump, functions.cuh:191-213, including the off-by-one offset of the
 * last round trip (quirk Q6). */
static void read_pump(int n, cplx *Ap, const cplx *total, int n_rt, int nn)
{
    long off;
    if (nn == 0) off = 0;
    else if (nn > 0 && nn < n_rt - 1) off = (long)nn * n;
    else off = (long)n * n_rt - 1 - n;
    for (int i = 0; i < n; i++) Ap[i] = total[off + i];
}

static double signal_power(int n, const cplx *As)
{
    double acc = 0.0;
    for (int i = 0; i < n; i++) {
        const double re = (double)creal(As[i]), im = (double)cimag(As[i]);
        acc += re * re + im * im;
    }
    return acc / (double)n;
}

/*
 * Runs round trips nn = rt_begin .. rt_begin+rt_count-1 of the loop body
 * src/cuOPO.cu:474-610 on the fields (Ap, As[, Ai]) in place.
 *
 *  pump      CW: n_t values copied to Ap every rt (cuOPO.cu:480);
 *            NS: the n_t * n_rt pump window read by ReadPump (cuOPO.cu:484).
 *  save_*    round trips nn in [save_first, save_first + save_count) are
 *            stored at slot nn - save_first (SaveRoundTrip,
 *            cuOPO.cu:570-608).  Any pointer may be NULL.
 *  ps_hist   if not NULL, receives (1/N) sum |As|^2 after each rt.
 * Returns 0, or -1 on a bad argument or allocation failure.
 */
int oracle_round_trips(const oracle_params *P, const real *w, const real *T,
                       cplx *Ap, cplx *As, cplx *Ai,
                       const cplx *pump, int n_rt,
                       int rt_begin, int rt_count,
                       cplx *sv_p, cplx *sv_s, cplx *sv_i,
                       int save_first, int save_count,
                       double *ps_hist)
{
    const int n = P->n_t;
    if (ilog2(n) < 1 || (P->n_eqs != 2 && P->n_eqs != 3)) return -1;
    if (P->n_eqs == 3 && !Ai) return -1;
    work W;
    if (work_init(&W, n) != 0) { work_free(&W); return -1; }
    const int three = (P->n_eqs == 3);
    const int use_tod_s = (P->tod_s != 0 && P->b3s != 0);
    const int use_tod_i = (P->tod_i != 0 && P->b3i != 0);
    for (int nn = rt_begin; nn < rt_begin + rt_count; nn++) {
        if (P->regime == 0) memcpy(Ap, pump, sizeof(cplx) * (size_t)n);
        else read_pump(n, Ap, pump, n_rt, nn);

        if (three) oracle_crystal_pass3(P, w, Ap, As, Ai, &W);
        else oracle_crystal_pass2(P, w, Ap, As, &W);

        if (P->use_eom) {
            eom(n, As, (real)P->mod_depth, (real)P->fpm, T);
            if (three && P->eom_idler) eom(n, Ai, (real)P->mod_depth, (real)P->fpm, T);
        }
        if (P->gdd != 0) {
            gdd_comp(As, W.Asw, w, (real)P->gdd, (real)P->tod_s, use_tod_s, &W);
            if (three) gdd_comp(Ai, W.Aiw, w, (real)P->gdd, (real)P->tod_i, use_tod_i, &W);
        }
        add_phase(n, As, (real)P->Rs, (real)P->delta);
        if (three) add_phase(n, Ai, (real)P->Ri, (real)P->delta);

        if (nn >= save_first && nn < save_first + save_count) {
            const size_t slot = (size_t)(nn - save_first) * (size_t)n;
            if (sv_s) memcpy(sv_s + slot, As, sizeof(cplx) * (size_t)n);
            if (sv_p) memcpy(sv_p + slot, Ap, sizeof(cplx) * (size_t)n);
            if (three && sv_i) memcpy(sv_i + slot, Ai, sizeof(cplx) * (size_t)n);
        }
        if (ps_hist) ps_hist[nn - rt_begin] = signal_power(n, As);
    }
    work_free(&W);
    return 0;
}

/* One crystal pass (EvolutionInCrystal) on the fields in place. */
int oracle_crystal_pass(const oracle_params *P, const real *w, cplx *Ap, cplx *As, cplx *Ai)
{
    work W;
    if (work_init(&W, P->n_t) != 0) { work_free(&W); return -1; }
    if (P->n_eqs == 3) {
        if (!Ai) { work_free(&W); return -1; }
        oracle_crystal_pass3(P, w, Ap, As, Ai, &W);
    } else {
        oracle_crystal_pass2(P, w, Ap, As, &W);
    }
    work_free(&W);
    return 0;
}

/*
 * Runs round trips until the relative change of the signal power between
 * consecutive round trips drops below tol (checked from the second rt on),
 * or max_rt round trips have run.  This is the convergence rule of the
 * batched CW sweep; the reference itself always runs a fixed NRT.
 * Returns the number of round trips run; *ps_out gets the final power.
 */
int oracle_solve(const oracle_params *P, const real *w, const real *T,
                 cplx *Ap, cplx *As, cplx *Ai, const cplx *pump, int n_rt,
                 int max_rt, double tol, double *ps_out, int *converged)
{
    double prev = -1.0, ps = 0.0;
    int rt;
    *converged = 0;
    for (rt = 0; rt < max_rt; rt++) {
        if (oracle_round_trips(P, w, T, Ap, As, Ai, pump, n_rt, rt, 1,
                               NULL, NULL, NULL, 0, 0, &ps) != 0)
            return -1;
        if (prev > 0.0 && ps > 0.0 && fabs(ps - prev) < tol * ps) {
            *converged = 1;
            rt++;
            break;
        }
        prev = ps;
    }
    *ps_out = ps;
    return rt;
}
