/*
 * params.c -- host-side set-up of the solver: crystal dispersion models,
 * phase-matching temperature scan, parameter derivation, time/frequency
 * grids and pump inputs.
 *
 * The reference evaluates all of this in single precision on the host
 * (src/cuOPO.cu:92-234).  The solver's results depend on these values, so
 * the arithmetic (setup_math.h) follows the reference's float/double
 * promotions exactly; compiled here for the host it is bit-exact.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "cuopo.h"
#include "internal.h"
#include "setup_math.h"

float cuopo_sellmeier(int crystal, int which, float L, float T)
{
    switch (which) {
    case 0: return cr_n(crystal, L, T);
    case 1: return cr_dndl(crystal, L, T);
    case 2: return cr_d2(crystal, L, T);
    case 3: return cr_d3(crystal, L, T);
    case 4: return cr_gv(crystal, L, T);
    case 5: return cr_gvd(crystal, L, T);
    case 6: return cr_tod(crystal, L, T);
    default: return NAN;
    }
}

void cuopo_linspace(float *out, long n, float xmin, float xmax)
{
    /* functions.cuh:12-18: the int index times a float step, in float. */
    const float span = xmax - xmin;
    const float den = (float)(int)(n - 1);
    for (long i = 0; i < n; i++) out[i] = xmin + (float)(int)i * span / den;
}

float cuopo_phase_matching_temp(int crystal, float lp, float ls, float lambda_um,
                                float t_min, float t_max)
{
    /* functions.cuh:23-54: 5000-point scan of the SHG form of the mismatch,
     * 2 pi / lp |n(ls) - n(lp)| - 2 pi / Lambda; first minimum of |dk|. */
    enum { M = 5000 };
    float *T = (float *)malloc(sizeof(float) * 2 * M);
    if (!T) return NAN;
    float *d = T + M;
    cuopo_linspace(T, M, t_min, t_max);
    for (int i = 0; i < M; i++) d[i] = pm_mismatch(crystal, lp, ls, lambda_um, T[i]);
    int pos = 0;
    for (int i = 1; i < M; i++)
        if (fabsf(d[i]) < fabsf(d[pos])) pos = i;
    const float t = T[pos];
    free(T);
    return t;
}

void cuopo_inputs_default(cuopo_inputs *in)
{
    memset(in, 0, sizeof(*in));
    in->crystal = CUOPO_PPLN;
    in->n_eqs = 2;
    in->regime = CUOPO_CW;
    in->n_t = 1 << 14;
    in->n_z = 150;
    in->n_rt = 10000;
    in->lp_nm = 532;
    in->temp_c = 27;
    in->lambda_um = 6.97;
    in->n_thr = 4;
    in->r_percent = 98;
    in->lcr_mm = 5;
    in->temp_from_scan = 1;
    in->lcav_um = 100e3;
    in->ri = 0.98;
    in->waist_um = 55;
    in->fwhm_ps = 10000;
}

static int is_pow2(long n) { return n > 0 && (n & (n - 1)) == 0; }

cuopo_status cuopo_derive_params(const cuopo_inputs *in, cuopo_params *p, cuopo_info *info)
{
    if (!in || !p) return cuopo_fail(CUOPO_EINVAL, "derive_params: NULL argument");
    if (in->n_eqs != 2 && in->n_eqs != 3) return cuopo_fail(CUOPO_EINVAL, "n_eqs must be 2 or 3");
    if (!is_pow2(in->n_t) || in->n_t < 16) return cuopo_fail(CUOPO_EINVAL, "n_t must be a power of 2 >= 16");
    if (in->n_z < 1) return cuopo_fail(CUOPO_EINVAL, "n_z must be >= 1");
    if (in->crystal != CUOPO_PPLN && in->crystal != CUOPO_SPPLT)
        return cuopo_fail(CUOPO_EINVAL, "unknown crystal");
    /* cuOPO.cu:92-101: the temperature comes from the scan (argv[2] is unused) */
    const float lp = (float)(in->lp_nm * 1e-3);
    const float ls = in->ls_nm > 0 ? (float)(in->ls_nm * 1e-3) : 2 * lp;
    const float Temp = in->temp_from_scan ? cuopo_phase_matching_temp(in->crystal, lp, ls, (float)in->lambda_um, 10, 150)
                                          : (float)in->temp_c;
    derive_core(in, Temp, p, info);
    return CUOPO_OK;
}

cuopo_status cuopo_make_grids(int n_t, double t_rt, float *T, float *w)
{
    if (!is_pow2(n_t) || n_t < 2) return cuopo_fail(CUOPO_EINVAL, "make_grids: n_t must be a power of 2");
    const float trt = (float)t_rt;
    if (T) cuopo_linspace(T, n_t, (float)(-0.5 * (double)trt), (float)(0.5 * (double)trt));
    if (w) {
        /* cuOPO.cu:151,183-189: F = linspace(-N dF/2, N dF/2), w = 2 pi fftshift(F). */
        const float dF = 1 / trt;
        float *F = (float *)malloc(sizeof(float) * (size_t)n_t);
        if (!F) return cuopo_fail(CUOPO_ENOMEM, "make_grids: out of host memory");
        cuopo_linspace(F, n_t, (float)(-0.5 * (double)(unsigned)n_t * (double)dF),
                       (float)(+0.5 * (double)(unsigned)n_t * (double)dF));
        const int c = n_t / 2;
        for (int i = 0; i < c; i++) {
            w[i + c] = F[i];
            w[i] = F[i + c];
        }
        for (int i = 0; i < n_t; i++) w[i] = 2 * F_PI * w[i];
        free(F);
    }
    return CUOPO_OK;
}

cuopo_status cuopo_pump_cw(float *out, int n_t, double ap0)
{
    if (!out || n_t < 1) return cuopo_fail(CUOPO_EINVAL, "pump_cw: bad argument");
    const float a = (float)ap0;
    for (int i = 0; i < n_t; i++) { out[2 * i] = a; out[2 * i + 1] = 0.f; }
    return CUOPO_OK;
}

cuopo_status cuopo_pump_ns(float *out, int n_t, int n_rt, double t_rt, double ap0, double fwhm_ps)
{
    if (!out || n_t < 1 || n_rt < 1) return cuopo_fail(CUOPO_EINVAL, "pump_ns: bad argument");
    const long n = (long)n_t * (long)n_rt;
    /* cuOPO.cu:165-166,174-175: Tp = linspace over SIZE*NRT points of the
     * saved window t_rt*NRT (the float index rounding included). */
    const float T_width = (float)t_rt * (float)(unsigned)n_rt;
    float *Tp = (float *)malloc(sizeof(float) * (size_t)n);
    if (!Tp) return cuopo_fail(CUOPO_ENOMEM, "pump_ns: out of host memory");
    cuopo_linspace(Tp, n, (float)(-0.5 * (double)T_width), (float)(0.5 * (double)T_width));
    /* cuOPO.cu:244-247 and functions.cuh:77-85 */
    const float FWHM = (float)fwhm_ps;
    const float sigmap = FWHM * sqrtf(2) / (2 * sqrtf(2 * logf(2)));
    const float A0 = (float)ap0;
    for (long i = 0; i < n; i++) {
        out[2 * i] = A0 * expf(-(Tp[i] * Tp[i]) / (2 * sigmap * sigmap));
        out[2 * i + 1] = 0.f;
    }
    free(Tp);
    return CUOPO_OK;
}
