/*
 * setup_math.h -- the reference's host-side set-up arithmetic, shared by the
 * host library code (params.c, bit-exact with the reference) and the
 * batched device set-up (params_dev.cu).  Sellmeier models of MgO:PPLN
 * (src/headers/ppln.cuh:33-189) and MgO:sPPLT (src/headers/spplt.cuh:31-153)
 * and the parameter derivation of src/cuOPO.cu:92-234.
 *
 * Every expression is evaluated with the same float/double promotions the
 * reference's C++ gets: a double literal promotes its operation to double;
 * std::pow(float,int) is pow(double,double); powf, sqrtf, logf stay in
 * float.  Casts are written out where C would otherwise promote
 * differently.  On the host (glibc) the results are bit-exact with the
 * reference's; on the device CUDA's powf/pow/logf may round differently in
 * the last bits.
 */
#ifndef CUOPO_SETUP_MATH_H
#define CUOPO_SETUP_MATH_H

#include <math.h>
#include <string.h>

#include "cuopo.h"

#ifdef __CUDACC__
#define CUOPO_HD __host__ __device__
#else
#define CUOPO_HD
#endif

/* Same constants as src/cuOPO.cu:24-26, rounded to float as there. */
#define F_PI ((float)3.14159265358979323846)
#define F_C ((float)(299792458 * 1E6 / 1E12))
#define F_EPS0 ((float)(8.8541878128E-12 * 1E12 / 1E6))

/* ------------------------------------------------- MgO:PPLN (ppln.cuh) */

/* Material constants, src/headers/ppln.cuh:21-26. */
#define PPLN_DEFF 25.2e-6f
#define PPLN_DQ ((float)(2.0 * (double)PPLN_DEFF / (double)F_PI))

/* Temperature-dependent Sellmeier coefficients (ppln.cuh:36-50). */
typedef struct { float G1, G2, G3, G4, a5, a6; } ppln_coef;

CUOPO_HD static inline ppln_coef ppln_coefs(float T)
{
    ppln_coef c;
    const float f = (float)(((double)T - 24.5) * ((double)T + 570.82));
    c.G1 = 5.756f + 2.860e-6f * f;
    c.G2 = 0.0983f + 4.700e-8f * f;
    c.G3 = 0.2020f + 6.113e-8f * f;
    c.G4 = 189.32f + 1.516e-4f * f;
    c.a5 = 12.52f;
    c.a6 = 1.32e-2f;
    return c;
}

CUOPO_HD static inline float ppln_n(float L, float T)
{
    const ppln_coef c = ppln_coefs(T);
    const float L2 = powf(L, 2);
    return sqrtf(c.G1 + c.G2 / (L2 - powf(c.G3, 2)) + c.G4 / (L2 - powf(c.a5, 2)) - c.a6 * L * L);
}

/* The pole sum of ppln.cuh:57-78. */
CUOPO_HD static inline float ppln_res(float L, float T, int p)
{
    const ppln_coef c = ppln_coefs(T);
    const float L2 = powf(L, 2);
    return c.G2 / powf(L2 - powf(c.G3, 2), (float)p) + c.G4 / powf(L2 - powf(c.a5, 2), (float)p);
}

CUOPO_HD static inline float ppln_dndl(float L, float T)
{
    return -L * (ppln_res(L, T, 2) + 1.32e-2f) / ppln_n(L, T);
}

CUOPO_HD static inline float ppln_d2ndl2(float L, float T)
{
    const float nn = ppln_n(L, T);
    const float A = (L * ppln_dndl(L, T) / powf(nn, 2) - 1 / nn) * (ppln_res(L, T, 2) + 1.32e-2f);
    const float B = 4 * L * L / nn * ppln_res(L, T, 3);
    return A + B;
}

CUOPO_HD static inline float ppln_d3ndl3(float L, float T)
{
    const float nn = ppln_n(L, T);
    const float d1 = ppln_dndl(L, T), d2 = ppln_d2ndl2(L, T);
    const float A1 = (2 * d1 + L * d2) / powf(nn, 2);
    const float A2 = -2 * L * powf(d1, 2) / powf(nn, 3);
    const float AA = (A1 + A2) * (ppln_res(L, T, 2) + 1.32e-2f);
    const float B1 = 12 * L / nn;
    const float B2 = -4 * L * L / nn * d2 * (1 - 1 / nn);
    const float BB = (B1 + B2) * ppln_res(L, T, 3);
    const float CC = -24 * L * L * L / nn * ppln_res(L, T, 4);
    return AA + BB + CC;
}

/* ----------------------------------------------- MgO:sPPLT (spplt.cuh) */

/* Material constants, src/headers/spplt.cuh:19-27. */
#define SPPLT_DEFF 11.00e-6f
#define SPPLT_DQ ((float)(2.0 * (double)SPPLT_DEFF / (double)F_PI))

typedef struct { float A, B, C, D, E, F, G, H, b, c; } spplt_coef;

/* spplt.cuh:31-46; b and c go through a double pow. */
CUOPO_HD static inline spplt_coef spplt_coefs(float T)
{
    spplt_coef k;
    k.A = 4.502483f; k.B = 0.007294f; k.C = 0.185087f; k.D = -0.02357f;
    k.E = 0.073423f; k.F = 0.199595f; k.G = 0.001f; k.H = 7.99724f;
    k.b = (float)(3.483933e-8 * pow((double)T + 273.15, 2));
    k.c = (float)(1.607839e-8 * pow((double)T + 273.15, 2));
    return k;
}

CUOPO_HD static inline float spplt_n(float L, float T)
{
    const spplt_coef k = spplt_coefs(T);
    const double L2 = pow((double)L, 2);
    const double s = (double)k.A + (double)(k.B + k.b) / (L2 - pow((double)(k.C + k.c), 2)) +
                     (double)k.E / (L2 - pow((double)k.F, 2)) +
                     (double)k.G / (L2 - pow((double)k.H, 2)) + (double)k.D * L2;
    return (float)sqrt(s);
}

CUOPO_HD static inline float spplt_res(float L, float T, int p)
{
    const spplt_coef k = spplt_coefs(T);
    const float L2 = powf(L, 2);
    return (k.B + k.b) / powf(L2 - powf(k.C + k.c, 2), (float)p) +
           k.E / powf(L2 - powf(k.F, 2), (float)p) +
           k.G / powf(L2 - powf(k.H, 2), (float)p);
}

CUOPO_HD static inline float spplt_dndl(float L, float T)
{
    return -L / spplt_n(L, T) * (spplt_res(L, T, 2) - (-0.02357f));
}

CUOPO_HD static inline float spplt_d2ndl2(float L, float T)
{
    const float nn = spplt_n(L, T);
    return (L / powf(nn, 2) * spplt_dndl(L, T) - 1 / nn) * (spplt_res(L, T, 2) - (-0.02357f)) +
           4 * L * L / nn * spplt_res(L, T, 3);
}

CUOPO_HD static inline float spplt_d3ndl3(float L, float T)
{
    const float nn = spplt_n(L, T);
    const float d1 = spplt_dndl(L, T), d2 = spplt_d2ndl2(L, T);
    const float A1 = (2 * d1 + L * d2) / powf(nn, 2);
    const float A2 = -2 * L * powf(d1, 2) / powf(nn, 3);
    const float AA = (A1 + A2) * (spplt_res(L, T, 2) - (-0.02357f));
    const float B1 = 12 * L / nn;
    const float B2 = -4 * L * L / nn * d2 * (1 - 1 / nn);
    const float BB = (B1 + B2) * spplt_res(L, T, 3);
    const float CC = -24 * L * L * L / nn * spplt_res(L, T, 4);
    return AA + BB + CC;
}

/* ------------------------------------------------------------ common */

CUOPO_HD static inline float cr_n(int cr, float L, float T) { return cr == CUOPO_SPPLT ? spplt_n(L, T) : ppln_n(L, T); }
CUOPO_HD static inline float cr_dndl(int cr, float L, float T) { return cr == CUOPO_SPPLT ? spplt_dndl(L, T) : ppln_dndl(L, T); }
CUOPO_HD static inline float cr_d2(int cr, float L, float T) { return cr == CUOPO_SPPLT ? spplt_d2ndl2(L, T) : ppln_d2ndl2(L, T); }
CUOPO_HD static inline float cr_d3(int cr, float L, float T) { return cr == CUOPO_SPPLT ? spplt_d3ndl3(L, T) : ppln_d3ndl3(L, T); }

/* GV, GVD, TOD: ppln.cuh:171-189 / spplt.cuh:130-153.  GVD of sPPLT uses
 * std::pow(L,3) (double); the others use powf. */
CUOPO_HD static inline float cr_gv(int cr, float L, float T) { return F_C / (cr_n(cr, L, T) - L * cr_dndl(cr, L, T)); }

CUOPO_HD static inline float cr_gvd(int cr, float L, float T)
{
    if (cr == CUOPO_SPPLT)
        return (float)(pow((double)L, 3) * (double)cr_d2(cr, L, T) / (double)(2 * F_PI * F_C * F_C));
    return powf(L, 3) * cr_d2(cr, L, T) / (2 * F_PI * F_C * F_C);
}

CUOPO_HD static inline float cr_tod(int cr, float L, float T)
{
    return -powf(L, 4) / (4 * F_PI * F_PI * F_C * F_C * F_C) * (3 * cr_d2(cr, L, T) + L * cr_d3(cr, L, T));
}

/* The phase mismatch the temperature scan minimises, functions.cuh:23-54:
 * the SHG form 2 pi / lp |n(ls) - n(lp)| - 2 pi / Lambda. */
CUOPO_HD static inline float pm_mismatch(int cr, float lp, float ls, float lambda_um, float T)
{
    return 2 * F_PI / lp * fabsf(cr_n(cr, ls, T) - cr_n(cr, lp, T)) - 2 * F_PI / lambda_um;
}

/* The parameter derivation of src/cuOPO.cu:92-234 for valid inputs and a
 * given crystal temperature (the scan of functions.cuh:23-54, or argv[2]). */
CUOPO_HD static inline void derive_core(const cuopo_inputs *in, float Temp, cuopo_params *p, cuopo_info *info)
{
    const int cr = in->crystal;
    const int three = in->n_eqs == 3;
    const float dQ = cr == CUOPO_SPPLT ? SPPLT_DQ : PPLN_DQ;
    const float alpha[3] = {0.025e-4f, 0.002e-4f, 0.002e-4f};   /* ppln.cuh:24-26 = spplt.cuh:23-25 */

    /* cuOPO.cu:92-101 */
    const float lp = (float)(in->lp_nm * 1e-3);
    const float ls = in->ls_nm > 0 ? (float)(in->ls_nm * 1e-3) : 2 * lp;
    const float li = lp * ls / (ls - lp);
    const float Lambda = (float)in->lambda_um;
    const float Lcr = (float)(in->lcr_mm * 1e3);

    /* cuOPO.cu:103-120; the TOD terms are multiplied by 0. (double) */
    const float np = cr_n(cr, lp, Temp), vp = cr_gv(cr, lp, Temp), b2p = cr_gvd(cr, lp, Temp);
    const float b3p = (float)(0. * (double)cr_tod(cr, lp, Temp));
    const float kp = 2 * F_PI * dQ / (np * lp);
    const float ns = cr_n(cr, ls, Temp), vs = cr_gv(cr, ls, Temp), b2s = cr_gvd(cr, ls, Temp);
    const float b3s = (float)(0. * (double)cr_tod(cr, ls, Temp));
    const float ks = 2 * F_PI * dQ / (ns * ls);
    float ni = 0, vi = 0, b2i = 0, b3i = 0, ki = 0;
    if (three) {
        ni = cr_n(cr, li, Temp);
        vi = cr_gv(cr, li, Temp);
        b2i = cr_gvd(cr, li, Temp);
        b3i = (float)(0. * (double)cr_tod(cr, li, Temp));
        ki = 2 * F_PI * dQ / (ni * li);
    }
    /* cuOPO.cu:122-126 */
    const float dk = three ? 2 * F_PI * (np / lp - ns / ls - ni / li - 1 / Lambda)
                           : 2 * F_PI * (np / lp - 2 * ns / ls - 1 / Lambda);
    const float dkp = 1 / vp - 1 / vs;
    /* cuOPO.cu:129-146 */
    const float Lcav = (float)in->lcav_um;
    const float Rs = (float)(in->r_percent * 0.01);
    const float alphas = (float)(0.5 * (double)((1 - Rs) + alpha[1] * Lcr));
    const float Ri = (float)in->ri;
    const float alphai = (float)(0.5 * (double)((1 - Ri) + alpha[2] * Lcr));
    const float t_rt = (Lcav + Lcr * (ns - 1)) / F_C;
    const float FSR = 1 / t_rt;
    const float finesse = 2 * F_PI / (1 - Rs);
    const float delta = (float)in->delta;
    const float epsilon = (float)(in->gdd_percent * 0.01);
    const float GDD = -epsilon * b2s * Lcr;
    const float TODs = (float)(-0.01 * in->tod_percent * (double)b3s * (double)Lcr);
    const float TODi = (float)(-0.01 * in->tod_percent * (double)b3i * (double)Lcr);
    /* cuOPO.cu:149-151 */
    const float dz = Lcr / (float)(unsigned)in->n_z;
    const float dT = t_rt / (float)(unsigned)in->n_t;
    const float dF = 1 / t_rt;
    /* cuOPO.cu:202-234; both fields resonant (cuOPO.cu:195-198) */
    const float waist = (float)in->waist_um;
    const float spot = F_PI * waist * waist;
    float Ith;
    if (three)
        Ith = F_EPS0 * F_C * np * ns * ni * ls * li * powf((1 / dQ / Lcr / F_PI), 2) * alphas * alphai / 8;
    else
        Ith = F_EPS0 * F_C * np * powf((ns * ls * alphas / dQ / Lcr / F_PI), 2) / 8;
    const float Pth = Ith * spot;
    const float Nth = (float)in->n_thr;
    const float Inten = (float)(in->n_thr * (double)Ith);
    const float Power = Inten * spot;
    const float Ap0 = sqrtf(2 * Inten / (np * F_EPS0 * F_C));
    const float GammaL = three ? 2 * F_PI * dQ * Ap0 * Lcr / sqrtf(ns * ni * ls * li)
                               : 2 * F_PI * dQ * Ap0 * Lcr / (ns * ls);
    /* cuOPO.cu:263-269 */
    float mod_depth = 0, fpm = 0;
    if (in->use_eom) {
        mod_depth = (float)(in->mod_depth_pi * (double)F_PI);
        const float df = (float)(in->freq_det_mhz * (double)sqrtf(Nth - 1) * (double)alphas /
                                 (double)(F_PI * mod_depth) * (double)FSR);
        fpm = FSR - df;
    }

    memset(p, 0, sizeof(*p));
    p->n_eqs = in->n_eqs;
    p->n_t = in->n_t;
    p->n_z = in->n_z;
    p->regime = in->regime;
    p->vp = vp; p->vs = vs; p->vi = vi;
    p->b2p = b2p; p->b2s = b2s; p->b2i = b2i;
    p->b3p = b3p; p->b3s = b3s; p->b3i = b3i;
    p->dk = dk; p->kp = kp; p->ks = ks; p->ki = ki; p->dz = dz;
    p->alpha_crp = alpha[0]; p->alpha_crs = alpha[1]; p->alpha_cri = alpha[2];
    p->Rs = Rs; p->Ri = Ri; p->delta = delta;
    p->gdd = GDD; p->tod_s = TODs; p->tod_i = TODi;
    p->use_eom = in->use_eom; p->eom_idler = 1;
    p->mod_depth = mod_depth; p->fpm = fpm;
    p->t_rt = t_rt;
    p->ap0 = Ap0;
    if (info) {
        memset(info, 0, sizeof(*info));
        info->temp_c = Temp; info->np = np; info->ns = ns; info->ni = ni; info->li = li;
        info->dkp = dkp; info->t_rt = t_rt; info->fsr = FSR; info->finesse = finesse;
        info->ith = Ith; info->pth = Pth; info->power = Power; info->gamma_l = GammaL;
        info->alphas = alphas; info->alphai = alphai;
        /* cuOPO.cu:245 */
        info->sigmap = (float)in->fwhm_ps * sqrtf(2) / (2 * sqrtf(2 * logf(2)));
        info->dT = dT; info->dF = dF;
    }
}


#endif
