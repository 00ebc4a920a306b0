/*
 * ref_harness.cu -- builds the reference's own SSFM code into a shared
 * library under oracle/_ref/ so that tests can run it as a parity oracle.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Nothing of the reference is copied: this file #includes the reference's
 * headers where they lie (src/headers/*.cuh) and supplies only what the
 * reference's main program (src/cuOPO.cu) would have supplied before those
 * includes, plus a loop body that calls the reference's own kernels in the
 * order of src/cuOPO.cu:474-610.  The harness-only changes are:
 *   - SIZE is chosen at compile time (-DREF_SIZE=...), NZ at run time;
 *   - initial fields and the pump come from the caller (no clock-seeded
 *     noise, src/headers/functions.cuh:58-71);
 *   - the round-trip loop is timed with CUDA events;
 *   - the signal power (1/N) sum |As|^2 can be taken after each round trip
 *     (a small reduction kernel defined here) for the convergence rule.
 * CHECK (src/headers/common.cuh:6-16) is replaced by one that records the
 * first CUDA error instead of calling exit().
 *
 * Build recipe: oracle/build_ref.sh.  Crystal: -DPPLN or -DSPPLT.
 */
#include <iostream>
#include <string>
#include <random>
#include <fstream>
#include <iomanip>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <chrono>
#include <sys/time.h>
#include <sys/types.h>
#include <cuda_runtime.h>
#include <cufft.h>

using real_t = float;
using complex_t = cufftComplex;

/* Same values as the reference's global constants (src/cuOPO.cu:24-26);
 * the headers below read them by these names. */
const real_t PI   = 3.14159265358979323846;
const real_t C    = 299792458*1E6/1E12;
const real_t EPS0 = 8.8541878128E-12*1E12/1E6;

#ifndef REF_SIZE
#error "REF_SIZE must be defined"
#endif
const uint SIZE = REF_SIZE;
static uint NZ = 100;          /* read only by host code in EvolutionInCrystal */
const uint BLKX = 16;

static cudaError_t g_first_error = cudaSuccess;
#define CHECK(call)                                                     \
    {                                                                   \
        const cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess && g_first_error == cudaSuccess)          \
            g_first_error = e_;                                         \
    }

#include "headers/operators.cuh"
#ifdef PPLN
#include "headers/ppln.cuh"
#endif
#ifdef SPPLT
#include "headers/spplt.cuh"
#endif
#include "headers/functions.cuh"
#include "headers/cwes2.cuh"
#include "headers/cwes3.cuh"

/* Mirror of oracle_params in ssfm_oracle.c (same field order). */
struct ref_params {
    int n_eqs, n_t, n_z, regime;
    double vp, vs, vi, b2p, b2s, b2i, b3p, b3s, b3i;
    double dk, kp, ks, ki, dz;
    double alpha_crp, alpha_crs, alpha_cri;
    double Rs, Ri, delta, gdd, tod_s, tod_i;
    int use_eom, eom_idler;
    double mod_depth, fpm;
};

/* Harness reduction: sum |A|^2 into one double (one block). */
__global__ void harness_power(const complex_t *A, double *out)
{
    __shared__ double part[256];
    double acc = 0.0;
    for (uint i = threadIdx.x; i < SIZE; i += blockDim.x) {
        const double re = A[i].x, im = A[i].y;
        acc += re * re + im * im;
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0] / (double)SIZE;
}

extern "C" {

int ref_size(void) { return (int)SIZE; }

/* ---- host-side reference functions (callable without a GPU) ---- */
float ref_n(float L, float T) { return n(L, T); }
float ref_dndl(float L, float T) { return dndl(L, T); }
float ref_d2ndl2(float L, float T) { return d2ndl2(L, T); }
float ref_d3ndl3(float L, float T) { return d3ndl3(L, T); }
float ref_GV(float L, float T) { return GV(L, T); }
float ref_GVD(float L, float T) { return GVD(L, T); }
float ref_TOD(float L, float T) { return TOD(L, T); }
float ref_dQ(void) { return dQ; }
float ref_deff(void) { return deff; }
float ref_alpha(int which) { return which == 0 ? alpha_crp : (which == 1 ? alpha_crs : alpha_cri); }
float ref_find_pm_temp(float lp, float ls, float Lambda, float tmin, float tmax)
{
    return findPhaseMatchingTemp(lp, ls, Lambda, tmin, tmax);
}
void ref_linspace(float *T, int n, float xmin, float xmax) { linspace(T, n, xmin, xmax); }
void ref_fftshift(float *out, float *in, int n) { fftshift(out, in, n); }
void ref_input_field_cw(float2 *A, float A0, int n) { input_field_T(A, A0, n); }
void ref_input_field_gauss(float2 *A, float A0, float *T, float T0, int n)
{
    input_field_T(A, A0, T, T0, n);
}

/*
 * The 2-equation CW set-up of the reference's main program
 * (src/cuOPO.cu:92-234), evaluated with the reference's own host functions
 * (Sellmeier n/GV/GVD, findPhaseMatchingTemp, linspace, fftshift,
 * input_field_T) in its float types: argv-level inputs in, the solver
 * parameters, the grids T and w (n_t = SIZE points) and the CW pump out.
 * Harness inputs beyond the reference's argv: gdd_ps2, the intracavity GDD
 * in ps^2 (the reference takes a percentage of the crystal GDD,
 * cuOPO.cu:141-142), and n_z.  Host only; needs no GPU.
 */
void ref_setup_cw2(double lp_nm, double Lambda_um, double Nth_in, double R_percent, double delta_pi,
                   double gdd_ps2, double Lcr_mm, int n_z, ref_params *p, float *w_out, float *T_out,
                   float2 *pump_out, double *t_rt_out, double *ap0_out)
{
    const real_t lp = lp_nm * 1e-3;                              /* cuOPO.cu:92-101 */
    const real_t ls = 2 * lp;
    const real_t Lambda = Lambda_um;
    const real_t Temp = findPhaseMatchingTemp(lp, ls, Lambda, 10, 150);
    const real_t Lcr = Lcr_mm * 1e3;
    const real_t np = n(lp, Temp), vp = GV(lp, Temp), b2p = GVD(lp, Temp);  /* :103-114 */
    const real_t kp = 2 * PI * dQ / (np * lp);
    const real_t ns = n(ls, Temp), vs = GV(ls, Temp), b2s = GVD(ls, Temp);
    const real_t ks = 2 * PI * dQ / (ns * ls);
    const real_t dk = 2 * PI * (np / lp - 2 * ns / ls - 1 / Lambda);          /* :125 */
    const real_t Lcav = 100e3;                                               /* :129-146 */
    const real_t Rs = R_percent * 0.01;
    const real_t alphas = 0.5 * ((1 - Rs) + alpha_crs * Lcr);
    const real_t t_rt = (Lcav + Lcr * (ns - 1)) / C;
    const real_t dz = Lcr / (real_t)(uint)n_z;                               /* :149-151 */
    const real_t dF = 1 / t_rt;
    linspace(T_out, SIZE, -0.5 * t_rt, 0.5 * t_rt);                          /* :170-189 */
    real_t *Fq = (real_t *)malloc(sizeof(real_t) * SIZE);
    linspace(Fq, SIZE, -0.5 * SIZE * dF, +0.5 * SIZE * dF);
    fftshift(w_out, Fq, SIZE);
    for (uint i = 0; i < SIZE; i++) w_out[i] = 2 * PI * w_out[i];
    free(Fq);
    const real_t waist = 55, spot = PI * waist * waist;                      /* :202-229 */
    (void)spot;
    const real_t Ith = EPS0 * C * np * powf((ns * ls * alphas / dQ / Lcr / PI), 2) / 8;
    const real_t Inten = Nth_in * Ith;
    const real_t Ap0 = sqrt(2 * Inten / (np * EPS0 * C));
    input_field_T(pump_out, Ap0, SIZE);                                      /* :238-241 */

    memset(p, 0, sizeof(*p));
    p->n_eqs = 2;
    p->n_t = (int)SIZE;
    p->n_z = n_z;
    p->regime = 0;
    p->vp = vp; p->vs = vs; p->b2p = b2p; p->b2s = b2s;
    p->dk = dk; p->kp = kp; p->ks = ks; p->dz = dz;
    p->alpha_crp = alpha_crp; p->alpha_crs = alpha_crs; p->alpha_cri = alpha_cri;
    p->Rs = Rs; p->Ri = 0.98f; p->delta = (real_t)delta_pi; p->gdd = (real_t)gdd_ps2;
    *t_rt_out = t_rt;
    *ap0_out = Ap0;
}

/* ---- the reference round-trip loop on the GPU ---- */

/*
 * Runs round trips nn = rt_begin .. rt_begin+rt_count-1 of src/cuOPO.cu:474-610
 * with the reference kernels.  Host buffers in, host buffers out (same
 * contract as oracle_round_trips in ssfm_oracle.c).  If tol > 0 the loop
 * stops after the first rt (from the second on) whose relative change of
 * the signal power is below tol; *rt_done receives the number of rts run.
 * *elapsed_ms is the CUDA-event time of the loop alone.
 * Returns 0 or the first CUDA error code.
 */
int ref_round_trips(const ref_params *p, const float *w_h, const float *T_h,
                    float2 *Ap_h, float2 *As_h, float2 *Ai_h,
                    const float2 *pump_h, int n_rt, int rt_begin, int rt_count,
                    float2 *sv_p, float2 *sv_s, float2 *sv_i,
                    int save_first, int save_count,
                    double *ps_hist, double tol, int *rt_done, float *elapsed_ms)
{
    g_first_error = cudaSuccess;
    if (p->n_t != (int)SIZE) return -1;
    NZ = (uint)p->n_z;
    const bool three = (p->n_eqs == 3);
    const size_t nBytes = sizeof(complex_t) * SIZE;
    const size_t pump_len = (p->regime == 0) ? SIZE : (size_t)SIZE * (size_t)n_rt;
    const int n_save = save_count > 0 ? save_count : 1;

    const real_t vp = p->vp, vs = p->vs, vi = p->vi;
    const real_t b2p = p->b2p, b2s = p->b2s, b2i = p->b2i;
    const real_t b3p = p->b3p, b3s = p->b3s, b3i = p->b3i;
    const real_t dk = p->dk, kp = p->kp, ks = p->ks, ki = p->ki, dz = p->dz;
    const real_t Rs = p->Rs, Ri = p->Ri, delta = p->delta;
    const real_t GDD = p->gdd, TODscomp = p->tod_s, TODicomp = p->tod_i;
    const real_t mod_depth = p->mod_depth, fpm = p->fpm;

    dim3 block(BLKX);
    dim3 grid((SIZE + BLKX - 1) / BLKX);

    real_t *w_gpu, *T_gpu;
    complex_t *Ap_gpu, *Ap_in_gpu, *As_gpu, *Apw_gpu, *Asw_gpu;
    complex_t *Ap_total_gpu, *As_total_gpu;
    complex_t *k1p, *k2p, *k3p, *k4p, *k1s, *k2s, *k3s, *k4s, *auxp, *auxs;
    complex_t *Ai_gpu = 0, *Aiw_gpu = 0, *Ai_total_gpu = 0;
    complex_t *k1i = 0, *k2i = 0, *k3i = 0, *k4i = 0, *auxi = 0;
    double *ps_gpu;
    CHECK(cudaMalloc((void **)&w_gpu, sizeof(real_t) * SIZE));
    CHECK(cudaMalloc((void **)&T_gpu, sizeof(real_t) * SIZE));
    CHECK(cudaMalloc((void **)&Ap_gpu, nBytes));
    CHECK(cudaMalloc((void **)&As_gpu, nBytes));
    CHECK(cudaMalloc((void **)&Ap_in_gpu, sizeof(complex_t) * pump_len));
    CHECK(cudaMalloc((void **)&Apw_gpu, nBytes));
    CHECK(cudaMalloc((void **)&Asw_gpu, nBytes));
    CHECK(cudaMalloc((void **)&Ap_total_gpu, nBytes * n_save));
    CHECK(cudaMalloc((void **)&As_total_gpu, nBytes * n_save));
    CHECK(cudaMalloc((void **)&k1p, nBytes)); CHECK(cudaMalloc((void **)&k2p, nBytes));
    CHECK(cudaMalloc((void **)&k3p, nBytes)); CHECK(cudaMalloc((void **)&k4p, nBytes));
    CHECK(cudaMalloc((void **)&k1s, nBytes)); CHECK(cudaMalloc((void **)&k2s, nBytes));
    CHECK(cudaMalloc((void **)&k3s, nBytes)); CHECK(cudaMalloc((void **)&k4s, nBytes));
    CHECK(cudaMalloc((void **)&auxp, nBytes)); CHECK(cudaMalloc((void **)&auxs, nBytes));
    CHECK(cudaMalloc((void **)&ps_gpu, sizeof(double)));
    if (three) {
        CHECK(cudaMalloc((void **)&Ai_gpu, nBytes));
        CHECK(cudaMalloc((void **)&Aiw_gpu, nBytes));
        CHECK(cudaMalloc((void **)&Ai_total_gpu, nBytes * n_save));
        CHECK(cudaMalloc((void **)&k1i, nBytes)); CHECK(cudaMalloc((void **)&k2i, nBytes));
        CHECK(cudaMalloc((void **)&k3i, nBytes)); CHECK(cudaMalloc((void **)&k4i, nBytes));
        CHECK(cudaMalloc((void **)&auxi, nBytes));
    }
    if (g_first_error != cudaSuccess) return (int)g_first_error;

    CHECK(cudaMemcpy(w_gpu, w_h, sizeof(real_t) * SIZE, cudaMemcpyHostToDevice));
    if (T_h) CHECK(cudaMemcpy(T_gpu, T_h, sizeof(real_t) * SIZE, cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(Ap_gpu, Ap_h, nBytes, cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(As_gpu, As_h, nBytes, cudaMemcpyHostToDevice));
    CHECK(cudaMemcpy(Ap_in_gpu, pump_h, sizeof(complex_t) * pump_len, cudaMemcpyHostToDevice));
    if (three) CHECK(cudaMemcpy(Ai_gpu, Ai_h, nBytes, cudaMemcpyHostToDevice));

    cufftHandle plan1D;
    cufftPlan1d(&plan1D, SIZE, CUFFT_C2C, 1);

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    double prev = -1.0;
    int done = 0;
    for (int nn = rt_begin; nn < rt_begin + rt_count; nn++) {
        if (p->regime == 0) {
            CHECK(cudaMemcpy(Ap_gpu, Ap_in_gpu, nBytes, cudaMemcpyDeviceToDevice));
        } else {
            ReadPump<<<grid, block>>>(Ap_gpu, Ap_in_gpu, n_rt, nn);
            CHECK(cudaDeviceSynchronize());
        }
        if (three)
            EvolutionInCrystal(w_gpu, Ap_gpu, As_gpu, Ai_gpu, Apw_gpu, Asw_gpu, Aiw_gpu,
                               k1p, k1s, k1i, k2p, k2s, k2i, k3p, k3s, k3i, k4p, k4s, k4i,
                               auxp, auxs, auxi, vp, vs, vi, b2p, b2s, b2i, b3p, b3s, b3i,
                               dk, kp, ks, ki, dz);
        else
            EvolutionInCrystal(w_gpu, Ap_gpu, As_gpu, Apw_gpu, Asw_gpu, k1p, k1s, k2p, k2s,
                               k3p, k3s, k4p, k4s, auxp, auxs, vp, vs, b2p, b2s, b3p, b3s,
                               dk, kp, ks, dz);
        if (p->use_eom) {
            PhaseModulatorIntraCavity<<<grid, block>>>(As_gpu, auxs, mod_depth, fpm, T_gpu);
            CHECK(cudaDeviceSynchronize());
            if (three && p->eom_idler) {
                PhaseModulatorIntraCavity<<<grid, block>>>(Ai_gpu, auxi, mod_depth, fpm, T_gpu);
                CHECK(cudaDeviceSynchronize());
            }
        }
        if (GDD != 0) {
            cufftExecC2C(plan1D, As_gpu, Asw_gpu, CUFFT_INVERSE);
            CHECK(cudaDeviceSynchronize());
            CUFFTscale<<<grid, block>>>(Asw_gpu, SIZE);
            CHECK(cudaDeviceSynchronize());
            if (TODscomp != 0 and b3s != 0) {
                AddGDDTOD<<<grid, block>>>(Asw_gpu, auxs, w_gpu, GDD, TODscomp);
            } else {
                AddGDD<<<grid, block>>>(Asw_gpu, auxs, w_gpu, GDD);
            }
            CHECK(cudaDeviceSynchronize());
            cufftExecC2C(plan1D, Asw_gpu, As_gpu, CUFFT_FORWARD);
            CHECK(cudaDeviceSynchronize());
            if (three) {
                cufftExecC2C(plan1D, Ai_gpu, Aiw_gpu, CUFFT_INVERSE);
                CHECK(cudaDeviceSynchronize());
                CUFFTscale<<<grid, block>>>(Aiw_gpu, SIZE);
                CHECK(cudaDeviceSynchronize());
                if (TODicomp != 0 and b3i != 0) {
                    AddGDDTOD<<<grid, block>>>(Aiw_gpu, auxi, w_gpu, GDD, TODicomp);
                } else {
                    AddGDD<<<grid, block>>>(Aiw_gpu, auxi, w_gpu, GDD);
                }
                CHECK(cudaDeviceSynchronize());
                cufftExecC2C(plan1D, Aiw_gpu, Ai_gpu, CUFFT_FORWARD);
                CHECK(cudaDeviceSynchronize());
            }
        }
        AddPhase<<<grid, block>>>(As_gpu, auxs, Rs, delta);
        CHECK(cudaDeviceSynchronize());
        if (three) {
            AddPhase<<<grid, block>>>(Ai_gpu, auxi, Ri, delta);
            CHECK(cudaDeviceSynchronize());
        }
        if (nn >= save_first && nn < save_first + save_count) {
            const uint slot = (uint)(nn - save_first);
            SaveRoundTrip<<<grid, block>>>(As_total_gpu, As_gpu, slot, (uint)save_count);
            CHECK(cudaDeviceSynchronize());
            SaveRoundTrip<<<grid, block>>>(Ap_total_gpu, Ap_gpu, slot, (uint)save_count);
            CHECK(cudaDeviceSynchronize());
            if (three) {
                SaveRoundTrip<<<grid, block>>>(Ai_total_gpu, Ai_gpu, slot, (uint)save_count);
                CHECK(cudaDeviceSynchronize());
            }
        }
        done++;
        if (ps_hist || tol > 0) {
            double ps = 0.0;
            harness_power<<<1, 256>>>(As_gpu, ps_gpu);
            CHECK(cudaMemcpy(&ps, ps_gpu, sizeof(double), cudaMemcpyDeviceToHost));
            if (ps_hist) ps_hist[nn - rt_begin] = ps;
            if (tol > 0 && prev > 0.0 && ps > 0.0 && std::fabs(ps - prev) < tol * ps) break;
            prev = ps;
        }
        if (g_first_error != cudaSuccess) break;
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (elapsed_ms) *elapsed_ms = ms;
    if (rt_done) *rt_done = done;

    CHECK(cudaMemcpy(Ap_h, Ap_gpu, nBytes, cudaMemcpyDeviceToHost));
    CHECK(cudaMemcpy(As_h, As_gpu, nBytes, cudaMemcpyDeviceToHost));
    if (three) CHECK(cudaMemcpy(Ai_h, Ai_gpu, nBytes, cudaMemcpyDeviceToHost));
    if (save_count > 0) {
        if (sv_s) CHECK(cudaMemcpy(sv_s, As_total_gpu, nBytes * save_count, cudaMemcpyDeviceToHost));
        if (sv_p) CHECK(cudaMemcpy(sv_p, Ap_total_gpu, nBytes * save_count, cudaMemcpyDeviceToHost));
        if (three && sv_i) CHECK(cudaMemcpy(sv_i, Ai_total_gpu, nBytes * save_count, cudaMemcpyDeviceToHost));
    }

    cufftDestroy(plan1D);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(w_gpu); cudaFree(T_gpu); cudaFree(Ap_gpu); cudaFree(As_gpu);
    cudaFree(Ap_in_gpu); cudaFree(Apw_gpu); cudaFree(Asw_gpu);
    cudaFree(Ap_total_gpu); cudaFree(As_total_gpu);
    cudaFree(k1p); cudaFree(k2p); cudaFree(k3p); cudaFree(k4p);
    cudaFree(k1s); cudaFree(k2s); cudaFree(k3s); cudaFree(k4s);
    cudaFree(auxp); cudaFree(auxs); cudaFree(ps_gpu);
    if (three) {
        cudaFree(Ai_gpu); cudaFree(Aiw_gpu); cudaFree(Ai_total_gpu);
        cudaFree(k1i); cudaFree(k2i); cudaFree(k3i); cudaFree(k4i); cudaFree(auxi);
    }
    return (int)g_first_error;
}

}  /* extern "C" */
