/*
 * ssfm.cuh -- the fused SSFM round-trip kernel (one CTA per OPO instance).
 *
 * One launch runs whole crystal passes and cavity round trips of the
 * reference loop (src/cuOPO.cu:474-610) with every field resident in
 * shared memory:
 *
 *   per round trip:  pump injection (cuOPO.cu:478-486, functions.cuh:191-213)
 *     per slice s:   RK4 half step at z_s (cwes2.cuh:147-166)
 *                    for each field: T->W transform (CUFFT_INVERSE), x D(w)/N
 *                    (LinearOperator + CUFFTscale, cwes2.cuh:103-121,
 *                    functions.cuh:126-135), W->T transform (CUFFT_FORWARD)
 *                    RK4 half step at z_s again (cwes2.cuh:188-207, quirk Q2)
 *     EOM (functions.cuh:242-253), GDD/TOD (cuOPO.cu:521-553), AddPhase
 *     (functions.cuh:139-152), SaveRoundTrip (functions.cuh:217-238), and
 *     the signal power for the convergence rule.
 *
 * The second half step of slice s and the first of slice s+1 are applied
 * back to back in one element-wise phase.  Element-wise phases touch only
 * the points t + e*T of each field that thread t holds before and after
 * every transform, so they need no barrier.
 *
 * Quirks kept: RK4 stages use aux = A + s k without the step (Q1); both
 * half steps of a slice use the same z (Q2); in the 3-equation model all
 * stages read the unperturbed fields (Q3), so the half step reduces to
 * A += c(z) * P(A) with one complex coefficient per field and slice.
 */
#pragma once
#include "fft.cuh"

namespace cuopo {

/* Per-plan device tables (type-erased; element type is cpx<R>). */
struct Tables {
    const void *disp;   /* [F][N]: slice dispersion x attenuation / N */
    const void *rk;     /* [n_z][6] (2 eqs) or [n_z][3] (3 eqs) RK4 coefficients */
    const void *eom;    /* [N]: exp(i m sin(2 pi fpm T)) or NULL */
    const float *w;     /* [N]: angular frequency grid (reference float values) */
    double h6;          /* (dz/2)/6 */
    double inv_n;       /* 1/N */
};

/* One OPO instance (one set of fields and cavity settings). */
struct Instance {
    void *Ap, *As, *Ai;         /* device fields, n_t values each */
    const void *pump;           /* CW: n_t values or NULL (constant ap0); NS: window */
    double ap0;                 /* constant CW pump amplitude when pump == NULL */
    int n_rt_total;             /* NRT of the NS pump window (ReadPump) */
    int rt_begin, rt_count;
    void *sv_p, *sv_s, *sv_i;   /* SaveRoundTrip buffers (may be NULL) */
    int save_first, save_count;
    double *ps_hist;            /* per-rt signal power (may be NULL) */
    double tol;                 /* convergence tolerance (<= 0: off) */
    int *rt_done;               /* number of round trips run (may be NULL) */
    double phase_s[2];          /* sqrt(Rs) exp(i pi delta) */
    double phase_i[2];          /* sqrt(Ri) exp(i pi delta) */
    double gdd;                 /* intracavity GDD [ps^2]; 0 = off */
    double tod_s, tod_i;        /* TOD compensation [ps^3] */
    int use_tod_s, use_tod_i;
    int patience;               /* consecutive rts below tol to stop (>= 1) */
    double *ps_out;             /* final signal power (may be NULL) */
    int *flag_out;              /* 1 converged, 0 max rts reached, 5 non-finite (may be NULL) */
};

struct LaunchArgs {
    Tables tab;
    Instance single;            /* used when inst == NULL */
    const Instance *inst;       /* batch of instances, or NULL */
    int n_inst;
    int *queue;                 /* work-queue counter for persistent batches */
    int n_z;
    int regime;                 /* CUOPO_CW / CUOPO_NS */
    int pass_only;              /* 1: one crystal pass, no cavity map */
    int use_eom, eom_idler;
    int *status;                /* first error code (atomicCAS from 0) */
};

enum { ST_OK = 0, ST_NONFINITE = 5 };

template <typename C>
__device__ __forceinline__ C ldc(const void *p, long i)
{
    return __ldg(reinterpret_cast<const C *>(p) + i);
}

/* RK4 half step, 2 equations: cwes2.cuh:30-87 with stage coefficients
 * co = {i kp e^{+i dk z_j}, i ks e^{-i dk z_j}}, z_j = z, z+dz/4, z+dz/2. */
template <typename C, typename R>
__device__ __forceinline__ void rk4_half2(C &Ap, C &As, const C *__restrict__ co, R h6)
{
    const C k1p = cmul(co[0], cmul(As, As));
    const C k1s = cmul(co[1], cmulc(Ap, As));
    C ap = caxpy(Ap, (R)0.5, k1p), as = caxpy(As, (R)0.5, k1s);
    const C k2p = cmul(co[2], cmul(as, as));
    const C k2s = cmul(co[3], cmulc(ap, as));
    ap = caxpy(Ap, (R)0.5, k2p);
    as = caxpy(As, (R)0.5, k2s);
    const C k3p = cmul(co[2], cmul(as, as));
    const C k3s = cmul(co[3], cmulc(ap, as));
    ap = cadd(Ap, k3p);
    as = cadd(As, k3s);
    const C k4p = cmul(co[4], cmul(as, as));
    const C k4s = cmul(co[5], cmulc(ap, as));
    const C sp = cadd(cadd(k1p, k4p), cscale(cadd(k2p, k3p), (R)2));
    const C ss = cadd(cadd(k1s, k4s), cscale(cadd(k2s, k3s), (R)2));
    Ap = caxpy(Ap, h6, sp);
    As = caxpy(As, h6, ss);
}

/* RK4 half step, 3 equations: cwes3.cuh:30-90 with Q3, folded to
 * A_f += co_f * P_f where P = (As Ai, Ap conj(Ai), Ap conj(As)). */
template <typename C>
__device__ __forceinline__ void rk4_half3(C &Ap, C &As, C &Ai, const C *__restrict__ co)
{
    const C Pp = cmul(As, Ai);
    const C Ps = cmulc(Ap, Ai);
    const C Pi = cmulc(Ap, As);
    Ap = cadd(Ap, cmul(co[0], Pp));
    As = cadd(As, cmul(co[1], Ps));
    Ai = cadd(Ai, cmul(co[2], Pi));
}

template <typename R, int F, int M, bool INPLACE>
struct Ssfm {
    using C = cpx<R>;
    using SP = StagePlan<M>;
    static constexpr int T = SP::T;
    static constexpr int P = SP::P;
    static constexpr int NCO = (F == 2) ? 6 : 3;

    /* Shared memory: home[F][M] (+ scratch[M]) complex values, then the
     * twiddle table of the middle FFT stages. */
    static constexpr size_t field_elems() { return (size_t)M * (F + (INPLACE ? 0 : 1)); }
    static constexpr size_t smem_bytes() { return sizeof(C) * (field_elems() + TwTable<M>::size()); }

    /* T->W, multiply by the table row (or the on-the-fly GDD factor),
     * W->T, on the field at home. */
    template <int MODE>  /* 0: table row mul, 1: GDD with TOD flag */
    static __device__ __forceinline__ void spectral(C *home, C *scratch, const C *__restrict__ row,
                                                    const float *__restrict__ w, double gdd,
                                                    double tod, int use_tod, double inv_n,
                                                    const StageTwiddles<M, C> &tw, int t)
    {
        C reg[16];
        load_own<M>(home, reg, t);
        C *bufA = INPLACE ? home : scratch;
        C *bufB = home;
        local_transform<+1, M, 0, INPLACE>(reg, bufA, bufB, tw, t);
        if constexpr (MODE == 0) {
#pragma unroll
            for (int e = 0; e < 16; e++) reg[e] = cmul(reg[e], __ldg(row + t + e * T));
        } else {
#pragma unroll 4
            for (int e = 0; e < 16; e++) {
                /* functions.cuh:156-186 with CUFFTscale folded in, formed in FP64 */
                const double wk = (double)__ldg(w + t + e * T);
                const double ph = use_tod ? 0.5 * wk * (wk * gdd + wk * wk * tod / 3.0)
                                          : 0.5 * wk * wk * gdd;
                double s, c;
                sincos(ph, &s, &c);
                reg[e] = cmul(reg[e], mk<C>((R)(c * inv_n), (R)(s * inv_n)));
            }
        }
        local_transform<-1, M, P - 1, INPLACE>(reg, bufA, bufB, tw, t);
        store_own<M>(home, reg, t);
    }

    static __device__ __forceinline__ double block_sum(double v, double *red, int t)
    {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((t & 31) == 0) red[t >> 5] = v;
        __syncthreads();
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < T / 32; q++) s += red[q];
        __syncthreads();
        return s;
    }

    static __device__ void run(const LaunchArgs &a)
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        C *home = reinterpret_cast<C *>(smem_raw);
        C *scratch = INPLACE ? home : home + (size_t)F * M;
        __shared__ double red[32];
        __shared__ int next_inst;
        const int t = threadIdx.x;

        C *twtab = home + field_elems();
        fill_twiddle_table<M>(twtab, t);
        StageTwiddles<M, C> tw;
        tw.init(t, twtab);
        __syncthreads();
        const R h6 = (R)a.tab.h6;
        const C *__restrict__ rk = reinterpret_cast<const C *>(a.tab.rk);
        const C *__restrict__ disp = reinterpret_cast<const C *>(a.tab.disp);
        const C *__restrict__ eomt = reinterpret_cast<const C *>(a.tab.eom);

        int idx = a.inst ? -1 : (int)blockIdx.x;
        for (;;) {
            if (a.inst) {
                if (a.queue) {
                    if (t == 0) next_inst = atomicAdd(a.queue, 1);
                    __syncthreads();
                    idx = next_inst;
                    __syncthreads();
                } else {
                    idx = (idx < 0) ? (int)blockIdx.x : idx + (int)gridDim.x;
                }
                if (idx >= a.n_inst) break;
            } else if (idx != 0) {
                break;
            }
            const Instance &I = a.inst ? a.inst[idx] : a.single;

            C *gf[3] = {reinterpret_cast<C *>(I.Ap), reinterpret_cast<C *>(I.As),
                        reinterpret_cast<C *>(I.Ai)};
#pragma unroll
            for (int f = 0; f < F; f++)
#pragma unroll
                for (int e = 0; e < 16; e++) home[f * M + swz<C>(t + e * T)] = gf[f][t + e * T];

            double prev_ps = -1.0, ps = 0.0;
            int rts = 0, calm = 0, flag = 0;
            bool stop = false;
            for (int rt = I.rt_begin; rt < I.rt_begin + I.rt_count && !stop; rt++) {
                /* pump injection + first half step of slice 0 */
                {
                    long poff = 0;
                    if (a.regime == 1) {
                        /* ReadPump offsets, functions.cuh:196-210 (Q6) */
                        const int nrt = I.n_rt_total;
                        poff = (rt == 0) ? 0 : ((rt > 0 && rt < nrt - 1) ? (long)rt * M
                                                                         : (long)M * nrt - 1 - M);
                    }
#pragma unroll 2
                    for (int e = 0; e < 16; e++) {
                        const int m = t + e * T;
                        const int sm = swz<C>(m);
                        C A[3];
#pragma unroll
                        for (int f = 0; f < F; f++) A[f] = home[f * M + sm];
                        if (!a.pass_only) {
                            if (I.pump) A[0] = ldc<C>(I.pump, poff + m);
                            else A[0] = mk<C>((R)I.ap0, (R)0);
                        }
                        if constexpr (F == 2) rk4_half2(A[0], A[1], rk, h6);
                        else rk4_half3(A[0], A[1], A[2], rk);
#pragma unroll
                        for (int f = 0; f < F; f++) home[f * M + sm] = A[f];
                    }
                }
                for (int s = 0; s < a.n_z; s++) {
#pragma unroll 1
                    for (int f = 0; f < F; f++)
                        spectral<0>(home + f * M, scratch, disp + (size_t)f * M, nullptr, 0.0, 0.0,
                                    0, 0.0, tw, t);
                    const C *co0 = rk + (size_t)s * NCO;
                    const C *co1 = rk + (size_t)(s + 1) * NCO;
                    const bool next = (s + 1 < a.n_z);
                    const bool eom = (!next && !a.pass_only && a.use_eom);
#pragma unroll 2
                    for (int e = 0; e < 16; e++) {
                        const int m = t + e * T;
                        const int sm = swz<C>(m);
                        C A[3];
#pragma unroll
                        for (int f = 0; f < F; f++) A[f] = home[f * M + sm];
                        if constexpr (F == 2) {
                            rk4_half2(A[0], A[1], co0, h6);
                            if (next) rk4_half2(A[0], A[1], co1, h6);
                        } else {
                            rk4_half3(A[0], A[1], A[2], co0);
                            if (next) rk4_half3(A[0], A[1], A[2], co1);
                        }
                        if (eom) {
                            const C ef = __ldg(eomt + m);
                            A[1] = cmul(A[1], ef);
                            if (F == 3 && a.eom_idler) A[F - 1] = cmul(A[F - 1], ef);
                        }
#pragma unroll
                        for (int f = 0; f < F; f++) home[f * M + sm] = A[f];
                    }
                }
                rts++;
                if (a.pass_only) break;

                /* GDD / TOD compensation of the resonant fields (cuOPO.cu:521-553) */
                if (I.gdd != 0.0) {
                    spectral<1>(home + 1 * M, scratch, nullptr, a.tab.w, I.gdd, I.tod_s, I.use_tod_s,
                                a.tab.inv_n, tw, t);
                    if constexpr (F == 3)
                        spectral<1>(home + 2 * M, scratch, nullptr, a.tab.w, I.gdd, I.tod_i,
                                    I.use_tod_i, a.tab.inv_n, tw, t);
                }

                /* AddPhase, SaveRoundTrip, signal power */
                const C ph_s = mk<C>((R)I.phase_s[0], (R)I.phase_s[1]);
                const C ph_i = mk<C>((R)I.phase_i[0], (R)I.phase_i[1]);
                const bool save = (rt >= I.save_first && rt < I.save_first + I.save_count);
                const size_t slot = save ? (size_t)(rt - I.save_first) * M : 0;
                C *sv[3] = {reinterpret_cast<C *>(I.sv_p), reinterpret_cast<C *>(I.sv_s),
                            reinterpret_cast<C *>(I.sv_i)};
                double acc = 0.0;
#pragma unroll 2
                for (int e = 0; e < 16; e++) {
                    const int m = t + e * T;
                    const int sm = swz<C>(m);
                    C A[3];
#pragma unroll
                    for (int f = 0; f < F; f++) A[f] = home[f * M + sm];
                    A[1] = cmul(A[1], ph_s);
                    if constexpr (F == 3) A[2] = cmul(A[2], ph_i);
                    home[1 * M + sm] = A[1];
                    if constexpr (F == 3) home[2 * M + sm] = A[2];
                    if (save) {
#pragma unroll
                        for (int f = 0; f < F; f++)
                            if (sv[f]) sv[f][slot + m] = A[f];
                    }
                    acc += cabs2d(A[1]);
                }
                ps = block_sum(acc, red, t) * a.tab.inv_n;
                if (t == 0 && I.ps_hist) I.ps_hist[rt - I.rt_begin] = ps;
                if (!(ps == ps) || ps > 1.0e300) {
                    if (t == 0 && a.status) atomicCAS(a.status, 0, (int)ST_NONFINITE);
                    flag = ST_NONFINITE;
                    stop = true;
                }
                /* convergence: relative change of the signal power per rt below
                 * tol for `patience` consecutive rts (from the second rt on) */
                if (I.tol > 0.0 && prev_ps > 0.0 && ps > 0.0 && fabs(ps - prev_ps) < I.tol * ps) {
                    if (++calm >= (I.patience > 0 ? I.patience : 1) && flag == 0) {
                        flag = 1;
                        stop = true;
                    }
                } else {
                    calm = 0;
                }
                prev_ps = ps;
            }
#pragma unroll
            for (int f = 0; f < F; f++)
#pragma unroll
                for (int e = 0; e < 16; e++) gf[f][t + e * T] = home[f * M + swz<C>(t + e * T)];
            if (t == 0) {
                if (I.rt_done) *I.rt_done = rts;
                if (I.ps_out) *I.ps_out = ps;
                if (I.flag_out) *I.flag_out = flag;
            }
            __syncthreads();
            if (!a.inst) break;
        }
    }
};

template <typename R, int F, int M, bool INPLACE, int MINB>
__global__ void __launch_bounds__(M / 16, MINB) ssfm_kernel(const LaunchArgs a)
{
    Ssfm<R, F, M, INPLACE>::run(a);
}

}  // namespace cuopo
