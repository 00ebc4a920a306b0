/*
 * ssfm.cuh -- the fused SSFM round-trip kernel.
 *
 * One launch runs whole crystal passes and cavity round trips of the
 * reference loop (src/cuOPO.cu:474-610) with every field resident in shared
 * memory, for one instance per CTA (CL = 1) or per thread-block cluster of
 * CL CTAs (grids up to CL x 8192 points):
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
 * Cluster decomposition (N = CL * M): CTA c holds time block n = n1 + M c.
 * The T->W transform is a radix-CL "cross" stage over the CTAs,
 *   y_k2[n1] = W_N^{n1 k2} sum_n2 x[n1 + M n2] W_CL^{n2 k2}   (stored on CTA k2),
 * followed by a local M-point transform on CTA k2 giving X[k2 + CL k1]; the
 * W->T transform runs the same two steps backwards.  Between the local W->T
 * transform of slice s and the local T->W transform of slice s+1 the
 * inverse cross stage, both RK4 half steps and the forward cross stage are
 * one element-wise pass over distributed shared memory, so each slice costs
 * one exchange between the CTAs and two cluster barriers.  The fields live
 * in the y domain between slices; the time domain exists only inside that
 * pass (and at round-trip ends).  With CL = 1 the cross stages are
 * identities and no barrier is needed around the element-wise passes.
 *
 * Quirks kept: RK4 stages use aux = A + s k without the step (Q1); both
 * half steps of a slice use the same z (Q2); in the 3-equation model all
 * stages read the unperturbed fields (Q3), so the half step reduces to
 * A += c(z) * P(A) with one complex coefficient per field and slice.
 */
#pragma once
#include <cooperative_groups.h>

#include "fft.cuh"

namespace cuopo {

/* Per-plan device tables (type-erased; element type is cpx<R>).  Tables
 * indexed by frequency are stored per CTA: entry [k2][k1] is frequency
 * index k2 + CL k1. */
struct Tables {
    const void *disp;   /* [F][CL][M]: slice dispersion x attenuation / N */
    const void *rk;     /* [n_z + 1][6] (2 eqs) or [n_z + 1][3] (3 eqs) RK4 coefficients */
    const void *eom;    /* [N]: exp(i m sin(2 pi fpm T)) or NULL */
    const float *w;     /* [CL][M]: angular frequency grid (reference float values) */
    const void *twN;    /* [N]: W_N^q (cross-stage twiddles; CL > 1) */
    const double2 *frame_u; /* [NFRAME]: random frame angles (u_s, u_i) in turns, |u| < 1/8 */
    const void *frame_c;    /* [NFRAME][3]: rotation (tan, sin) for pump, signal, idler */
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
    /* resumable state of a batch instance (all NULL for single launches):
     * round trips run so far, last signal power, calm-rt counter and flag
     * (0 running, 1 converged, 2 round-trip limit reached, 5 non-finite) */
    int *st_rt;
    double *st_ps;
    int *st_calm;
    int *st_flag;
    /* the instance's own physics tables (batches whose instances differ in
     * crystal, wavelengths, length or modulator); NULL disp: the launch's */
    const void *disp, *rk, *eom;
    const float *w;
    double h6;
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
    /* batch launches: continue each running instance by up to `chunk` round
     * trips, stopping at max_rt; convergence tolerance and patience */
    int chunk, max_rt, patience;
    double tol;
};

enum { ST_OK = 0, ST_CONVERGED = 1, ST_LIMIT = 2, ST_NONFINITE = 5 };

/* Random frame rotations.  The coupled-wave equations are invariant under
 * (Ap, As, Ai) -> (Ap e^{i(a+b)}, As e^{ia}, Ai e^{ib}) (and Ap e^{2ia} in the
 * degenerate 2-equation model), and the linear steps commute with it.  Each
 * slice the kernel moves the fields to a new frame drawn from a fixed table
 * and returns them to the laboratory frame before the cavity map; the
 * rounding errors of the float transforms then have random phase relative
 * to the field, so they do not add up coherently over the ~10^5 slices of a
 * run.  Entry of slice s of round trip rt: frame_index(rt, s). */
enum { NFRAME = 1024 };

__host__ __device__ __forceinline__ int frame_index(int rt, int s)
{
    unsigned long long z = ((unsigned long long)(unsigned)rt << 32) ^ (unsigned)s ^ 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (int)(z & (NFRAME - 1));
}

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


namespace cg = cooperative_groups;

/* Where the fields live during a launch (HM):
 *   0  shared memory: home[F][M] and a scratch[M] for the local transforms
 *   1  shared memory, in place: home[F][M], the local transforms exchange
 *      through the field's own home
 *   2  global memory: the caller's field buffers, L2-resident between
 *      passes, with one shared scratch[M] for the local transforms; for grids
 *      whose fields exceed a cluster's shared memory (3 FP64 fields of 2^17
 *      points are 6 MiB, a 16-CTA cluster has 3.6 MB).  Every access to
 *      the fields goes to L2 (ld/st .cg), ordered by the cluster barriers. */
template <typename R, int F, int M, int CL, int HM>
struct Ssfm {
    static constexpr bool GH = (HM == 2);
    static constexpr bool INPLACE = (HM != 0); /* one exchange buffer per local transform */
    using C = cpx<R>;
    using SP = StagePlan<M>;
    static constexpr int T = SP::T;
    static constexpr int P = SP::P;
    static constexpr int N = M * CL;
    static constexpr int J = 16 / CL;  /* n1 values per thread in a cross stage */
    static constexpr int NCO = (F == 2) ? 6 : 3;
    static constexpr unsigned ALL = (1u << F) - 1u;
    static_assert(CL == 1 || CL == 2 || CL == 4 || CL == 8 || CL == 16, "cluster size must be 1..16, power of 2");

    /* Shared memory: home[F][M] (+ scratch[M]) complex values, or scratch[M]
     * alone (HM = 2), then the twiddle table of the middle FFT stages. */
    static constexpr size_t field_elems() { return GH ? (size_t)M : (size_t)M * (F + (INPLACE ? 0 : 1)); }
    static constexpr size_t smem_bytes() { return sizeof(C) * (field_elems() + TwTable<M>::size()); }

    /* Element-wise work of one cross stage (uniform over the cluster). */
    struct Ops {
        int inject;         /* pump injection */
        long poff;          /* NS pump window offset of this round trip */
        const C *rk0, *rk1; /* RK4 half steps to apply (NULL: none) */
        int eom;            /* intracavity phase modulator */
        int rotate;         /* frame rotation: quarter turns rq[f], then the shear rotation rf[f] */
        C rf[3];
        int rq[3];
        int addphase;       /* AddPhase on the resonant fields */
        double2 ph_s, ph_i;
        int save;           /* SaveRoundTrip into slot */
        size_t slot;
        int power;          /* accumulate |As|^2 */
    };

    /* Move to the frame of table entry q (rotation by 2 pi u per field, built
     * from shears); th accumulates each field's frame angle in turns. */
    static __device__ __forceinline__ void frame_step(Ops &op, const Tables &tab, int q, double (&th)[3])
    {
        const C *fc = reinterpret_cast<const C *>(tab.frame_c) + 3 * q;
        const double2 u = tab.frame_u[q];
        op.rotate = 1;
#pragma unroll
        for (int f = 0; f < 3; f++) {
            op.rf[f] = fc[f];
            op.rq[f] = 0;
        }
        th[1] += u.x;
        th[2] += u.y;
        th[0] += (F == 2) ? 2.0 * u.x : u.x + u.y;
    }

    /* Back to the laboratory frame: rotation by -th = quarter turns plus a
     * residual of at most 1/8 turn, formed in FP64. */
    static __device__ __forceinline__ void frame_back(Ops &op, const double (&th)[3])
    {
        op.rotate = 1;
#pragma unroll
        for (int f = 0; f < 3; f++) {
            const double back = -th[f];
            const double qt = rint(4.0 * back);
            const double res = back - 0.25 * qt; /* turns, |res| <= 1/8 */
            double sh, ch, sn, cs;
            sincospi(res, &sh, &ch);
            sincospi(2.0 * res, &sn, &cs);
            op.rq[f] = ((int)fmod(qt, 4.0) + 4) & 3;
            op.rf[f] = mk<C>((R)(sh / ch), (R)sn);
        }
    }

    /* Round-trip limit of a batch instance: the launch's, and for a
     * nanosecond instance also the end of its pump window. */
    static __device__ __forceinline__ int rt_limit(const LaunchArgs &a, const Instance &I)
    {
        return (a.regime == 1 && I.n_rt_total > 0) ? min(a.max_rt, I.n_rt_total) : a.max_rt;
    }

    /* Cluster barrier (release / acquire).  Every call site is reached by
     * all threads of the cluster with uniform control flow, so the
     * warp-aligned form applies; it runs batches of 2^15-point instances
     * 1.4 % faster than the generic form (4.5 % for one instance alone). */
    static __device__ __forceinline__ void csync()
    {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }

    static __device__ __forceinline__ void xsync()
    {
        if constexpr (GH) {
            /* the cross passes write other CTAs' positions of global memory */
            __threadfence();
            if constexpr (CL > 1) csync();
            else __syncthreads();
        } else if constexpr (CL > 1) {
            csync();
        }
    }

    static __device__ __forceinline__ void bar()
    {
        if constexpr (CL > 1) csync();
        else __syncthreads();
    }

    template <typename X>
    static __device__ __forceinline__ X *peer(X *p, int rank)
    {
        if constexpr (CL == 1) return p;
        else return cg::this_cluster().map_shared_rank(p, rank);
    }

    static __device__ __forceinline__ C mul_fp64(C a, double2 f)
    {
        const double re = (double)a.x * f.x - (double)a.y * f.y;
        const double im = (double)a.x * f.y + (double)a.y * f.x;
        return mk<C>((R)re, (R)im);
    }

    /* co0 / co1: the coefficients of op.rk0 / op.rk1, loaded once per cross
     * pass (through a pointer they would be reloaded for every point: the
     * shared-memory stores between points may alias it for the compiler) */
    static __device__ __forceinline__ void pointwise(C (&A)[3], int n, const Ops &op, const C (&co0)[NCO],
                                                     const C (&co1)[NCO], const Instance &I, const Tables &tab, R h6,
                                                     int eom_idler, double &acc)
    {
        if (op.inject) A[0] = I.pump ? ldc<C>(I.pump, op.poff + n) : mk<C>((R)I.ap0, (R)0);
        if (op.rk0) {
            if constexpr (F == 2) rk4_half2(A[0], A[1], co0, h6);
            else rk4_half3(A[0], A[1], A[2], co0);
        }
        if (op.rk1) {
            if constexpr (F == 2) rk4_half2(A[0], A[1], co1, h6);
            else rk4_half3(A[0], A[1], A[2], co1);
        }
        if (op.eom) {
            const C ef = ldc<C>(tab.eom, n);
            A[1] = cmul(A[1], ef);
            if (F == 3 && eom_idler) A[F - 1] = cmul(A[F - 1], ef);
        }
        if (op.rotate) {
#pragma unroll
            for (int f = 0; f < F; f++) A[f] = shear_rot(iq_rt(A[f], op.rq[f]), op.rf[f].x, op.rf[f].y);
        }
        if (op.addphase) {
            /* in FP64 so that sqrt(R) exp(i pi delta) carries no float rounding
             * bias into the round-trip gain */
            A[1] = mul_fp64(A[1], op.ph_s);
            if constexpr (F == 3) A[2] = mul_fp64(A[2], op.ph_i);
        }
        if (op.save) {
            C *sv[3] = {reinterpret_cast<C *>(I.sv_p), reinterpret_cast<C *>(I.sv_s),
                        reinterpret_cast<C *>(I.sv_i)};
#pragma unroll
            for (int f = 0; f < F; f++)
                if (sv[f]) sv[f][op.slot + n] = A[f];
        }
        if (op.power) acc += cabs2d(A[1]);
    }

    /* The radix-CL stage of one field at the owned position n1 (S = -1: the
     * inverse cross stage, y -> time; S = +1: the forward one), on global
     * memory. */
    template <int S>
    static __device__ __forceinline__ void cross_field(C *g, const C *__restrict__ twN, int n1)
    {
        C v[CL];
#pragma unroll
        for (int c = 0; c < CL; c++) v[c] = __ldcg(g + (size_t)c * M + n1);
        if constexpr (S < 0) {
#pragma unroll
            for (int c = 1; c < CL; c++) {
                const long q = (long)n1 * c;
                const C w = __ldg(twN + q);
                v[c] = shear_rot(iq_rt(v[c], (-(int)(((4 * q + N / 2) / N) & 3)) & 3), -w.x, -w.y);
            }
            dft<-1, CL>(v);
        } else {
            dft<+1, CL>(v);
#pragma unroll
            for (int c = 1; c < CL; c++) {
                const long q = (long)n1 * c;
                const C w = __ldg(twN + q);
                v[c] = shear_rot(iq_rt(v[c], (int)(((4 * q + N / 2) / N) & 3)), w.x, w.y);
            }
        }
#pragma unroll
        for (int c = 0; c < CL; c++) __stcg(g + (size_t)c * M + n1, v[c]);
    }

    /* The element-wise pass of `cross` with the fields in global memory
     * (HM = 2): the same arithmetic in the same order, but one field's
     * radix-CL stage at a time, the intermediate values going through L2 (CL
     * values of 3 FP64 fields would not fit in registers).  Thread t still
     * reads and writes only its own positions, so these steps need no
     * barrier between them. */
    static __device__ __forceinline__ void cross_global(C *const (&gf)[3], unsigned in_y, unsigned out_y,
                                                        const Ops &op, const Instance &I, const Tables &tab, R h6,
                                                        int eom_idler, double &acc, int t, int rank)
    {
        const C *__restrict__ twN = reinterpret_cast<const C *>(tab.twN);
        C co0[NCO], co1[NCO];
#pragma unroll
        for (int k = 0; k < NCO; k++) {
            co0[k] = op.rk0 ? ldc<C>(op.rk0, k) : mk<C>((R)0, (R)0);
            co1[k] = op.rk1 ? ldc<C>(op.rk1, k) : mk<C>((R)0, (R)0);
        }
#pragma unroll 1
        for (int j = 0; j < J; j++) {
            const int n1 = rank * (M / CL) + t + j * T;
            if constexpr (CL > 1) {
#pragma unroll 1
                for (int f = 0; f < F; f++)
                    if ((in_y >> f) & 1u) cross_field<-1>(gf[f], twN, n1);
            }
#pragma unroll 2
            for (int c = 0; c < CL; c++) {
                C A[3];
#pragma unroll
                for (int f = 0; f < F; f++) A[f] = __ldcg(gf[f] + (size_t)c * M + n1);
                pointwise(A, n1 + M * c, op, co0, co1, I, tab, h6, eom_idler, acc);
#pragma unroll
                for (int f = 0; f < F; f++) __stcg(gf[f] + (size_t)c * M + n1, A[f]);
            }
            if constexpr (CL > 1) {
#pragma unroll 1
                for (int f = 0; f < F; f++)
                    if ((out_y >> f) & 1u) cross_field<+1>(gf[f], twN, n1);
            }
        }
    }

    /* One element-wise pass over the cluster.  Fields with their bit set in
     * in_y are read in the y domain (inverse cross stage applied), the
     * others as time values; out_y likewise for the write-back.  Thread t
     * of CTA `rank` owns positions n1 = rank M/CL + t + j T, j < J, in every
     * CTA's home; it reads and writes only those. */
    static __device__ __forceinline__ void cross(C *home, C *const (&gf)[3], unsigned in_y, unsigned out_y,
                                                 const Ops &op, const Instance &I, const Tables &tab, R h6,
                                                 int eom_idler, double &acc, int t, int rank)
    {
        if constexpr (GH) {
            cross_global(gf, in_y, out_y, op, I, tab, h6, eom_idler, acc, t, rank);
            return;
        }
        const C *__restrict__ twN = reinterpret_cast<const C *>(tab.twN);
        C co0[NCO], co1[NCO];
#pragma unroll
        for (int k = 0; k < NCO; k++) {
            co0[k] = op.rk0 ? ldc<C>(op.rk0, k) : mk<C>((R)0, (R)0);
            co1[k] = op.rk1 ? ldc<C>(op.rk1, k) : mk<C>((R)0, (R)0);
        }
#pragma unroll 1
        for (int j = 0; j < J; j++) {
            const int n1 = rank * (M / CL) + t + j * T;
            const int sm = swz<C>(n1);
            C v[3][CL];
#pragma unroll
            for (int c = 0; c < CL; c++) {
                const C *src = peer(home, c);
#pragma unroll
                for (int f = 0; f < F; f++) v[f][c] = src[f * M + sm];
            }
            /* cross-stage twiddles W_N^{n1 c}: quarter turn m and the residual
             * rotation (tan, sin) from the table */
            if constexpr (CL > 1) {
#pragma unroll
                for (int f = 0; f < F; f++) {
                    if ((in_y >> f) & 1u) {
#pragma unroll
                        for (int c = 1; c < CL; c++) {
                            const long q = (long)n1 * c;
                            const C w = __ldg(twN + q);
                            const int qm = (int)(((4 * q + N / 2) / N) & 3);
                            v[f][c] = shear_rot(iq_rt(v[f][c], (-qm) & 3), -w.x, -w.y);
                        }
                        dft<-1, CL>(v[f]);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CL; c++) {
                C A[3];
#pragma unroll
                for (int f = 0; f < F; f++) A[f] = v[f][c];
                pointwise(A, n1 + M * c, op, co0, co1, I, tab, h6, eom_idler, acc);
#pragma unroll
                for (int f = 0; f < F; f++) v[f][c] = A[f];
            }
            if constexpr (CL > 1) {
#pragma unroll
                for (int f = 0; f < F; f++) {
                    if ((out_y >> f) & 1u) {
                        dft<+1, CL>(v[f]);
#pragma unroll
                        for (int c = 1; c < CL; c++) {
                            const long q = (long)n1 * c;
                            const C w = __ldg(twN + q);
                            const int qm = (int)(((4 * q + N / 2) / N) & 3);
                            v[f][c] = shear_rot(iq_rt(v[f][c], qm), w.x, w.y);
                        }
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CL; c++) {
                C *dst = peer(home, c);
#pragma unroll
                for (int f = 0; f < F; f++) dst[f * M + sm] = v[f][c];
            }
        }
    }

    /* Local T->W, multiply by a table row (or the GDD factor), local W->T. */
    template <int MODE> /* 0: table row, 1: GDD/TOD factor formed in FP64 */
    static __device__ __forceinline__ void spectral(C *home, C *scratch, const C *__restrict__ row,
                                                    const float *__restrict__ w, double gdd, double tod,
                                                    int use_tod, double inv_n, const StageTwiddles<M, C> &tw,
                                                    int t)
    {
        C reg[16];
        if constexpr (GH) {
            /* home: this CTA's M points of the field in global memory */
#pragma unroll
            for (int e = 0; e < 16; e++) reg[e] = __ldcg(home + t + e * T);
        } else {
            load_own<M>(home, reg, t);
        }
        C *bufA = GH ? scratch : (INPLACE ? home : scratch);
        C *bufB = GH ? scratch : home;
        local_transform<+1, M, 0, INPLACE>(reg, bufA, bufB, tw, t);
        /* the factor F = 1 + d is applied as (A + A d) / N (1/N is exact) */
        const R s_n = (R)inv_n;
        if constexpr (MODE == 0) {
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const C x = cscale(reg[e], s_n);
                reg[e] = cadd(x, cmul(x, __ldg(row + t + e * T)));
            }
        } else {
#pragma unroll 4
            for (int e = 0; e < 16; e++) {
                /* functions.cuh:156-186, formed in FP64 */
                const double wk = (double)__ldg(w + t + e * T);
                const double ph = use_tod ? 0.5 * wk * (wk * gdd + wk * wk * tod / 3.0) : 0.5 * wk * wk * gdd;
                double sn, cs;
                sincos(ph, &sn, &cs);
                /* cos(ph) - 1 = -2 sin^2(ph/2), exact for small ph */
                const double sh = sin(0.5 * ph);
                const C x = cscale(reg[e], s_n);
                reg[e] = cadd(x, cmul(x, mk<C>((R)(-2.0 * sh * sh), (R)sn)));
            }
        }
        local_transform<-1, M, P - 1, INPLACE>(reg, bufA, bufB, tw, t);
        if constexpr (GH) {
#pragma unroll
            for (int e = 0; e < 16; e++) __stcg(home + t + e * T, reg[e]);
        } else {
            store_own<M>(home, reg, t);
        }
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

    static __device__ __forceinline__ void run(const LaunchArgs &a)
    {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        C *const sm = reinterpret_cast<C *>(smem_raw);
        C *home = GH ? nullptr : sm;
        C *scratch = GH ? sm : (INPLACE ? home : home + (size_t)F * M);
        __shared__ double red[32];
        __shared__ double red_cl;
        __shared__ int next_inst;
        const int t = threadIdx.x;
        int rank = 0;
        if constexpr (CL > 1) rank = (int)cg::this_cluster().block_rank();

        C *twtab = sm + field_elems();
        fill_twiddle_table<M>(twtab, t);
        StageTwiddles<M, C> tw;
        tw.init(t, twtab);
        __syncthreads();

        bool first = true;
        for (;;) {
            int idx;
            if (a.inst) {
                if (rank == 0 && t == 0) next_inst = atomicAdd(a.queue, 1);
                bar();
                idx = *peer(&next_inst, 0);
                bar();
                if (idx >= a.n_inst) break;
            } else {
                if (!first) break;
                idx = 0;
            }
            first = false;
            const Instance &I = a.inst ? a.inst[idx] : a.single;
            /* this instance's tables: its own where it has them, else the launch's */
            Tables tab = a.tab;
            int use_eom = a.use_eom;
            if (I.disp) {
                tab.disp = I.disp;
                tab.rk = I.rk;
                tab.w = I.w;
                tab.h6 = I.h6;
                tab.eom = I.eom;
                use_eom = I.eom != nullptr;
            }
            const R h6 = (R)tab.h6;
            const C *__restrict__ rk = reinterpret_cast<const C *>(tab.rk);
            const C *__restrict__ disp = reinterpret_cast<const C *>(tab.disp);
            const float *__restrict__ wtab = tab.w + (size_t)rank * M;
            int rt_begin = I.rt_begin, rt_count = I.rt_count, patience = I.patience, calm = 0;
            double tol = I.tol, prev_ps = -1.0;
            if (I.st_flag) {
                /* batch instance: resume from its saved state, skip if done */
                if (*(volatile int *)I.st_flag != 0) continue;
                rt_begin = *(volatile int *)I.st_rt;
                rt_count = min(a.chunk, rt_limit(a, I) - rt_begin);
                prev_ps = rt_begin > 0 ? *(volatile double *)I.st_ps : -1.0;
                calm = *(volatile int *)I.st_calm;
                tol = a.tol;
                patience = a.patience;
            }

            C *const gf[3] = {reinterpret_cast<C *>(I.Ap), reinterpret_cast<C *>(I.As),
                              reinterpret_cast<C *>(I.Ai)};
            /* the field f of this CTA for the local transforms */
            auto fld = [&](int f) -> C * { return GH ? gf[f] + (size_t)rank * M : home + (size_t)f * M; };
            if constexpr (!GH) {
#pragma unroll
                for (int f = 0; f < F; f++)
#pragma unroll
                    for (int e = 0; e < 16; e++)
                        home[f * M + swz<C>(t + e * T)] = gf[f][(size_t)rank * M + t + e * T];
            }
            xsync();

            double ps = prev_ps, acc = 0.0;
            int rts = 0, flag = 0;
            bool stop = false;
            const C *last_row = rk + (size_t)(a.n_z - 1) * NCO;
            for (int rt = rt_begin; rt < rt_begin + rt_count && !stop; rt++) {
                double th[3] = {0.0, 0.0, 0.0};
                {
                    Ops op{};
                    op.inject = !a.pass_only;
                    if (a.regime == 1) {
                        /* ReadPump offsets, functions.cuh:196-210 (Q6) */
                        const int nrt = I.n_rt_total;
                        op.poff = (rt == 0) ? 0 : ((rt > 0 && rt < nrt - 1) ? (long)rt * N : (long)N * nrt - 1 - N);
                    }
                    op.rk0 = rk;
                    frame_step(op, tab, frame_index(rt, 0), th);
                    cross(home, gf, 0u, ALL, op, I, tab, h6, a.eom_idler, acc, t, rank);
                    xsync();
                }
                for (int s = 0; s < a.n_z; s++) {
#pragma unroll 1
                    for (int f = 0; f < F; f++)
                        spectral<0>(fld(f), scratch, disp + ((size_t)f * CL + rank) * M, nullptr, 0.0, 0.0, 0,
                                    tab.inv_n, tw, t);
                    xsync();
                    if (s + 1 < a.n_z) {
                        Ops op{};
                        op.rk0 = rk + (size_t)s * NCO;
                        op.rk1 = rk + (size_t)(s + 1) * NCO;
                        frame_step(op, tab, frame_index(rt, s + 1), th);
                        cross(home, gf, ALL, ALL, op, I, tab, h6, a.eom_idler, acc, t, rank);
                        xsync();
                    }
                }
                rts++;
                if (a.pass_only) {
                    Ops op{};
                    op.rk0 = last_row;
                    frame_back(op, th);
                    cross(home, gf, ALL, 0u, op, I, tab, h6, a.eom_idler, acc, t, rank);
                    xsync();
                    break;
                }
                const bool save = (rt >= I.save_first && rt < I.save_first + I.save_count);
                Ops end{};
                end.addphase = 1;
                end.ph_s = make_double2(I.phase_s[0], I.phase_s[1]);
                end.ph_i = make_double2(I.phase_i[0], I.phase_i[1]);
                end.save = save;
                end.slot = save ? (size_t)(rt - I.save_first) * N : 0;
                end.power = 1;
                acc = 0.0;
                if (I.gdd != 0.0) {
                    /* GDD / TOD compensation of the resonant fields (cuOPO.cu:521-553):
                     * signal and idler go to the frequency domain, the pump stays in time */
                    Ops op{};
                    op.rk0 = last_row;
                    op.eom = use_eom;
                    const unsigned res = ALL & ~1u;
                    cross(home, gf, ALL, res, op, I, tab, h6, a.eom_idler, acc, t, rank);
                    xsync();
                    spectral<1>(fld(1), scratch, nullptr, wtab, I.gdd, I.tod_s, I.use_tod_s, tab.inv_n, tw, t);
                    if constexpr (F == 3)
                        spectral<1>(fld(2), scratch, nullptr, wtab, I.gdd, I.tod_i, I.use_tod_i, tab.inv_n, tw, t);
                    xsync();
                    frame_back(end, th);
                    cross(home, gf, res, 0u, end, I, tab, h6, a.eom_idler, acc, t, rank);
                } else {
                    end.rk0 = last_row;
                    end.eom = use_eom;
                    frame_back(end, th);
                    cross(home, gf, ALL, 0u, end, I, tab, h6, a.eom_idler, acc, t, rank);
                }
                /* signal power over the cluster, summed in rank order by every CTA */
                double part = block_sum(acc, red, t);
                if constexpr (CL > 1) {
                    if (t == 0) red_cl = part;
                    csync();
                    part = 0.0;
#pragma unroll
                    for (int c = 0; c < CL; c++) part += *peer(&red_cl, c);
                }
                ps = part * tab.inv_n;
                /* single launches record from rt_begin, batch instances by round trip */
                if (rank == 0 && t == 0 && I.ps_hist) I.ps_hist[I.st_flag ? rt : rt - rt_begin] = ps;
                if (!(ps == ps) || ps > 1.0e300) {
                    if (rank == 0 && t == 0 && a.status) atomicCAS(a.status, 0, (int)ST_NONFINITE);
                    flag = ST_NONFINITE;
                    stop = true;
                }
                /* convergence: relative change of the signal power per rt below
                 * tol for `patience` consecutive rts (from the second rt on) */
                if (tol > 0.0 && prev_ps > 0.0 && ps > 0.0 && fabs(ps - prev_ps) < tol * ps) {
                    if (++calm >= (patience > 0 ? patience : 1) && flag == 0) {
                        flag = ST_CONVERGED;
                        stop = true;
                    }
                } else {
                    calm = 0;
                }
                prev_ps = ps;
            }
            if constexpr (!GH) {
#pragma unroll
                for (int f = 0; f < F; f++)
#pragma unroll
                    for (int e = 0; e < 16; e++)
                        gf[f][(size_t)rank * M + t + e * T] = home[f * M + swz<C>(t + e * T)];
            }
            if (rank == 0 && t == 0) {
                if (I.rt_done) *I.rt_done = rts;
                if (I.ps_out) *I.ps_out = ps;
                if (I.flag_out) *I.flag_out = flag;
                if (I.st_flag) {
                    *I.st_rt = rt_begin + rts;
                    *I.st_ps = ps;
                    *I.st_calm = calm;
                    *I.st_flag = flag != 0 ? flag : (rt_begin + rts >= rt_limit(a, I) ? (int)ST_LIMIT : 0);
                }
            }
            bar();
        }
    }
};

template <typename R, int F, int M, int CL, int HM, int MINB>
__global__ void __launch_bounds__(M / 16, MINB) ssfm_kernel(const LaunchArgs a)
{
    Ssfm<R, F, M, CL, HM>::run(a);
}

}  // namespace cuopo
