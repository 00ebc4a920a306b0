/*
 * solver.cu -- plans, table construction and the GPU entry points of the
 * C ABI (include/cuopo.h).
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <array>
#include <mutex>
#include <vector>

#include "cuopo.h"
#include "internal.h"
#include "ssfm.cuh"

using namespace cuopo;

struct cuopo_plan {
    cuopo_params p;
    int precision;    /* CUOPO_F32 or CUOPO_F64: the field type and kernel */
    int phase32;      /* CUOPO_F32_PHASE32 plans: phase factors in FP32 */
    int F;            /* number of fields */
    int N;            /* grid points */
    int threads;      /* CTA size */
    int cluster;      /* CTAs per instance */
    size_t smem;      /* dynamic shared memory per CTA */
    void *d_disp;     /* [F][CL][M], entry [f][k2][k1] = D_f(k2 + CL k1) */
    void *d_rk;       /* [(n_z+1)][NCO] */
    void *d_eom;      /* [N] or NULL */
    float *d_w;       /* [CL][M], same permutation */
    void *d_twN;      /* [N] W_N^q (cluster plans) or NULL */
    double2 *d_frame_u; /* [NFRAME] random frame angles */
    void *d_frame_c;    /* [NFRAME][3] their phasors */
    int *d_status;
    double h6;
};

/* ---------------------------------------------------------------- errors */

static thread_local char g_err[512] = "no error";

extern "C" cuopo_status cuopo_fail(cuopo_status st, const char *msg)
{
    snprintf(g_err, sizeof(g_err), "%s", msg);
    return st;
}

static cuopo_status cuda_fail(cudaError_t e, const char *what)
{
    char buf[400];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return cuopo_fail(CUOPO_ECUDA, buf);
}

extern "C" const char *cuopo_last_error(void) { return g_err; }
extern "C" const char *cuopo_version(void) { return "cuopo_b200 0.1.0 (sm_100a)"; }

/* -------------------------------------------------------- kernel registry */

typedef cudaError_t (*launch_fn)(const LaunchArgs &, int clusters, cudaStream_t);
typedef int (*occ_fn)(void);

template <typename R, int F, int M, int CL, int HM, int MINB>
static cudaError_t prepare_kernel()
{
    using K = Ssfm<R, F, M, CL, HM>;
    static cudaError_t st = [] {
        cudaError_t e = cudaFuncSetAttribute(ssfm_kernel<R, F, M, CL, HM, MINB>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)K::smem_bytes());
        if (e == cudaSuccess && CL > 8)
            e = cudaFuncSetAttribute(ssfm_kernel<R, F, M, CL, HM, MINB>,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        return e;
    }();
    return st;
}

template <typename R, int F, int M, int CL, int HM, int MINB>
static cudaLaunchConfig_t make_config(int clusters, cudaStream_t st, cudaLaunchAttribute *attr)
{
    using K = Ssfm<R, F, M, CL, HM>;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(clusters * CL));
    cfg.blockDim = dim3(K::T);
    cfg.dynamicSmemBytes = K::smem_bytes();
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

template <typename R, int F, int M, int CL, int HM, int MINB>
static cudaError_t launch_impl(const LaunchArgs &a, int clusters, cudaStream_t st)
{
    cudaError_t e = prepare_kernel<R, F, M, CL, HM, MINB>();
    if (e != cudaSuccess) return e;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = make_config<R, F, M, CL, HM, MINB>(clusters, st, attr);
    e = cudaLaunchKernelEx(&cfg, ssfm_kernel<R, F, M, CL, HM, MINB>, a);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

/* Clusters (of CL CTAs) of this kernel that can be resident at once (0 on error). */
template <typename R, int F, int M, int CL, int HM, int MINB>
static int occupancy_impl()
{
    if (prepare_kernel<R, F, M, CL, HM, MINB>() != cudaSuccess) return 0;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = make_config<R, F, M, CL, HM, MINB>(1, 0, attr);
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, ssfm_kernel<R, F, M, CL, HM, MINB>, &cfg) != cudaSuccess) return 0;
    return n;
}

struct KernelEntry {
    int precision, F, M, CL;
    int home; /* 0, 1: fields in shared memory (1: in place); 2: in global memory */
    size_t smem;
    launch_fn fn;
    occ_fn occ;
};

#define CUOPO_K(R, PREC, F, M, CL, HM, MINB)                                                  \
    {PREC, F, M, CL, HM, Ssfm<R, F, M, CL, HM>::smem_bytes(), &launch_impl<R, F, M, CL, HM, MINB>, \
     &occupancy_impl<R, F, M, CL, HM, MINB>}

/* Built configurations (R, precision, equations, points per CTA, CTAs per
 * cluster, field placement as Ssfm's HM, minimum CTAs per SM).  Where a grid
 * size has more than one, cuopo_autotune times them and records the winner;
 * without a recorded choice the first entry with M * CL == n_t is used (the
 * entries are in order of measured batch throughput on the B200: 2-eq 2^13,
 * 2^14 and 2^15 run faster as clusters of 2, 4 and 8 4096-point CTAs, two
 * CTAs per SM, than as 1, 2 and 4 8192-point CTAs, one per SM).  The
 * single-CTA entries stay reachable for callers that need one
 * (crystal_pass_noalloc). */
static const KernelEntry k_kernels[] = {
    CUOPO_K(float, CUOPO_F32, 2, 512, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 1024, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 2048, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 4096, 1, false, 2),
    CUOPO_K(float, CUOPO_F32, 2, 4096, 2, false, 2),
    CUOPO_K(float, CUOPO_F32, 2, 8192, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 4096, 4, false, 2),
    CUOPO_K(float, CUOPO_F32, 2, 4096, 8, false, 2),
    CUOPO_K(float, CUOPO_F32, 2, 8192, 2, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 8192, 4, false, 1),
    CUOPO_K(float, CUOPO_F32, 2, 8192, 8, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 512, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 1024, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 2048, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 4096, 1, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 8192, 1, true, 1),
    CUOPO_K(float, CUOPO_F32, 3, 4096, 4, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 4096, 8, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 4096, 16, false, 1),
    CUOPO_K(float, CUOPO_F32, 3, 8192, 16, true, 1),
    CUOPO_K(double, CUOPO_F64, 2, 512, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 1024, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 2048, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 4096, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 4096, 2, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 4096, 4, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 4096, 8, false, 1),
    CUOPO_K(double, CUOPO_F64, 2, 4096, 16, false, 1),
    CUOPO_K(double, CUOPO_F64, 3, 512, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 3, 1024, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 3, 2048, 1, false, 1),
    CUOPO_K(double, CUOPO_F64, 3, 4096, 1, true, 1),
    CUOPO_K(double, CUOPO_F64, 3, 4096, 2, true, 1),
    CUOPO_K(double, CUOPO_F64, 3, 2048, 8, false, 1),
    CUOPO_K(double, CUOPO_F64, 3, 4096, 8, true, 1),
    CUOPO_K(double, CUOPO_F64, 3, 4096, 16, true, 1),
    /* 2^17 FP64 points of 3 fields (6 MiB) exceed the shared memory of a
     * 16-CTA cluster: the fields stay in global memory (L2) */
    CUOPO_K(double, CUOPO_F64, 3, 8192, 16, 2, 1),
};

/* Autotuned choices, process-wide: (precision, F, N) -> entry. */
struct TunedChoice {
    int precision, F, N;
    const KernelEntry *k;
};
static std::mutex g_tune_mu;
static std::vector<TunedChoice> g_tuned;
/* set by cuopo_autotune on its own thread while it times one candidate */
static thread_local const KernelEntry *g_force = nullptr;

static const KernelEntry *find_kernel(int precision, int F, int N, bool single_cta = false)
{
    if (!single_cta) {
        if (g_force && g_force->precision == precision && g_force->F == F && g_force->M * g_force->CL == N)
            return g_force;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (const TunedChoice &c : g_tuned)
            if (c.precision == precision && c.F == F && c.N == N) return c.k;
    }
    for (const KernelEntry &k : k_kernels)
        if (k.precision == precision && k.F == F && k.M * k.CL == N && (!single_cta || k.CL == 1)) return &k;
    return nullptr;
}

/* ------------------------------------------------------------ host tables */

static int is_pow2i(long n) { return n > 0 && (n & (n - 1)) == 0; }

/* Stage times of the RK4 half steps: z_s accumulated as the reference does
 * (cwes2.cuh:142,209: real_t z += dz), stage offsets dz/4 and dz/2
 * (cwes2.cuh:152,157,162). */
template <typename ZT>
static void stage_times(const cuopo_params &p, int s_count, std::vector<double> &zs)
{
    zs.resize((size_t)s_count * 3);
    ZT z = 0;
    const ZT dz = (ZT)p.dz;
    for (int s = 0; s < s_count; s++) {
        zs[3 * s + 0] = (double)z;
        zs[3 * s + 1] = (double)(ZT)(z + dz / 4);
        zs[3 * s + 2] = (double)(ZT)(z + dz / 2);
        z += dz;
    }
}

/* sin and cos of a phase: in FP64, or (p32) in FP32 after reducing the
 * argument to [-pi, pi] in FP64 -- the CUOPO_F32_PHASE32 variant, the
 * cheapest way a float build forms e^{i ph} without losing a large argument
 * (the reference uses FP32 cos/sin of a float argument,
 * src/headers/operators.cuh:120-126). */
static void phase_sc(double ph, bool p32, double &sn, double &cs)
{
    if (p32) {
        const float r = (float)std::remainder(ph, 2.0 * M_PI);
        sn = (double)sinf(r);
        cs = (double)cosf(r);
    } else {
        sn = std::sin(ph);
        cs = std::cos(ph);
    }
}

template <typename R>
static std::vector<unsigned char> build_tables(const cuopo_params &p, const float *w, const float *T, int CL,
                                               std::vector<unsigned char> &rk_out,
                                               std::vector<unsigned char> &eom_out,
                                               std::vector<unsigned char> &twn_out, double &h6, bool p32 = false)
{
    using C = cpx<R>;
    const int N = p.n_t;
    const int F = p.n_eqs;
    /* LinearOperator, cwes2.cuh:103-121 / cwes3.cuh:107-128: per field the
     * group-velocity term (Q4), GVD, TOD, attenuation exp(-alpha dz/2);
     * CUFFTscale's 1/N (functions.cuh:126-135) is applied in the kernel. */
    double gvm[3], b2[3], b3[3], al[3];
    if (F == 2) {
        gvm[0] = 1.0 / p.vp - 1.0 / p.vs;
        gvm[1] = 0.0;
    } else {
        gvm[0] = 1.0 / p.vp - 1.0 / p.vi;
        gvm[1] = 0.0;
        gvm[2] = 1.0 / p.vi - 1.0 / p.vs;
    }
    b2[0] = p.b2p; b2[1] = p.b2s; b2[2] = p.b2i;
    b3[0] = p.b3p; b3[1] = p.b3s; b3[2] = p.b3i;
    al[0] = p.alpha_crp; al[1] = p.alpha_crs; al[2] = p.alpha_cri;
    std::vector<unsigned char> disp(sizeof(C) * (size_t)F * N);
    C *D = reinterpret_cast<C *>(disp.data());
    const double z = p.dz;
    const int M = N / CL;
    for (int f = 0; f < F; f++) {
        const double att = std::exp(-0.5 * al[f] * z) / (double)N;
        for (int k = 0; k < N; k++) {
            const double wk = (double)w[k];
            const double ph = z * wk * (gvm[f] + 0.5 * wk * b2[f] + wk * wk * b3[f] / 6.0);
            /* frequency k = k2 + CL k1 is entry k1 of CTA k2's row.  Stored as
             * d = N D - 1 and applied as (A + A d) / N: the factor's float
             * rounding error then scales with |d| (tiny near w = 0, where CW
             * fields live) instead of biasing every slice by up to half an
             * ulp of att, which would compound over thousands of round trips. */
            const int k2 = k % CL, k1 = k / CL;
            const double a = att * (double)N;
            double sn, cs;
            phase_sc(ph, p32, sn, cs);
            const double dre = (ph == 0.0) ? a - 1.0 : a * cs - 1.0;
            D[(size_t)f * N + (size_t)k2 * M + k1] = mk<C>((R)dre, (R)(a * sn));
        }
    }
    /* cross-stage twiddles W_N^q = exp(2 pi i q / N) as a quarter turn
     * m = round(4q/N) (recomputed in the kernel) and the residual rotation
     * phi = 2 pi q/N - m pi/2, |phi| <= pi/4, stored as (tan(phi/2), sin(phi)) */
    twn_out.clear();
    if (CL > 1) {
        twn_out.resize(sizeof(C) * (size_t)N);
        C *W = reinterpret_cast<C *>(twn_out.data());
        for (long q = 0; q < N; q++) {
            const long m = (4 * q + N / 2) / N;
            const double phi = 2.0 * M_PI * (double)(4 * q - m * N) / (4.0 * (double)N);
            W[q] = mk<C>((R)std::tan(0.5 * phi), (R)std::sin(phi));
        }
    }
    /* RK4 stage coefficients per slice (one extra zero row at the end). */
    const int nco = (F == 2) ? 6 : 3;
    std::vector<double> zs;
    if (sizeof(R) == 4) stage_times<float>(p, p.n_z, zs);
    else stage_times<double>(p, p.n_z, zs);
    rk_out.assign(sizeof(C) * (size_t)(p.n_z + 1) * nco, 0);
    C *co = reinterpret_cast<C *>(rk_out.data());
    const double h = (sizeof(R) == 4) ? (double)(float)((float)p.dz / 2) : p.dz / 2;
    h6 = h / 6.0;
    for (int s = 0; s < p.n_z; s++) {
        if (F == 2) {
            /* dAdz, cwes2.cuh:37-38: i kp e^{+i dk z}, i ks e^{-i dk z} */
            for (int j = 0; j < 3; j++) {
                const double ph = p.dk * zs[3 * s + j];
                double c, sn;
                phase_sc(ph, p32, sn, c);
                co[s * 6 + 2 * j + 0] = mk<C>((R)(-p.kp * sn), (R)(p.kp * c));
                co[s * 6 + 2 * j + 1] = mk<C>((R)(p.ks * sn), (R)(p.ks * c));
            }
        } else {
            /* dAdz, cwes3.cuh:37-39 with k2 = k3 (Q3): the half step is
             * A += (h/6) i kappa (E(z) + 4 E(z+dz/4) + E(z+dz/2)) P. */
            double er = 0, ei = 0;
            const double wgt[3] = {1.0, 4.0, 1.0};
            for (int j = 0; j < 3; j++) {
                double c, sn;
                phase_sc(p.dk * zs[3 * s + j], p32, sn, c);
                er += wgt[j] * c;
                ei += wgt[j] * sn;
            }
            /* pump: E- = conj(E+) */
            const double kap[3] = {p.kp, p.ks, p.ki};
            for (int f = 0; f < 3; f++) {
                const double sr = er, si = (f == 0) ? -ei : ei;
                /* h6 * i * kappa * (sr + i si) = h6 kappa (-si + i sr) */
                co[s * 3 + f] = mk<C>((R)(h6 * kap[f] * -si), (R)(h6 * kap[f] * sr));
            }
        }
    }
    /* EOM factor exp(i m sin(2 pi fpm T)), functions.cuh:242-253 */
    eom_out.clear();
    if (p.use_eom) {
        eom_out.resize(sizeof(C) * (size_t)N);
        C *E = reinterpret_cast<C *>(eom_out.data());
        for (int k = 0; k < N; k++) {
            double s1, c1, sn, cs;
            phase_sc(2.0 * M_PI * p.fpm * (double)T[k], p32, s1, c1);
            phase_sc(p.mod_depth * s1, p32, sn, cs);
            E[k] = mk<C>((R)cs, (R)sn);
        }
    }
    return disp;
}

extern "C" cuopo_status cuopo_plan_create(cuopo_plan **out, const cuopo_params *p,
                                          const float *w_host, const float *T_host, int precision)
{
    cuopo::Range range_("cuopo_plan_create");
    if (!out || !p) return cuopo_fail(CUOPO_EINVAL, "plan_create: NULL argument");
    *out = nullptr;
    if (p->n_eqs != 2 && p->n_eqs != 3) return cuopo_fail(CUOPO_EINVAL, "n_eqs must be 2 or 3");
    if (!is_pow2i(p->n_t)) return cuopo_fail(CUOPO_EINVAL, "n_t must be a power of 2");
    if (p->n_z < 1) return cuopo_fail(CUOPO_EINVAL, "n_z must be >= 1");
    if (precision != CUOPO_F32 && precision != CUOPO_F64 && precision != CUOPO_F32_PHASE32)
        return cuopo_fail(CUOPO_EINVAL, "precision must be CUOPO_F32, CUOPO_F64 or CUOPO_F32_PHASE32");
    const bool phase32 = precision == CUOPO_F32_PHASE32;
    if (phase32) precision = CUOPO_F32;
    const KernelEntry *k = find_kernel(precision, p->n_eqs, p->n_t);
    if (!k) return cuopo_fail(CUOPO_EUNSUPPORTED, "no kernel built for this (precision, n_eqs, n_t)");

    std::vector<float> w((size_t)p->n_t), T((size_t)p->n_t);
    if (w_host) std::memcpy(w.data(), w_host, sizeof(float) * p->n_t);
    if (T_host) std::memcpy(T.data(), T_host, sizeof(float) * p->n_t);
    if (!w_host || !T_host) {
        if (p->t_rt <= 0) return cuopo_fail(CUOPO_EINVAL, "t_rt must be > 0 when grids are not given");
        cuopo_status st = cuopo_make_grids(p->n_t, p->t_rt, T_host ? nullptr : T.data(),
                                           w_host ? nullptr : w.data());
        if (st != CUOPO_OK) return st;
    }

    std::vector<unsigned char> disp, rk, eom, twn;
    double h6 = 0;
    const int CL = k->CL;
    if (precision == CUOPO_F32) disp = build_tables<float>(*p, w.data(), T.data(), CL, rk, eom, twn, h6, phase32);
    else disp = build_tables<double>(*p, w.data(), T.data(), CL, rk, eom, twn, h6);
    /* frequency grid in the same per-CTA order as the dispersion table */
    std::vector<float> wp((size_t)p->n_t);
    for (int q = 0; q < p->n_t; q++) wp[(size_t)(q % CL) * (p->n_t / CL) + q / CL] = w[q];

    cuopo_plan *pl = new (std::nothrow) cuopo_plan();
    if (!pl) return cuopo_fail(CUOPO_ENOMEM, "plan_create: out of host memory");
    pl->p = *p;
    pl->precision = precision;
    pl->phase32 = phase32;
    pl->F = p->n_eqs;
    pl->N = p->n_t;
    pl->threads = k->M / 16;
    pl->cluster = k->CL;
    pl->smem = k->smem;
    pl->h6 = h6;
    cudaError_t e;
    if ((e = cudaMalloc(&pl->d_disp, disp.size())) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_rk, rk.size())) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_w, sizeof(float) * p->n_t)) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_status, sizeof(int))) != cudaSuccess ||
        (!eom.empty() && (e = cudaMalloc(&pl->d_eom, eom.size())) != cudaSuccess) ||
        (!twn.empty() && (e = cudaMalloc(&pl->d_twN, twn.size())) != cudaSuccess)) {
        cuopo_plan_destroy(pl);
        return e == cudaErrorMemoryAllocation ? cuopo_fail(CUOPO_ENOMEM, "plan_create: device allocation failed")
                                              : cuda_fail(e, "plan_create: cudaMalloc");
    }
    if ((e = cudaMemcpy(pl->d_disp, disp.data(), disp.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(pl->d_rk, rk.data(), rk.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(pl->d_w, wp.data(), sizeof(float) * p->n_t, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(pl->d_status, 0, sizeof(int))) != cudaSuccess ||
        (!eom.empty() && (e = cudaMemcpy(pl->d_eom, eom.data(), eom.size(), cudaMemcpyHostToDevice)) != cudaSuccess) ||
        (!twn.empty() && (e = cudaMemcpy(pl->d_twN, twn.data(), twn.size(), cudaMemcpyHostToDevice)) != cudaSuccess)) {
        cuopo_plan_destroy(pl);
        return cuda_fail(e, "plan_create: upload");
    }
    {
        /* random frame table: u_s, u_i uniform in [0,1) turns (fixed seed) */
        std::vector<double2> fu(NFRAME);
        const size_t csz = precision == CUOPO_F32 ? sizeof(float2) : sizeof(double2);
        std::vector<unsigned char> fc(csz * 3 * NFRAME);
        unsigned long long st = 0x2545F4914F6CDD1Dull;
        auto next = [&st]() {
            st += 0x9E3779B97F4A7C15ull;
            unsigned long long z = st;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
        };
        for (int q = 0; q < NFRAME; q++) {
            /* frame angles in [-1/8, 1/8) turns; the pump turns by their sum,
             * at most a quarter turn, so no quarter-turn step is needed */
            const double us = 0.25 * next() - 0.125, ui = 0.25 * next() - 0.125;
            fu[q] = make_double2(us, ui);
            const double up = (p->n_eqs == 2) ? 2.0 * us : us + ui;
            const double ang[3] = {2.0 * M_PI * up, 2.0 * M_PI * us, 2.0 * M_PI * ui};
            for (int f = 0; f < 3; f++) {
                const double tt = std::tan(0.5 * ang[f]), ss = std::sin(ang[f]);
                if (precision == CUOPO_F32) ((float2 *)fc.data())[3 * q + f] = make_float2((float)tt, (float)ss);
                else ((double2 *)fc.data())[3 * q + f] = make_double2(tt, ss);
            }
        }
        if ((e = cudaMalloc(&pl->d_frame_u, sizeof(double2) * NFRAME)) != cudaSuccess ||
            (e = cudaMalloc(&pl->d_frame_c, fc.size())) != cudaSuccess ||
            (e = cudaMemcpy(pl->d_frame_u, fu.data(), sizeof(double2) * NFRAME, cudaMemcpyHostToDevice)) !=
                cudaSuccess ||
            (e = cudaMemcpy(pl->d_frame_c, fc.data(), fc.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
            cuopo_plan_destroy(pl);
            return cuda_fail(e, "plan_create: frame table");
        }
    }
    *out = pl;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_plan_destroy(cuopo_plan *pl)
{
    if (!pl) return CUOPO_OK;
    cudaFree(pl->d_disp);
    cudaFree(pl->d_rk);
    cudaFree(pl->d_eom);
    cudaFree(pl->d_w);
    cudaFree(pl->d_twN);
    cudaFree(pl->d_frame_u);
    cudaFree(pl->d_frame_c);
    cudaFree(pl->d_status);
    delete pl;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_plan_config(const cuopo_plan *pl, int *cluster, int *threads, int *smem)
{
    if (!pl) return cuopo_fail(CUOPO_EINVAL, "plan_config: NULL plan");
    if (cluster) *cluster = pl->cluster;
    if (threads) *threads = pl->threads;
    if (smem) *smem = (int)pl->smem;
    return CUOPO_OK;
}

static LaunchArgs base_args(const cuopo_plan *pl)
{
    LaunchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.tab.disp = pl->d_disp;
    a.tab.rk = pl->d_rk;
    a.tab.eom = pl->d_eom;
    a.tab.w = pl->d_w;
    a.tab.twN = pl->d_twN;
    a.tab.frame_u = pl->d_frame_u;
    a.tab.frame_c = pl->d_frame_c;
    a.tab.h6 = pl->h6;
    a.tab.inv_n = 1.0 / (double)pl->N;
    a.n_z = pl->p.n_z;
    a.regime = pl->p.regime;
    a.use_eom = pl->p.use_eom && pl->d_eom != nullptr;
    a.eom_idler = pl->p.eom_idler;
    a.status = pl->d_status;
    return a;
}

static void cavity_factors(const cuopo_params &p, Instance &I, bool p32 = false)
{
    /* AddPhase: sqrt(R) * exp(i pi delta), functions.cuh:145 */
    double sn, cs;
    phase_sc(M_PI * p.delta, p32, sn, cs);
    const double rs = std::sqrt(p.Rs), ri = std::sqrt(p.Ri);
    I.phase_s[0] = rs * cs;
    I.phase_s[1] = rs * sn;
    I.phase_i[0] = ri * cs;
    I.phase_i[1] = ri * sn;
    I.gdd = p.gdd;
    I.tod_s = p.tod_s;
    I.tod_i = p.tod_i;
    I.use_tod_s = (p.tod_s != 0 && p.b3s != 0);
    I.use_tod_i = (p.tod_i != 0 && p.b3i != 0);
}

static cuopo_status launch(cuopo_plan *pl, const LaunchArgs &a, int grid, void *stream)
{
    const KernelEntry *k = find_kernel(pl->precision, pl->F, pl->N);
    if (!k) return cuopo_fail(CUOPO_EUNSUPPORTED, "no kernel for plan");
    cudaError_t e = k->fn(a, grid, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_crystal_pass(cuopo_plan *pl, void *Ap, void *As, void *Ai, void *stream)
{
    cuopo::Range range_("cuopo_crystal_pass");
    if (!pl || !Ap || !As || (pl->F == 3 && !Ai)) return cuopo_fail(CUOPO_EINVAL, "crystal_pass: NULL argument");
    LaunchArgs a = base_args(pl);
    a.pass_only = 1;
    a.single.Ap = Ap;
    a.single.As = As;
    a.single.Ai = Ai;
    a.single.rt_begin = 0;
    a.single.rt_count = 1;
    a.single.save_first = 0;
    a.single.save_count = 0;
    return launch(pl, a, 1, stream);
}

extern "C" cuopo_status cuopo_round_trips(cuopo_plan *pl, void *Ap, void *As, void *Ai, const void *pump,
                                          int n_rt, int rt_begin, int rt_count, void *save_p, void *save_s,
                                          void *save_i, int save_first, int save_count, double *ps_hist,
                                          double tol, int *rt_done_dev, void *stream)
{
    cuopo::Range range_("cuopo_round_trips");
    if (!pl || !Ap || !As || (pl->F == 3 && !Ai)) return cuopo_fail(CUOPO_EINVAL, "round_trips: NULL field");
    if (rt_count < 0 || rt_begin < 0 || save_count < 0) return cuopo_fail(CUOPO_EINVAL, "round_trips: negative count");
    if (pl->p.regime == CUOPO_NS && (!pump || n_rt < 2))
        return cuopo_fail(CUOPO_EINVAL, "round_trips: NS regime needs the pump window and n_rt >= 2");
    if (pl->p.regime == CUOPO_NS && rt_begin + rt_count > n_rt)
        return cuopo_fail(CUOPO_EINVAL, "round_trips: round trips beyond the NS pump window");
    LaunchArgs a = base_args(pl);
    Instance &I = a.single;
    I.Ap = Ap;
    I.As = As;
    I.Ai = Ai;
    I.pump = pump;
    I.ap0 = pl->p.ap0;
    I.n_rt_total = n_rt;
    I.rt_begin = rt_begin;
    I.rt_count = rt_count;
    I.sv_p = save_p;
    I.sv_s = save_s;
    I.sv_i = save_i;
    I.save_first = save_first;
    I.save_count = save_count;
    I.ps_hist = ps_hist;
    I.tol = tol;
    I.rt_done = rt_done_dev;
    cavity_factors(pl->p, I, pl->phase32);
    return launch(pl, a, 1, stream);
}

extern "C" cuopo_status cuopo_plan_status(cuopo_plan *pl, int *status, int reset)
{
    if (!pl || !status) return cuopo_fail(CUOPO_EINVAL, "plan_status: NULL argument");
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, pl->d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "plan_status");
    if (reset && (e = cudaMemset(pl->d_status, 0, sizeof(int))) != cudaSuccess) return cuda_fail(e, "plan_status");
    *status = v;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_sync(void *stream)
{
    cudaError_t e = stream ? cudaStreamSynchronize((cudaStream_t)stream) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "sync");
    return CUOPO_OK;
}

/* ------------------------------------------------------------------ batches */

/* Instances of one launch: same number of fields, grid size, slices and
 * modulator target; their physics tables may differ (one plan each). */
struct BatchGroup {
    int F, n_t, n_z, eom_idler, regime;
    std::vector<cuopo_plan *> plans; /* plans[0] supplies the launch's tables */
    std::vector<int> members;
    Instance *d_inst;
    int *d_queue;
    cudaStream_t stream;
    cudaEvent_t done;
    int grid;
};

struct cuopo_batch {
    int count;
    int precision;
    std::vector<int> n_t, F;
    std::vector<uint64_t> seed;
    std::vector<size_t> offset;   /* element offset of each instance's fields */
    size_t total;                 /* total signal elements */
    void *d_pump;                 /* pump-field work buffers (n_t per instance) */
    void *d_signal;               /* signal fields, concatenated */
    void *d_idler;                /* idler fields (same offsets) when an instance has 3 fields */
    void *d_win;                  /* nanosecond instances: their pump windows (n_t x n_rt each) */
    double *d_hist;               /* nanosecond instances: signal power per round trip */
    std::vector<long> hist_off;   /* offset into d_hist, -1 for CW instances */
    std::vector<int> n_rt;        /* pump-window round trips (nanosecond instances) */
    double *d_ps;     /* per-instance resumable state (see Instance::st_*) */
    int *d_rt;
    int *d_flag;
    int *d_calm;
    std::vector<BatchGroup> groups;
    cudaEvent_t fork;
    std::vector<Instance> h_inst;
};

extern "C" cuopo_status cuopo_batch_destroy(cuopo_batch *b)
{
    if (!b) return CUOPO_OK;
    for (BatchGroup &g : b->groups)
        if (g.stream) cudaStreamSynchronize(g.stream);
    for (BatchGroup &g : b->groups) {
        for (cuopo_plan *pl : g.plans) cuopo_plan_destroy(pl);
        cudaFree(g.d_inst);
        cudaFree(g.d_queue);
        if (g.stream) cudaStreamDestroy(g.stream);
        if (g.done) cudaEventDestroy(g.done);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    cudaFree(b->d_pump);
    cudaFree(b->d_signal);
    cudaFree(b->d_idler);
    cudaFree(b->d_win);
    cudaFree(b->d_hist);
    cudaFree(b->d_ps);
    cudaFree(b->d_rt);
    cudaFree(b->d_flag);
    cudaFree(b->d_calm);
    delete b;
    return CUOPO_OK;
}

/* Parameters that go into a plan's tables (dispersion, RK4 coefficients,
 * grids, modulator); the rest (pump amplitude, mirrors, detuning, GDD/TOD)
 * is per instance. */
static std::vector<double> physics_key(const cuopo_params &p)
{
    return {(double)p.n_eqs, (double)p.n_t, (double)p.n_z, (double)p.regime, p.vp, p.vs, p.vi, p.b2p, p.b2s,
            p.b2i, p.b3p, p.b3s, p.b3i, p.dk, p.kp, p.ks, p.ki, p.dz, p.alpha_crp, p.alpha_crs, p.alpha_cri,
            (double)p.use_eom, (double)p.eom_idler, p.mod_depth, p.fpm, p.t_rt};
}

/* A batch of instances, each with its full parameter set; nanosecond
 * instances also with their pump window's round trips and pulse width
 * (ns_rt / ns_fwhm, NULL when there are none). */
static cuopo_status batch_build(cuopo_batch **out, const std::vector<cuopo_params> &prm,
                                const std::vector<uint64_t> &seeds, int precision,
                                const std::vector<int> *ns_rt = nullptr,
                                const std::vector<double> *ns_fwhm = nullptr)
{
    const int count = (int)prm.size();
    if (precision != CUOPO_F32 && precision != CUOPO_F64)
        return cuopo_fail(CUOPO_EINVAL, "batch_create: bad precision");
    bool any3 = false;
    size_t win_total = 0, hist_total = 0;
    for (int i = 0; i < count; i++) {
        const cuopo_params &p = prm[(size_t)i];
        if (p.regime == CUOPO_NS) {
            if (!ns_rt || !ns_fwhm)
                return cuopo_fail(CUOPO_EUNSUPPORTED,
                                  "batch_create: nanosecond instances need cuopo_batch_create_inputs (n_rt, pulse)");
            if ((*ns_rt)[(size_t)i] < 2) return cuopo_fail(CUOPO_EINVAL, "batch_create: nanosecond n_rt must be >= 2");
            win_total += (size_t)p.n_t * (size_t)(*ns_rt)[(size_t)i];
            hist_total += (size_t)(*ns_rt)[(size_t)i];
        } else if (p.regime != CUOPO_CW) {
            return cuopo_fail(CUOPO_EINVAL, "batch_create: bad regime");
        }
        if (p.n_eqs != 2 && p.n_eqs != 3) return cuopo_fail(CUOPO_EINVAL, "batch_create: n_eqs must be 2 or 3");
        if (!is_pow2i(p.n_t) || !find_kernel(precision, p.n_eqs, p.n_t))
            return cuopo_fail(CUOPO_EUNSUPPORTED, "batch_create: an instance has an unsupported n_t");
        if (p.n_z < 1) return cuopo_fail(CUOPO_EINVAL, "batch_create: n_z must be >= 1");
        if (!(p.Rs >= 0.0 && p.Rs <= 1.0) || !(p.Ri >= 0.0 && p.Ri <= 1.0))
            return cuopo_fail(CUOPO_EINVAL, "batch_create: reflectivity out of [0,1]");
        any3 = any3 || p.n_eqs == 3;
    }
    cuopo_batch *b = new (std::nothrow) cuopo_batch();
    if (!b) return cuopo_fail(CUOPO_ENOMEM, "batch_create: out of host memory");
    b->count = count;
    b->precision = precision;
    b->seed = seeds;
    b->offset.resize((size_t)count);
    size_t off = 0;
    for (int i = 0; i < count; i++) {
        b->n_t.push_back(prm[(size_t)i].n_t);
        b->F.push_back(prm[(size_t)i].n_eqs);
        b->offset[(size_t)i] = off;
        off += (size_t)prm[(size_t)i].n_t;
    }
    b->total = off;
    const size_t esz = precision == CUOPO_F32 ? 8 : 16;
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_pump, esz * off)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_signal, esz * off)) != cudaSuccess ||
        (any3 && (e = cudaMalloc(&b->d_idler, esz * off)) != cudaSuccess) ||
        (win_total && (e = cudaMalloc(&b->d_win, esz * win_total)) != cudaSuccess) ||
        (hist_total && (e = cudaMalloc(&b->d_hist, sizeof(double) * hist_total)) != cudaSuccess) ||
        (e = cudaMalloc(&b->d_ps, sizeof(double) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_rt, sizeof(int) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_flag, sizeof(int) * count)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_calm, sizeof(int) * count)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess) {
        cuopo_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? cuopo_fail(CUOPO_ENOMEM, "batch_create: device allocation failed")
                                              : cuda_fail(e, "batch_create");
    }
    cudaMemset(b->d_pump, 0, esz * off);
    cudaMemset(b->d_signal, 0, esz * off);
    if (b->d_idler) cudaMemset(b->d_idler, 0, esz * off);
    cudaMemset(b->d_ps, 0, sizeof(double) * count);
    cudaMemset(b->d_rt, 0, sizeof(int) * count);
    cudaMemset(b->d_flag, 0, sizeof(int) * count);
    cudaMemset(b->d_calm, 0, sizeof(int) * count);
    if (b->d_hist) cudaMemset(b->d_hist, 0, sizeof(double) * hist_total);
    /* nanosecond pump windows (cuOPO.cu:164-175,243-248), built on the host as
     * the reference does, one per nanosecond instance */
    std::vector<size_t> win_off((size_t)count, 0);
    b->hist_off.assign((size_t)count, -1);
    b->n_rt.assign((size_t)count, 0);
    {
        size_t wo = 0, ho = 0;
        std::vector<float> wf;
        std::vector<double> wd;
        for (int i = 0; i < count; i++) {
            const cuopo_params &p = prm[(size_t)i];
            if (p.regime != CUOPO_NS) continue;
            const int nrt = (*ns_rt)[(size_t)i];
            const size_t n = (size_t)p.n_t * (size_t)nrt;
            wf.resize(2 * n);
            cuopo_status st = cuopo_pump_ns(wf.data(), p.n_t, nrt, p.t_rt, p.ap0, (*ns_fwhm)[(size_t)i]);
            if (st != CUOPO_OK) {
                cuopo_batch_destroy(b);
                return st;
            }
            const void *src = wf.data();
            if (precision == CUOPO_F64) {
                wd.assign(wf.begin(), wf.end());
                src = wd.data();
            }
            if ((e = cudaMemcpy((char *)b->d_win + esz * wo, src, esz * n, cudaMemcpyHostToDevice)) != cudaSuccess) {
                cuopo_batch_destroy(b);
                return cuda_fail(e, "batch_create: pump windows");
            }
            win_off[(size_t)i] = wo;
            b->hist_off[(size_t)i] = (long)ho;
            b->n_rt[(size_t)i] = nrt;
            wo += n;
            ho += (size_t)nrt;
        }
    }

    /* one persistent launch per (fields, grid size, slices, modulator target, regime),
     * largest grids first; one plan (tables) per distinct physics */
    std::vector<std::array<int, 5>> keys;
    for (const cuopo_params &p : prm) {
        const std::array<int, 5> k = {p.n_eqs, p.n_t, p.n_z, p.eom_idler, p.regime};
        if (std::find(keys.begin(), keys.end(), k) == keys.end()) keys.push_back(k);
    }
    std::sort(keys.begin(), keys.end(), [](const std::array<int, 5> &x, const std::array<int, 5> &y) {
        return x[1] != y[1] ? x[1] > y[1] : x < y;
    });
    b->h_inst.resize((size_t)count);
    for (const std::array<int, 5> &key : keys) {
        b->groups.push_back(BatchGroup{});
        BatchGroup &g = b->groups.back();
        g.F = key[0];
        g.n_t = key[1];
        g.n_z = key[2];
        g.eom_idler = key[3];
        g.regime = key[4];
        std::vector<std::vector<double>> pkeys;
        std::vector<int> plan_of;
        for (int i = 0; i < count; i++) {
            const cuopo_params &p = prm[(size_t)i];
            if (p.n_eqs != g.F || p.n_t != g.n_t || p.n_z != g.n_z || p.eom_idler != g.eom_idler ||
                p.regime != g.regime)
                continue;
            g.members.push_back(i);
            const std::vector<double> pk = physics_key(p);
            size_t q = std::find(pkeys.begin(), pkeys.end(), pk) - pkeys.begin();
            if (q == pkeys.size()) {
                cuopo_plan *pl = nullptr;
                cuopo_status st = cuopo_plan_create(&pl, &p, nullptr, nullptr, precision);
                if (st != CUOPO_OK) {
                    cuopo_batch_destroy(b);
                    return st;
                }
                g.plans.push_back(pl);
                pkeys.push_back(pk);
            }
            plan_of.push_back((int)q);
        }
        const KernelEntry *k = find_kernel(precision, g.F, g.n_t);
        /* persistent grid: as many clusters as can be resident at once */
        const int occ = k->occ();
        if (occ < 1) {
            cuopo_batch_destroy(b);
            return cuopo_fail(CUOPO_ECUDA, "batch_create: kernel does not fit on the device");
        }
        g.grid = std::min((int)g.members.size(), occ);
        if ((e = cudaMalloc(&g.d_inst, sizeof(Instance) * g.members.size())) != cudaSuccess ||
            (e = cudaMalloc(&g.d_queue, sizeof(int))) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming)) != cudaSuccess) {
            cuopo_batch_destroy(b);
            return cuda_fail(e, "batch_create");
        }
        std::vector<Instance> hi(g.members.size());
        for (size_t j = 0; j < g.members.size(); j++) {
            const int i = g.members[j];
            const cuopo_params &p = prm[(size_t)i];
            const cuopo_plan *pl = g.plans[(size_t)plan_of[j]];
            Instance &I = hi[j];
            std::memset(&I, 0, sizeof(I));
            I.Ap = (char *)b->d_pump + esz * b->offset[(size_t)i];
            I.As = (char *)b->d_signal + esz * b->offset[(size_t)i];
            I.Ai = g.F == 3 ? (char *)b->d_idler + esz * b->offset[(size_t)i] : nullptr;
            I.pump = nullptr;
            I.ap0 = p.ap0;
            if (p.regime == CUOPO_NS) {
                I.pump = (char *)b->d_win + esz * win_off[(size_t)i];
                I.n_rt_total = b->n_rt[(size_t)i];
                I.ps_hist = b->d_hist + b->hist_off[(size_t)i];
            }
            cavity_factors(p, I);
            I.disp = pl->d_disp;
            I.rk = pl->d_rk;
            I.w = pl->d_w;
            I.eom = (p.use_eom && pl->d_eom) ? pl->d_eom : nullptr;
            I.h6 = pl->h6;
            I.st_ps = b->d_ps + i;
            I.st_rt = b->d_rt + i;
            I.st_flag = b->d_flag + i;
            I.st_calm = b->d_calm + i;
            b->h_inst[(size_t)i] = I;
        }
        if ((e = cudaMemcpy(g.d_inst, hi.data(), sizeof(Instance) * hi.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
            cuopo_batch_destroy(b);
            return cuda_fail(e, "batch_create: upload");
        }
    }
    *out = b;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_create(cuopo_batch **out, const cuopo_params *base, const cuopo_instance *inst,
                                           int count, int precision)
{
    cuopo::Range range_("cuopo_batch_create");
    if (!out || !base || !inst || count < 1) return cuopo_fail(CUOPO_EINVAL, "batch_create: bad argument");
    *out = nullptr;
    std::vector<cuopo_params> prm((size_t)count, *base);
    std::vector<uint64_t> seeds((size_t)count);
    for (int i = 0; i < count; i++) {
        cuopo_params &p = prm[(size_t)i];
        p.n_t = inst[i].n_t;
        p.ap0 = inst[i].ap0;
        p.Rs = inst[i].Rs;
        p.delta = inst[i].delta;
        p.gdd = inst[i].gdd;
        seeds[(size_t)i] = inst[i].seed;
    }
    return batch_build(out, prm, seeds, precision);
}

extern "C" cuopo_status cuopo_batch_create_inputs(cuopo_batch **out, const cuopo_inputs *in, const uint64_t *seeds,
                                                  int count, int precision)
{
    cuopo::Range range_("cuopo_batch_create_inputs");
    if (!out || !in || count < 1) return cuopo_fail(CUOPO_EINVAL, "batch_create_inputs: bad argument");
    *out = nullptr;
    std::vector<cuopo_params> prm((size_t)count);
    std::vector<uint64_t> sd((size_t)count);
    std::vector<int> nrt((size_t)count);
    std::vector<double> fwhm((size_t)count);
    for (int i = 0; i < count; i++) {
        cuopo_info info;
        cuopo_status st = cuopo_derive_params(&in[i], &prm[(size_t)i], &info);
        if (st != CUOPO_OK) return st;
        sd[(size_t)i] = seeds ? seeds[i] : (uint64_t)i;
        nrt[(size_t)i] = in[i].n_rt;
        fwhm[(size_t)i] = in[i].fwhm_ps;
    }
    return batch_build(out, prm, sd, precision, &nrt, &fwhm);
}

extern "C" cuopo_status cuopo_batch_total_elements(const cuopo_batch *b, long *n)
{
    if (!b || !n) return cuopo_fail(CUOPO_EINVAL, "batch_total_elements: NULL argument");
    *n = (long)b->total;
    return CUOPO_OK;
}

/* `st` waits for the latest step of every group.  Steps do not join the
 * caller's stream themselves: a group that finishes its part of step k
 * starts step k+1 while larger grids still finish theirs, so the SMs a
 * group's last wave leaves idle go to the others.  Every call that reads
 * or writes the batch's state joins here first. */
static cuopo_status join_groups(cuopo_batch *b, cudaStream_t st, const char *what)
{
    for (BatchGroup &g : b->groups) {
        cudaError_t e = cudaStreamWaitEvent(st, g.done, 0);
        if (e != cudaSuccess) return cuda_fail(e, what);
    }
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_wait(cuopo_batch *b, void *stream)
{
    if (!b) return cuopo_fail(CUOPO_EINVAL, "batch_wait: NULL batch");
    return join_groups(b, (cudaStream_t)stream, "batch_wait");
}

extern "C" cuopo_status cuopo_batch_seed_noise(cuopo_batch *b, double sigma, void *stream)
{
    if (!b) return cuopo_fail(CUOPO_EINVAL, "batch_seed_noise: NULL batch");
    {
        cuopo_status js = join_groups(b, (cudaStream_t)stream, "batch_seed_noise");
        if (js != CUOPO_OK) return js;
    }
    if (b->precision != CUOPO_F32) return cuopo_fail(CUOPO_EUNSUPPORTED, "batch_seed_noise: F32 batches only");
    for (int i = 0; i < b->count; i++) {
        cuopo_status st = cuopo_noise_device((char *)b->d_signal + 8 * b->offset[(size_t)i], b->n_t[(size_t)i], sigma,
                                             b->seed[(size_t)i], 0, stream);
        if (st == CUOPO_OK && b->F[(size_t)i] == 3)
            st = cuopo_noise_device((char *)b->d_idler + 8 * b->offset[(size_t)i], b->n_t[(size_t)i], sigma,
                                    b->seed[(size_t)i], 1, stream);
        if (st != CUOPO_OK) return st;
    }
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_set_signal(cuopo_batch *b, const void *src, int on_device, void *stream)
{
    if (!b || !src) return cuopo_fail(CUOPO_EINVAL, "batch_set_signal: NULL argument");
    cuopo_status js = join_groups(b, (cudaStream_t)stream, "batch_set_signal");
    if (js != CUOPO_OK) return js;
    const size_t esz = b->precision == CUOPO_F32 ? 8 : 16;
    cudaError_t e = cudaMemcpyAsync(b->d_signal, src, esz * b->total,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    (cudaStream_t)stream);
    return e == cudaSuccess ? CUOPO_OK : cuda_fail(e, "batch_set_signal");
}

extern "C" cuopo_status cuopo_batch_get_signal(cuopo_batch *b, void *dst, int on_device, void *stream)
{
    if (!b || !dst) return cuopo_fail(CUOPO_EINVAL, "batch_get_signal: NULL argument");
    cuopo_status js = join_groups(b, (cudaStream_t)stream, "batch_get_signal");
    if (js != CUOPO_OK) return js;
    const size_t esz = b->precision == CUOPO_F32 ? 8 : 16;
    cudaError_t e = cudaMemcpyAsync(dst, b->d_signal, esz * b->total,
                                    on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    return e == cudaSuccess ? CUOPO_OK : cuda_fail(e, "batch_get_signal");
}

extern "C" cuopo_status cuopo_batch_reset(cuopo_batch *b, void *stream)
{
    if (!b) return cuopo_fail(CUOPO_EINVAL, "batch_reset: NULL batch");
    cudaStream_t st = (cudaStream_t)stream;
    cuopo_status js = join_groups(b, st, "batch_reset");
    if (js != CUOPO_OK) return js;
    cudaError_t e;
    if ((e = cudaMemsetAsync(b->d_rt, 0, sizeof(int) * b->count, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->d_flag, 0, sizeof(int) * b->count, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->d_calm, 0, sizeof(int) * b->count, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->d_ps, 0, sizeof(double) * b->count, st)) != cudaSuccess)
        return cuda_fail(e, "batch_reset");
    if (b->d_hist) {
        size_t n = 0;
        for (int v : b->n_rt) n += (size_t)v;
        if ((e = cudaMemsetAsync(b->d_hist, 0, sizeof(double) * n, st)) != cudaSuccess)
            return cuda_fail(e, "batch_reset");
    }
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_step(cuopo_batch *b, int chunk, int max_rt, double tol, int patience,
                                         void *stream)
{
    cuopo::Range range_("cuopo_batch_step");
    if (!b || chunk < 1 || max_rt < 1) return cuopo_fail(CUOPO_EINVAL, "batch_step: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaEventRecord(b->fork, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch_step");
    for (BatchGroup &g : b->groups) {
        if ((e = cudaStreamWaitEvent(g.stream, b->fork, 0)) != cudaSuccess) return cuda_fail(e, "batch_step");
        if ((e = cudaMemsetAsync(g.d_queue, 0, sizeof(int), g.stream)) != cudaSuccess)
            return cuda_fail(e, "batch_step");
        LaunchArgs a = base_args(g.plans[0]);
        a.inst = g.d_inst;
        a.n_inst = (int)g.members.size();
        a.queue = g.d_queue;
        a.chunk = chunk;
        a.max_rt = max_rt;
        a.tol = tol;
        a.patience = patience;
        cuopo_status s2 = launch(g.plans[0], a, g.grid, g.stream);
        if (s2 != CUOPO_OK) return s2;
        if ((e = cudaEventRecord(g.done, g.stream)) != cudaSuccess) return cuda_fail(e, "batch_step");
    }
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_run(cuopo_batch *b, int max_rt, double tol, int patience, void *stream)
{
    cuopo_status st = cuopo_batch_reset(b, stream);
    if (st != CUOPO_OK) return st;
    return cuopo_batch_step(b, max_rt, max_rt, tol, patience, stream);
}

extern "C" cuopo_status cuopo_batch_pending(cuopo_batch *b, int *running, void *stream)
{
    if (!b || !running) return cuopo_fail(CUOPO_EINVAL, "batch_pending: NULL argument");
    cuopo_status js = join_groups(b, (cudaStream_t)stream, "batch_pending");
    if (js != CUOPO_OK) return js;
    std::vector<int> f((size_t)b->count);
    cudaError_t e = cudaMemcpyAsync(f.data(), b->d_flag, sizeof(int) * b->count, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch_pending");
    int n = 0;
    for (int v : f) n += (v == 0);
    *running = n;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_results(cuopo_batch *b, double *ps, int *rts, int *flags, void *stream)
{
    if (!b) return cuopo_fail(CUOPO_EINVAL, "batch_results: NULL batch");
    cudaStream_t st = (cudaStream_t)stream;
    cuopo_status js = join_groups(b, st, "batch_results");
    if (js != CUOPO_OK) return js;
    cudaError_t e = cudaSuccess;
    if (ps && (e = cudaMemcpyAsync(ps, b->d_ps, sizeof(double) * b->count, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "batch_results");
    if (rts && (e = cudaMemcpyAsync(rts, b->d_rt, sizeof(int) * b->count, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "batch_results");
    if (flags &&
        (e = cudaMemcpyAsync(flags, b->d_flag, sizeof(int) * b->count, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_fail(e, "batch_results");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "batch_results");
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_batch_history(cuopo_batch *b, int i, double *ps, int n, void *stream)
{
    if (!b || !ps || i < 0 || i >= b->count) return cuopo_fail(CUOPO_EINVAL, "batch_history: bad argument");
    if (b->hist_off[(size_t)i] < 0)
        return cuopo_fail(CUOPO_EINVAL, "batch_history: only nanosecond instances keep a history");
    const int m = std::min(n, b->n_rt[(size_t)i]);
    cudaStream_t st = (cudaStream_t)stream;
    cuopo_status js = join_groups(b, st, "batch_history");
    if (js != CUOPO_OK) return js;
    cudaError_t e = cudaMemcpyAsync(ps, b->d_hist + b->hist_off[(size_t)i], sizeof(double) * (size_t)m,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? CUOPO_OK : cuda_fail(e, "batch_history");
}

/* --------------------------------------------------------------- autotuner */

extern "C" cuopo_status cuopo_autotune(const cuopo_params *base, int precision, int count, int n_rt, int *points_per_cta,
                                       int *cluster, double *ms)
{
    cuopo::Range range_("cuopo_autotune");
    if (!base || count < 1 || n_rt < 1) return cuopo_fail(CUOPO_EINVAL, "autotune: bad argument");
    const int F = base->n_eqs, N = base->n_t;
    std::vector<const KernelEntry *> cand;
    for (const KernelEntry &k : k_kernels)
        if (k.precision == precision && k.F == F && k.M * k.CL == N) cand.push_back(&k);
    if (cand.empty()) return cuopo_fail(CUOPO_EUNSUPPORTED, "autotune: no kernel built for this (precision, n_eqs, n_t)");
    const KernelEntry *best = cand[0];
    double best_ms = -1.0;
    if (cand.size() > 1) {
        if (F != 2 || base->regime != CUOPO_CW)
            return cuopo_fail(CUOPO_EUNSUPPORTED, "autotune: timing runs use CW 2-equation batches");
        /* `count` copies of the base instance, seeded noise, n_rt round trips
         * with the convergence test off (fixed work), per candidate */
        std::vector<cuopo_instance> inst((size_t)count);
        for (int i = 0; i < count; i++) {
            inst[(size_t)i].n_t = N;
            inst[(size_t)i].ap0 = base->ap0;
            inst[(size_t)i].Rs = base->Rs;
            inst[(size_t)i].delta = base->delta;
            inst[(size_t)i].gdd = base->gdd;
            inst[(size_t)i].seed = (uint64_t)i;
        }
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaError_t e;
        if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) {
            if (e0) cudaEventDestroy(e0);
            return cuda_fail(e, "autotune");
        }
        cuopo_status st = CUOPO_OK;
        for (const KernelEntry *k : cand) {
            g_force = k;
            cuopo_batch *b = nullptr;
            st = cuopo_batch_create(&b, base, inst.data(), count, precision);
            if (st == CUOPO_OK) st = cuopo_batch_seed_noise(b, 1e-15, nullptr);
            if (st == CUOPO_OK) st = cuopo_batch_run(b, 1, 0.0, 1, nullptr); /* warm-up: module load, tables */
            /* best of two timed runs */
            float t = -1.f;
            for (int rep = 0; rep < 2 && st == CUOPO_OK; rep++) {
                float ti = 0.f;
                if ((st = cuopo_batch_reset(b, nullptr)) != CUOPO_OK) break;
                cudaEventRecord(e0, nullptr);
                st = cuopo_batch_step(b, n_rt, n_rt, 0.0, 1, nullptr);
                if (st == CUOPO_OK) st = cuopo_batch_wait(b, nullptr);
                cudaEventRecord(e1, nullptr);
                if (st == CUOPO_OK && (e = cudaEventSynchronize(e1)) != cudaSuccess) st = cuda_fail(e, "autotune");
                if (st == CUOPO_OK) cudaEventElapsedTime(&ti, e0, e1);
                if (t < 0.f || ti < t) t = ti;
            }
            g_force = nullptr;
            if (b) cuopo_batch_destroy(b);
            if (st != CUOPO_OK) break;
            /* the built-in choice (first candidate) stays unless another is
             * faster by more than the run-to-run noise of such timings */
            if (best_ms < 0.0 || t < 0.97 * best_ms) {
                best_ms = t;
                best = k;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != CUOPO_OK) return st;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        bool found = false;
        for (TunedChoice &c : g_tuned)
            if (c.precision == precision && c.F == F && c.N == N) {
                c.k = best;
                found = true;
            }
        if (!found) g_tuned.push_back(TunedChoice{precision, F, N, best});
    }
    if (points_per_cta) *points_per_cta = best->M;
    if (cluster) *cluster = best->CL;
    if (ms) *ms = best_ms;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_kernel_select(int precision, int n_eqs, int n_t, int points_per_cta, int cluster)
{
    for (const KernelEntry &k : k_kernels)
        if (k.precision == precision && k.F == n_eqs && k.M == points_per_cta && k.CL == cluster &&
            k.M * k.CL == n_t) {
            std::lock_guard<std::mutex> lock(g_tune_mu);
            for (TunedChoice &c : g_tuned)
                if (c.precision == precision && c.F == n_eqs && c.N == n_t) {
                    c.k = &k;
                    return CUOPO_OK;
                }
            g_tuned.push_back(TunedChoice{precision, n_eqs, n_t, &k});
            return CUOPO_OK;
        }
    return cuopo_fail(CUOPO_EUNSUPPORTED, "kernel_select: no such built configuration");
}

extern "C" cuopo_status cuopo_autotune_reset(void)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned.clear();
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_kernel_config(int precision, int n_eqs, int n_t, int *points_per_cta, int *cluster)
{
    const KernelEntry *k = find_kernel(precision, n_eqs, n_t);
    if (!k) return cuopo_fail(CUOPO_EUNSUPPORTED, "kernel_config: no kernel built for this (precision, n_eqs, n_t)");
    if (points_per_cta) *points_per_cta = k->M;
    if (cluster) *cluster = k->CL;
    return CUOPO_OK;
}

/* ------------------------------------------------- allocation-free pass */

/*
 * cuopo_crystal_pass_noalloc: one crystal pass for callers that must not
 * allocate device memory -- processes whose device memory is owned by
 * another allocator or budget, or plugins loaded into such processes.  Its
 * tables live in the file-scope array below (every GPU that loads the
 * library holds it until exit); the host side builds them in a static host
 * buffer and uploads them with cudaMemcpyAsync (a pageable source: the
 * copy has left the buffer when the call returns, so the next call may
 * overwrite it).  The array is shared by every call, so calls that overlap
 * on the GPU (different streams, or different host threads without
 * ordering) race; calls ordered on one stream do not.  The array's device
 * address is looked up once per device and kept, so the library must not
 * be used across a cudaDeviceReset of that device.
 */
#define CUOPO_NOALLOC_BYTES (384u * 1024u)
#define CUOPO_NOALLOC_MAX_N 8192
#define CUOPO_NOALLOC_MAX_NZ 1024
#define CUOPO_NOALLOC_MAX_DEV 64

static __device__ __align__(256) unsigned char g_noalloc_scratch[CUOPO_NOALLOC_BYTES];
static unsigned char g_noalloc_host[CUOPO_NOALLOC_BYTES];
static void *g_noalloc_dev[CUOPO_NOALLOC_MAX_DEV];
static std::mutex g_noalloc_mu;

extern "C" cuopo_status cuopo_crystal_pass_noalloc(const cuopo_params *p, const float *w_host, void *Ap, void *As,
                                                   void *Ai, void *stream)
{
    if (!p || !Ap || !As || (p->n_eqs == 3 && !Ai)) return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: NULL argument");
    if (p->n_eqs != 2 && p->n_eqs != 3) return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: n_eqs must be 2 or 3");
    if (!is_pow2i(p->n_t) || p->n_t < 512 || p->n_t > CUOPO_NOALLOC_MAX_N)
        return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: n_t must be a power of 2 in [512, 8192] "
                                        "(its tables live in a fixed 384 KiB device array)");
    if (p->n_z < 1 || p->n_z > CUOPO_NOALLOC_MAX_NZ)
        return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: n_z must be in [1, 1024]");
    const KernelEntry *k = find_kernel(CUOPO_F32, p->n_eqs, p->n_t, true);
    if (!k) return cuopo_fail(CUOPO_EUNSUPPORTED, "crystal_pass_noalloc: no single-CTA kernel for n_t");
    const int N = p->n_t, F = p->n_eqs, nco = (F == 2) ? 6 : 3;

    /* layout of the scratch array (bytes, 256-aligned pieces) */
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_disp = 0;
    const size_t o_rk = o_disp + up(sizeof(float2) * (size_t)F * N);
    const size_t o_w = o_rk + up(sizeof(float2) * (size_t)(p->n_z + 1) * nco);
    const size_t o_fu = o_w + up(sizeof(float) * (size_t)N);
    const size_t o_fc = o_fu + up(sizeof(double2) * NFRAME);
    const size_t o_st = o_fc + up(sizeof(float2) * 3 * NFRAME);
    const size_t total = o_st + 256;
    if (total > CUOPO_NOALLOC_BYTES) return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: tables exceed 384 KiB");

    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "crystal_pass_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= CUOPO_NOALLOC_MAX_DEV) return cuopo_fail(CUOPO_EUNSUPPORTED, "crystal_pass_noalloc: device index");
    if (!g_noalloc_dev[dev]) {
        /* once per device, with that device current: the array's device address */
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return cuda_fail(e, "crystal_pass_noalloc: cudaGetSymbolAddress");
        g_noalloc_dev[dev] = ptr;
    }
    unsigned char *H = g_noalloc_host;
    unsigned char *D = (unsigned char *)g_noalloc_dev[dev];

    /* grid w (reference linspace/fftshift unless given) */
    float *w = (float *)(H + o_w);
    if (w_host) std::memcpy(w, w_host, sizeof(float) * N);
    else {
        if (p->t_rt <= 0) return cuopo_fail(CUOPO_EINVAL, "crystal_pass_noalloc: t_rt must be > 0 when w is not given");
        /* cuOPO.cu:151,183-189 without a temporary: F[i] = linspace(-N dF/2, N dF/2), w = 2 pi fftshift(F) */
        const float trt = (float)p->t_rt, dF = 1 / trt;
        const float lo = (float)(-0.5 * (double)(unsigned)N * (double)dF);
        const float hi = (float)(+0.5 * (double)(unsigned)N * (double)dF);
        const float span = hi - lo, den = (float)(N - 1);
        const float twopi = 2 * (float)3.14159265358979323846;
        for (int i = 0; i < N; i++) {
            const int src = (i < N / 2) ? i + N / 2 : i - N / 2;
            w[i] = twopi * (lo + (float)src * span / den);
        }
    }
    /* dispersion rows (1 + d form), as in the plan's tables */
    float2 *Dt = (float2 *)(H + o_disp);
    double gvm[3], b2[3], b3[3], al[3];
    if (F == 2) { gvm[0] = 1.0 / p->vp - 1.0 / p->vs; gvm[1] = 0.0; }
    else { gvm[0] = 1.0 / p->vp - 1.0 / p->vi; gvm[1] = 0.0; gvm[2] = 1.0 / p->vi - 1.0 / p->vs; }
    b2[0] = p->b2p; b2[1] = p->b2s; b2[2] = p->b2i;
    b3[0] = p->b3p; b3[1] = p->b3s; b3[2] = p->b3i;
    al[0] = p->alpha_crp; al[1] = p->alpha_crs; al[2] = p->alpha_cri;
    for (int f = 0; f < F; f++) {
        const double a = std::exp(-0.5 * al[f] * p->dz);
        for (int q = 0; q < N; q++) {
            const double wk = (double)w[q];
            const double ph = p->dz * wk * (gvm[f] + 0.5 * wk * b2[f] + wk * wk * b3[f] / 6.0);
            const double dre = (ph == 0.0) ? a - 1.0 : a * std::cos(ph) - 1.0;
            Dt[(size_t)f * N + q] = make_float2((float)dre, (float)(a * std::sin(ph)));
        }
    }
    /* RK4 stage coefficients (z accumulated in float, as the reference) */
    float2 *co = (float2 *)(H + o_rk);
    std::memset(co, 0, sizeof(float2) * (size_t)(p->n_z + 1) * nco);
    const double h6 = (double)(float)((float)p->dz / 2) / 6.0;
    float z = 0;
    const float dzf = (float)p->dz;
    for (int s = 0; s < p->n_z; s++) {
        const double zj[3] = {(double)z, (double)(float)(z + dzf / 4), (double)(float)(z + dzf / 2)};
        if (F == 2) {
            for (int j = 0; j < 3; j++) {
                const double ph = p->dk * zj[j], c = std::cos(ph), sn = std::sin(ph);
                co[s * 6 + 2 * j + 0] = make_float2((float)(-p->kp * sn), (float)(p->kp * c));
                co[s * 6 + 2 * j + 1] = make_float2((float)(p->ks * sn), (float)(p->ks * c));
            }
        } else {
            double er = 0, ei = 0;
            const double wgt[3] = {1.0, 4.0, 1.0};
            for (int j = 0; j < 3; j++) {
                er += wgt[j] * std::cos(p->dk * zj[j]);
                ei += wgt[j] * std::sin(p->dk * zj[j]);
            }
            const double kap[3] = {p->kp, p->ks, p->ki};
            for (int f = 0; f < 3; f++) {
                const double si = (f == 0) ? -ei : ei;
                co[s * 3 + f] = make_float2((float)(h6 * kap[f] * -si), (float)(h6 * kap[f] * er));
            }
        }
        z += dzf;
    }
    /* random frame table (same fixed sequence as the plans') */
    double2 *fu = (double2 *)(H + o_fu);
    float2 *fc = (float2 *)(H + o_fc);
    unsigned long long rs = 0x2545F4914F6CDD1Dull;
    for (int q = 0; q < NFRAME; q++) {
        double u[2];
        for (int j = 0; j < 2; j++) {
            rs += 0x9E3779B97F4A7C15ull;
            unsigned long long x = rs;
            x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
            x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
            u[j] = 0.25 * ((double)((x ^ (x >> 31)) >> 11) * (1.0 / 9007199254740992.0)) - 0.125;
        }
        fu[q] = make_double2(u[0], u[1]);
        const double upump = (F == 2) ? 2.0 * u[0] : u[0] + u[1];
        const double ang[3] = {2.0 * M_PI * upump, 2.0 * M_PI * u[0], 2.0 * M_PI * u[1]};
        for (int f = 0; f < 3; f++) fc[3 * q + f] = make_float2((float)std::tan(0.5 * ang[f]), (float)std::sin(ang[f]));
    }

    cudaStream_t st = (cudaStream_t)stream;
    if ((e = cudaMemcpyAsync(D, H, o_st, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(D + o_st, 0, sizeof(int), st)) != cudaSuccess)
        return cuda_fail(e, "crystal_pass_noalloc: table upload");

    LaunchArgs a;
    std::memset(&a, 0, sizeof(a));
    a.tab.disp = D + o_disp;
    a.tab.rk = D + o_rk;
    a.tab.eom = nullptr;
    a.tab.w = (const float *)(D + o_w);
    a.tab.twN = nullptr;
    a.tab.frame_u = (const double2 *)(D + o_fu);
    a.tab.frame_c = D + o_fc;
    a.tab.h6 = h6;
    a.tab.inv_n = 1.0 / (double)N;
    a.n_z = p->n_z;
    a.regime = p->regime;
    a.pass_only = 1;
    a.status = (int *)(D + o_st);
    a.single.Ap = Ap;
    a.single.As = As;
    a.single.Ai = Ai;
    a.single.rt_count = 1;
    e = k->fn(a, 1, st);
    if (e != cudaSuccess) return cuda_fail(e, "crystal_pass_noalloc: kernel launch");
    return CUOPO_OK;
}
