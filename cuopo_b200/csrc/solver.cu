/*
 * solver.cu -- plans, table construction and the GPU entry points of the
 * C ABI (include/cuopo.h).
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cuopo.h"
#include "internal.h"
#include "ssfm.cuh"

using namespace cuopo;

struct cuopo_plan {
    cuopo_params p;
    int precision;
    int F;            /* number of fields */
    int N;            /* grid points */
    int threads;      /* CTA size */
    int cluster;      /* CTAs per instance */
    size_t smem;      /* dynamic shared memory per CTA */
    void *d_disp;     /* [F][N] */
    void *d_rk;       /* [(n_z+1)][NCO] */
    void *d_eom;      /* [N] or NULL */
    float *d_w;       /* [N] */
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

typedef cudaError_t (*launch_fn)(const LaunchArgs &, int grid, cudaStream_t);

template <typename R, int F, int M, bool INPLACE>
static cudaError_t launch_impl(const LaunchArgs &a, int grid, cudaStream_t st)
{
    using K = Ssfm<R, F, M, INPLACE>;
    const size_t smem = K::smem_bytes();
    static bool attr_done = false;  /* per-instantiation, set on first use */
    if (!attr_done) {
        cudaError_t e = cudaFuncSetAttribute(ssfm_kernel<R, F, M, INPLACE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    ssfm_kernel<R, F, M, INPLACE><<<grid, K::T, smem, st>>>(a);
    return cudaGetLastError();
}

struct KernelEntry {
    int precision, F, M;
    bool inplace;
    size_t smem;
    launch_fn fn;
};

#define CUOPO_K(R, PREC, F, M, IP) \
    {PREC, F, M, IP, Ssfm<R, F, M, IP>::smem_bytes(), &launch_impl<R, F, M, IP>}

static const KernelEntry k_kernels[] = {
    CUOPO_K(float, CUOPO_F32, 2, 512, false),
    CUOPO_K(float, CUOPO_F32, 2, 1024, false),
    CUOPO_K(float, CUOPO_F32, 2, 2048, false),
    CUOPO_K(float, CUOPO_F32, 2, 4096, false),
    CUOPO_K(float, CUOPO_F32, 2, 8192, false),
    CUOPO_K(float, CUOPO_F32, 3, 512, false),
    CUOPO_K(float, CUOPO_F32, 3, 1024, false),
    CUOPO_K(float, CUOPO_F32, 3, 2048, false),
    CUOPO_K(float, CUOPO_F32, 3, 4096, false),
    CUOPO_K(float, CUOPO_F32, 3, 8192, true),
    CUOPO_K(double, CUOPO_F64, 2, 512, false),
    CUOPO_K(double, CUOPO_F64, 2, 1024, false),
    CUOPO_K(double, CUOPO_F64, 2, 2048, false),
    CUOPO_K(double, CUOPO_F64, 2, 4096, false),
    CUOPO_K(double, CUOPO_F64, 3, 512, false),
    CUOPO_K(double, CUOPO_F64, 3, 1024, false),
    CUOPO_K(double, CUOPO_F64, 3, 2048, false),
    CUOPO_K(double, CUOPO_F64, 3, 4096, true),
};

static const KernelEntry *find_kernel(int precision, int F, int N)
{
    for (const KernelEntry &k : k_kernels)
        if (k.precision == precision && k.F == F && k.M == N) return &k;
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

template <typename R>
static std::vector<unsigned char> build_tables(const cuopo_params &p, const float *w, const float *T,
                                               std::vector<unsigned char> &rk_out,
                                               std::vector<unsigned char> &eom_out, double &h6)
{
    using C = cpx<R>;
    const int N = p.n_t;
    const int F = p.n_eqs;
    /* LinearOperator, cwes2.cuh:103-121 / cwes3.cuh:107-128: per field the
     * group-velocity term (Q4), GVD, TOD, attenuation exp(-alpha dz/2),
     * and CUFFTscale's 1/N (functions.cuh:126-135). */
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
    for (int f = 0; f < F; f++) {
        const double att = std::exp(-0.5 * al[f] * z) / (double)N;
        for (int k = 0; k < N; k++) {
            const double wk = (double)w[k];
            const double ph = z * wk * (gvm[f] + 0.5 * wk * b2[f] + wk * wk * b3[f] / 6.0);
            D[(size_t)f * N + k] = mk<C>((R)(std::cos(ph) * att), (R)(std::sin(ph) * att));
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
                const double c = std::cos(ph), sn = std::sin(ph);
                co[s * 6 + 2 * j + 0] = mk<C>((R)(-p.kp * sn), (R)(p.kp * c));
                co[s * 6 + 2 * j + 1] = mk<C>((R)(p.ks * sn), (R)(p.ks * c));
            }
        } else {
            /* dAdz, cwes3.cuh:37-39 with k2 = k3 (Q3): the half step is
             * A += (h/6) i kappa (E(z) + 4 E(z+dz/4) + E(z+dz/2)) P. */
            double er = 0, ei = 0;
            const double wgt[3] = {1.0, 4.0, 1.0};
            for (int j = 0; j < 3; j++) {
                const double ph = p.dk * zs[3 * s + j];
                er += wgt[j] * std::cos(ph);
                ei += wgt[j] * std::sin(ph);
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
            const double ph = p.mod_depth * std::sin(2.0 * M_PI * p.fpm * (double)T[k]);
            E[k] = mk<C>((R)std::cos(ph), (R)std::sin(ph));
        }
    }
    return disp;
}

extern "C" cuopo_status cuopo_plan_create(cuopo_plan **out, const cuopo_params *p,
                                          const float *w_host, const float *T_host, int precision)
{
    if (!out || !p) return cuopo_fail(CUOPO_EINVAL, "plan_create: NULL argument");
    *out = nullptr;
    if (p->n_eqs != 2 && p->n_eqs != 3) return cuopo_fail(CUOPO_EINVAL, "n_eqs must be 2 or 3");
    if (!is_pow2i(p->n_t)) return cuopo_fail(CUOPO_EINVAL, "n_t must be a power of 2");
    if (p->n_z < 1) return cuopo_fail(CUOPO_EINVAL, "n_z must be >= 1");
    if (precision != CUOPO_F32 && precision != CUOPO_F64)
        return cuopo_fail(CUOPO_EINVAL, "precision must be CUOPO_F32 or CUOPO_F64");
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

    std::vector<unsigned char> disp, rk, eom;
    double h6 = 0;
    if (precision == CUOPO_F32) disp = build_tables<float>(*p, w.data(), T.data(), rk, eom, h6);
    else disp = build_tables<double>(*p, w.data(), T.data(), rk, eom, h6);

    cuopo_plan *pl = new (std::nothrow) cuopo_plan();
    if (!pl) return cuopo_fail(CUOPO_ENOMEM, "plan_create: out of host memory");
    pl->p = *p;
    pl->precision = precision;
    pl->F = p->n_eqs;
    pl->N = p->n_t;
    pl->threads = k->M / 16;
    pl->cluster = 1;
    pl->smem = k->smem;
    pl->h6 = h6;
    cudaError_t e;
    if ((e = cudaMalloc(&pl->d_disp, disp.size())) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_rk, rk.size())) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_w, sizeof(float) * p->n_t)) != cudaSuccess ||
        (e = cudaMalloc(&pl->d_status, sizeof(int))) != cudaSuccess ||
        (!eom.empty() && (e = cudaMalloc(&pl->d_eom, eom.size())) != cudaSuccess)) {
        cuopo_plan_destroy(pl);
        return e == cudaErrorMemoryAllocation ? cuopo_fail(CUOPO_ENOMEM, "plan_create: device allocation failed")
                                              : cuda_fail(e, "plan_create: cudaMalloc");
    }
    if ((e = cudaMemcpy(pl->d_disp, disp.data(), disp.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(pl->d_rk, rk.data(), rk.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(pl->d_w, w.data(), sizeof(float) * p->n_t, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(pl->d_status, 0, sizeof(int))) != cudaSuccess ||
        (!eom.empty() && (e = cudaMemcpy(pl->d_eom, eom.data(), eom.size(), cudaMemcpyHostToDevice)) != cudaSuccess)) {
        cuopo_plan_destroy(pl);
        return cuda_fail(e, "plan_create: upload");
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
    a.tab.h6 = pl->h6;
    a.tab.inv_n = 1.0 / (double)pl->N;
    a.n_z = pl->p.n_z;
    a.regime = pl->p.regime;
    a.use_eom = pl->p.use_eom && pl->d_eom != nullptr;
    a.eom_idler = pl->p.eom_idler;
    a.status = pl->d_status;
    return a;
}

static void cavity_factors(const cuopo_params &p, Instance &I)
{
    /* AddPhase: sqrt(R) * exp(i pi delta), functions.cuh:145 */
    const double ph = M_PI * p.delta;
    const double rs = std::sqrt(p.Rs), ri = std::sqrt(p.Ri);
    I.phase_s[0] = rs * std::cos(ph);
    I.phase_s[1] = rs * std::sin(ph);
    I.phase_i[0] = ri * std::cos(ph);
    I.phase_i[1] = ri * std::sin(ph);
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
    cavity_factors(pl->p, I);
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
