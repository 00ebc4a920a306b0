/*
 * cuopo -- drop-in replacement of the reference executable (src/cuOPO.cu).
 *
 * Same 12 positional arguments as the reference (src/cuOPO.sh:159, parsed at
 * src/cuOPO.cu:92-267):
 *
 *   cuopo [options] lp_nm temp lambda_um N R_percent delta eps_percent
 *         tod_percent use_eom mod_depth freq_det lcr_mm
 *
 * and the same output files in the working directory (src/cuOPO.cu:273-286,
 * 620-635; format src/headers/files.cuh:21-62, one value per line, 20
 * significant digits): pump_input_{r,i}.dat, signal_input_{r,i}.dat,
 * idler_input_{r,i}.dat (3 equations), Tp.dat, freq.dat, T.dat,
 * signal_output_{r,i}.dat, pump_output_{r,i}.dat, idler_output_{r,i}.dat.
 *
 * The reference selects regime, model and crystal at compile time
 * (-DCW_OPO / -DNS_OPO, -DTHREE_EQS, -DPPLN / -DSPPLT) and fixes SIZE, NZ and
 * NRT in the source (cuOPO.cu:28-30).  The same -D switches (and -DSIZE=,
 * -DNZ=, -DNRT=) set this program's defaults; the options below override
 * them at run time:
 *
 *   --cw | --ns              regime
 *   --two-eqs | --three-eqs  coupled-wave model
 *   --ppln | --spplt         crystal
 *   --n-t N --n-z NZ --n-rt NRT
 *   --ls-nm X                signal wavelength (default 2 lp, cuOPO.cu:93)
 *   --seed S                 noise seed (default: clock, like cuOPO.cu's
 *                            NoiseGeneratorCPU, functions.cuh:58-71); printed
 *   --signal-input PREFIX    read the initial signal from PREFIX_{r,i}.dat
 *   --idler-input PREFIX     read the initial idler from PREFIX_{r,i}.dat
 *   --f64                    FP64 fields (default FP32 like the reference)
 *   --format dat|bin         bin: raw little-endian float32 (<name>.f32) and
 *                            interleaved complex64 (<name>.c64) instead of text
 *   --outdir DIR             write the files there (default: working directory)
 *   --setup-only             write the inputs and grids, run nothing on the GPU
 *   --quiet                  no parameter report
 *
 * Exit status: 0 on success, 2 on bad arguments, 1 on a library or CUDA error.
 */
#include <cuda_runtime_api.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cuopo.h"

#ifndef SIZE
#define SIZE (1 << 14)
#endif
#ifndef NZ
#define NZ 150
#endif
#ifndef NRT
#define NRT 10000
#endif

namespace {

struct Options {
    cuopo_inputs in;
    unsigned long long seed = 0;
    bool seed_given = false;
    std::string signal_input, idler_input, outdir, format = "dat";
    int precision = CUOPO_F32;
    bool setup_only = false, quiet = false;
};

[[noreturn]] void usage(const char *msg)
{
    if (msg) std::fprintf(stderr, "cuopo: %s\n", msg);
    std::fprintf(stderr,
                 "usage: cuopo [--cw|--ns] [--two-eqs|--three-eqs] [--ppln|--spplt] [--n-t N] [--n-z NZ]\n"
                 "             [--n-rt NRT] [--ls-nm X] [--seed S] [--signal-input PREFIX] [--idler-input PREFIX]\n"
                 "             [--f64] [--format dat|bin] [--outdir DIR] [--setup-only] [--quiet]\n"
                 "             lp_nm temp lambda_um N R_percent delta eps_percent tod_percent use_eom\n"
                 "             mod_depth freq_det lcr_mm\n");
    std::exit(2);
}

double num(const char *s, const char *what)
{
    char *end = nullptr;
    const double v = std::strtod(s, &end);
    if (end == s || *end != '\0') {
        std::fprintf(stderr, "cuopo: %s: not a number: '%s'\n", what, s);
        std::exit(2);
    }
    return v;
}

long inum(const char *s, const char *what)
{
    char *end = nullptr;
    const long v = std::strtol(s, &end, 10);
    if (end == s || *end != '\0') {
        std::fprintf(stderr, "cuopo: %s: not an integer: '%s'\n", what, s);
        std::exit(2);
    }
    return v;
}

Options parse(int argc, char **argv)
{
    Options o;
    cuopo_inputs_default(&o.in);
#if defined(NS_OPO)
    o.in.regime = CUOPO_NS;
#else
    o.in.regime = CUOPO_CW;
#endif
#if defined(THREE_EQS)
    o.in.n_eqs = 3;
#else
    o.in.n_eqs = 2;
#endif
#if defined(SPPLT)
    o.in.crystal = CUOPO_SPPLT;
#else
    o.in.crystal = CUOPO_PPLN;
#endif
    o.in.n_t = SIZE;
    o.in.n_z = NZ;
    o.in.n_rt = NRT;
    std::vector<const char *> pos;
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        auto val = [&](const char *name) -> const char * {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "cuopo: %s needs a value\n", name);
                std::exit(2);
            }
            return argv[++i];
        };
        if (!std::strcmp(a, "--cw")) o.in.regime = CUOPO_CW;
        else if (!std::strcmp(a, "--ns")) o.in.regime = CUOPO_NS;
        else if (!std::strcmp(a, "--two-eqs")) o.in.n_eqs = 2;
        else if (!std::strcmp(a, "--three-eqs")) o.in.n_eqs = 3;
        else if (!std::strcmp(a, "--ppln")) o.in.crystal = CUOPO_PPLN;
        else if (!std::strcmp(a, "--spplt")) o.in.crystal = CUOPO_SPPLT;
        else if (!std::strcmp(a, "--n-t")) o.in.n_t = (int)inum(val(a), a);
        else if (!std::strcmp(a, "--n-z")) o.in.n_z = (int)inum(val(a), a);
        else if (!std::strcmp(a, "--n-rt")) o.in.n_rt = (int)inum(val(a), a);
        else if (!std::strcmp(a, "--ls-nm")) o.in.ls_nm = num(val(a), a);
        else if (!std::strcmp(a, "--seed")) {
            o.seed = (unsigned long long)inum(val(a), a);
            o.seed_given = true;
        } else if (!std::strcmp(a, "--signal-input")) o.signal_input = val(a);
        else if (!std::strcmp(a, "--idler-input")) o.idler_input = val(a);
        else if (!std::strcmp(a, "--f64")) o.precision = CUOPO_F64;
        else if (!std::strcmp(a, "--format")) {
            o.format = val(a);
            if (o.format != "dat" && o.format != "bin") usage("--format must be dat or bin");
        } else if (!std::strcmp(a, "--outdir")) o.outdir = val(a);
        else if (!std::strcmp(a, "--setup-only")) o.setup_only = true;
        else if (!std::strcmp(a, "--quiet")) o.quiet = true;
        else if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) usage(nullptr);
        else if (a[0] == '-' && a[1] == '-') usage((std::string("unknown option ") + a).c_str());
        else pos.push_back(a);
    }
    if (pos.size() != 12) usage("expected 12 positional arguments");
    /* src/cuOPO.cu:92-267: argv[1] .. argv[12] */
    o.in.lp_nm = num(pos[0], "lp_nm");
    o.in.temp_c = num(pos[1], "temp");
    o.in.lambda_um = num(pos[2], "lambda_um");
    o.in.n_thr = num(pos[3], "N");
    o.in.r_percent = num(pos[4], "R_percent");
    o.in.delta = num(pos[5], "delta");
    o.in.gdd_percent = num(pos[6], "eps_percent");
    o.in.tod_percent = num(pos[7], "tod_percent");
    o.in.use_eom = (int)inum(pos[8], "use_eom");
    o.in.mod_depth_pi = num(pos[9], "mod_depth");
    o.in.freq_det_mhz = num(pos[10], "freq_det");
    o.in.lcr_mm = num(pos[11], "lcr_mm");
    if (o.in.n_rt < 1) usage("--n-rt must be >= 1");
    if (!o.seed_given)
        o.seed = (unsigned long long)std::chrono::system_clock::now().time_since_epoch().count();
    return o;
}

int fail_lib(const char *what)
{
    std::fprintf(stderr, "cuopo: %s: %s\n", what, cuopo_last_error());
    return 1;
}

int fail_cuda(const char *what, cudaError_t e)
{
    std::fprintf(stderr, "cuopo: %s: %s\n", what, cudaGetErrorString(e));
    return 1;
}

std::string path(const Options &o, const std::string &name)
{
    return o.outdir.empty() ? name : o.outdir + "/" + name;
}

bool write_raw(const std::string &p, const void *v, size_t bytes)
{
    FILE *f = std::fopen(p.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

/* Real vector: <name>.dat (SaveVectorReal, files.cuh:21-32) or <name>.f32. */
int save_real(const Options &o, const char *name, const float *v, long n)
{
    if (o.format == "bin") {
        if (!write_raw(path(o, std::string(name) + ".f32"), v, sizeof(float) * (size_t)n)) {
            std::fprintf(stderr, "cuopo: cannot write %s.f32\n", name);
            return 1;
        }
        return 0;
    }
    if (cuopo_write_dat_real(path(o, std::string(name) + ".dat").c_str(), v, n) != CUOPO_OK)
        return fail_lib(name);
    return 0;
}

/* Complex vector: <name>_r.dat/<name>_i.dat (SaveVectorComplex,
 * files.cuh:47-62) or <name>.c64. */
int save_complex(const Options &o, const char *name, const float *v, long n)
{
    if (o.format == "bin") {
        if (!write_raw(path(o, std::string(name) + ".c64"), v, 2 * sizeof(float) * (size_t)n)) {
            std::fprintf(stderr, "cuopo: cannot write %s.c64\n", name);
            return 1;
        }
        return 0;
    }
    if (cuopo_write_dat_complex(path(o, name).c_str(), v, n) != CUOPO_OK) return fail_lib(name);
    return 0;
}

/* Device buffers of the run, freed on every exit path. */
struct Device {
    std::vector<void *> ptrs;
    cuopo_plan *plan = nullptr;
    ~Device()
    {
        if (plan) cuopo_plan_destroy(plan);
        for (void *p : ptrs) cudaFree(p);
    }
    cudaError_t alloc(void **p, size_t bytes)
    {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) {
            ptrs.push_back(*p);
            e = cudaMemset(*p, 0, bytes);
        }
        return e;
    }
};

/* float complex host vector -> field precision on the device */
cudaError_t upload(void *dst, const std::vector<float> &h, int precision)
{
    if (precision == CUOPO_F32) return cudaMemcpy(dst, h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice);
    std::vector<double> d(h.begin(), h.end());
    return cudaMemcpy(dst, d.data(), sizeof(double) * d.size(), cudaMemcpyHostToDevice);
}

cudaError_t download(std::vector<float> &h, const void *src, int precision)
{
    if (precision == CUOPO_F32) return cudaMemcpy(h.data(), src, sizeof(float) * h.size(), cudaMemcpyDeviceToHost);
    std::vector<double> d(h.size());
    cudaError_t e = cudaMemcpy(d.data(), src, sizeof(double) * d.size(), cudaMemcpyDeviceToHost);
    for (size_t k = 0; k < d.size(); k++) h[k] = (float)d[k];
    return e;
}

}  // namespace

int main(int argc, char **argv)
{
    const auto t0 = std::chrono::steady_clock::now();
    Options o = parse(argc, argv);
    const cuopo_inputs &in = o.in;

    cuopo_params prm;
    cuopo_info info;
    if (cuopo_derive_params(&in, &prm, &info) != CUOPO_OK) return fail_lib("parameters");

    const int three = prm.n_eqs == 3;
    const int ns_regime = prm.regime == CUOPO_NS;
    const long n = prm.n_t;
    const unsigned n_rt = (unsigned)in.n_rt;
    /* cuOPO.cu:154-166: CW saves the last Nrts = 64 round trips, NS all */
    const unsigned nrts = 64;
    const long sizel = ns_regime ? n * (long)n_rt : n * (long)nrts;
    const float t_rt = (float)prm.t_rt;
    const float t_width = ns_regime ? t_rt * (float)n_rt : t_rt * (float)nrts;

    if (!o.quiet) {
        std::printf("Regime: %s\n%s equations\n", ns_regime ? "nanosecond" : "continuous wave", three ? "Three" : "Two");
        std::printf("Crystal: %s\n", in.crystal == CUOPO_SPPLT ? "MgO:sPPLT" : "MgO:PPLN");
        std::printf("Number of round trips   = %u\n", n_rt);
        std::printf("Grid points (SIZE)      = %ld\nSlices (NZ)             = %d\n", n, prm.n_z);
        std::printf("Temp                    = %.6g C\n", info.temp_c);
        std::printf("np, ns                  = %.8g, %.8g\n", info.np, info.ns);
        std::printf("dk                      = %.8g 1/um\n", prm.dk);
        std::printf("t_rt                    = %.8g ps\n", prm.t_rt);
        std::printf("GDD                     = %.8g ps^2\n", prm.gdd);
        std::printf("Pump power / threshold  = %.6g (Ap0 = %.8g V/um)\n", in.n_thr, prm.ap0);
        std::printf("Noise seed              = %llu\n", (unsigned long long)o.seed);
        std::fflush(stdout);
    }

    /* grids (cuOPO.cu:169-189) */
    std::vector<float> T(n), w(n), Tp(sizel), Fp(sizel);
    if (cuopo_make_grids((int)n, prm.t_rt, T.data(), w.data()) != CUOPO_OK) return fail_lib("grids");
    cuopo_linspace(Tp.data(), sizel, (float)(-0.5 * (double)t_width), (float)(0.5 * (double)t_width));
    const float dFp = 1 / t_width;
    cuopo_linspace(Fp.data(), sizel, (float)(-0.5 * (double)sizel * (double)dFp),
                   (float)(+0.5 * (double)sizel * (double)dFp));

    /* inputs (cuOPO.cu:237-258): pump, noise signal/idler */
    const long n_pump = ns_regime ? sizel : n;
    std::vector<float> pump(2 * n_pump), As0(2 * n), Ai0(three ? 2 * n : 0);
    if (ns_regime) {
        if (cuopo_pump_ns(pump.data(), (int)n, (int)n_rt, prm.t_rt, prm.ap0, in.fwhm_ps) != CUOPO_OK)
            return fail_lib("pump");
    } else if (cuopo_pump_cw(pump.data(), (int)n, prm.ap0) != CUOPO_OK) {
        return fail_lib("pump");
    }
    const double sigma = 1.0e-15; /* functions.cuh:62 */
    if (!o.signal_input.empty()) {
        if (cuopo_read_dat_complex(o.signal_input.c_str(), As0.data(), n) != CUOPO_OK) return fail_lib("signal input");
    } else if (cuopo_noise_host(As0.data(), n, sigma, o.seed, 1) != CUOPO_OK) {
        return fail_lib("noise");
    }
    if (three) {
        if (!o.idler_input.empty()) {
            if (cuopo_read_dat_complex(o.idler_input.c_str(), Ai0.data(), n) != CUOPO_OK) return fail_lib("idler input");
        } else if (cuopo_noise_host(Ai0.data(), n, sigma, o.seed, 2) != CUOPO_OK) {
            return fail_lib("noise");
        }
    }
    /* cuOPO.cu:273-285 */
    if (save_complex(o, "pump_input", pump.data(), n_pump) || save_complex(o, "signal_input", As0.data(), n) ||
        (three && save_complex(o, "idler_input", Ai0.data(), n)))
        return 1;
    if (o.setup_only) {
        if (save_real(o, "Tp", Tp.data(), sizel) || save_real(o, "freq", Fp.data(), sizel) ||
            save_real(o, "T", T.data(), n))
            return 1;
        return 0;
    }

    /* device state (cuOPO.cu:384-442) */
    const size_t es = o.precision == CUOPO_F64 ? 2 * sizeof(double) : 2 * sizeof(float);
    Device d;
    void *Ap = nullptr, *As = nullptr, *Ai = nullptr, *pin = nullptr, *svp = nullptr, *svs = nullptr, *svi = nullptr;
    cudaError_t e;
    if ((e = d.alloc(&Ap, es * n)) || (e = d.alloc(&As, es * n)) || (e = d.alloc(&pin, es * n_pump)) ||
        (e = d.alloc(&svp, es * sizel)) || (e = d.alloc(&svs, es * sizel)))
        return fail_cuda("device memory", e);
    if (three && ((e = d.alloc(&Ai, es * n)) || (e = d.alloc(&svi, es * sizel)))) return fail_cuda("device memory", e);
    if ((e = upload(As, As0, o.precision)) || (e = upload(pin, pump, o.precision)) ||
        (three && (e = upload(Ai, Ai0, o.precision))))
        return fail_cuda("upload", e);
    if (cuopo_plan_create(&d.plan, &prm, w.data(), T.data(), o.precision) != CUOPO_OK) return fail_lib("plan");

    /* the loop of cuOPO.cu:474-610 in chunks of 500 round trips (progress as
     * the reference prints it); CW saves round trips NRT-64..NRT-1 (none when
     * NRT < 64: the reference's unsigned NRT-Nrts wraps around), NS every one */
    int save_first, save_count;
    if (ns_regime) {
        save_first = 0;
        save_count = (int)n_rt;
    } else if (n_rt >= nrts) {
        save_first = (int)(n_rt - nrts);
        save_count = (int)nrts;
    } else {
        save_first = 0;
        save_count = 0;
    }
    const int chunk = 500;
    for (unsigned rt = 0; rt < n_rt; rt += chunk) {
        const int cnt = (int)(n_rt - rt < (unsigned)chunk ? n_rt - rt : (unsigned)chunk);
        if (!o.quiet) {
            std::printf("#round trip: %u - Completed %u%%\t\r", rt, (unsigned)((unsigned long long)rt * 100 / n_rt));
            std::fflush(stdout);
        }
        if (cuopo_round_trips(d.plan, Ap, As, three ? Ai : nullptr, pin, (int)n_rt, (int)rt, cnt, svp, svs,
                              three ? svi : nullptr, save_first, save_count, nullptr, 0.0, nullptr, nullptr) != CUOPO_OK)
            return fail_lib("round trips");
    }
    if (cuopo_sync(nullptr) != CUOPO_OK) return fail_lib("round trips");
    int nonfinite = 0;
    if (cuopo_plan_status(d.plan, &nonfinite, 0) != CUOPO_OK) return fail_lib("status");
    if (nonfinite) std::fprintf(stderr, "cuopo: warning: non-finite signal power during the run\n");
    if (!o.quiet) std::printf("#round trip: %u - Completed 100%%\n", n_rt - 1);

    /* outputs (cuOPO.cu:620-635) */
    std::vector<float> out(2 * sizel);
    if (save_real(o, "Tp", Tp.data(), sizel) || save_real(o, "freq", Fp.data(), sizel) || save_real(o, "T", T.data(), n))
        return 1;
    if ((e = download(out, svs, o.precision))) return fail_cuda("download", e);
    if (save_complex(o, "signal_output", out.data(), sizel)) return 1;
    if ((e = download(out, svp, o.precision))) return fail_cuda("download", e);
    if (save_complex(o, "pump_output", out.data(), sizel)) return 1;
    if (three) {
        if ((e = download(out, svi, o.precision))) return fail_cuda("download", e);
        if (save_complex(o, "idler_output", out.data(), sizel)) return 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!o.quiet) std::printf("\n...time elapsed %.3f seconds\n", secs);
    return 0;
}
