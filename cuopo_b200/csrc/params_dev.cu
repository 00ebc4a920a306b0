/*
 * params_dev.cu -- the parameter derivation of src/cuOPO.cu:92-234 for a
 * whole sweep on the device: one warp per instance, the 5000-point
 * phase-matching temperature scan of src/headers/functions.cuh:23-54
 * spread over the warp's lanes, then the derivation itself
 * (setup_math.h, the same source as the host's cuopo_derive_params).
 *
 * Compiled without FMA contraction (-fmad=false) so that every float
 * operation rounds as the host's does; what can still differ from the
 * host (and so from the reference) is CUDA's powf, pow and logf against
 * glibc's, in the last bits.
 */
#include <cuda_runtime.h>

#include <cmath>

#include "cuopo.h"
#include "internal.h"
#include "setup_math.h"

namespace {

__global__ void derive_kernel(const cuopo_inputs *in, int count, cuopo_params *out, int *status)
{
    const int inst = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (inst >= count) return;
    const cuopo_inputs I = in[inst];
    const bool ok = (I.n_eqs == 2 || I.n_eqs == 3) && I.n_t >= 16 && (I.n_t & (I.n_t - 1)) == 0 && I.n_z >= 1 &&
                    (I.crystal == CUOPO_PPLN || I.crystal == CUOPO_SPPLT);
    if (!ok) {
        if (lane == 0) status[inst] = CUOPO_EINVAL;
        return;
    }
    const float lp = (float)(I.lp_nm * 1e-3);
    const float ls = I.ls_nm > 0 ? (float)(I.ls_nm * 1e-3) : 2 * lp;
    float Temp = (float)I.temp_c;
    if (I.temp_from_scan) {
        /* linspace(10, 150, 5000) (functions.cuh:12-18) and the first minimum of |mismatch| */
        const float span = 150.0f - 10.0f, den = (float)(int)(5000 - 1);
        float best = INFINITY;
        int bi = 0;
        for (int i = lane; i < 5000; i += 32) {
            const float T = 10.0f + (float)i * span / den;
            const float d = fabsf(pm_mismatch(I.crystal, lp, ls, (float)I.lambda_um, T));
            if (d < best) {
                best = d;
                bi = i;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob < best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        Temp = 10.0f + (float)bi * span / den;
    }
    if (lane == 0) {
        derive_core(&I, Temp, out + inst, nullptr);
        status[inst] = CUOPO_OK;
    }
}

}  // namespace

extern "C" cuopo_status cuopo_derive_params_device(const cuopo_inputs *in_dev, int count, cuopo_params *out_dev,
                                                   int *status_dev, void *stream)
{
    if (!in_dev || !out_dev || !status_dev || count < 1)
        return cuopo_fail(CUOPO_EINVAL, "derive_params_device: bad argument");
    const int threads = 256;
    const long blocks = ((long)count * 32 + threads - 1) / threads;
    derive_kernel<<<(unsigned)blocks, threads, 0, (cudaStream_t)stream>>>(in_dev, count, out_dev, status_dev);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    return CUOPO_OK;
}
