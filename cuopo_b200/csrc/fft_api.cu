/*
 * fft_api.cu -- the library's FFT as a stand-alone batched C2C transform,
 * a drop-in for the reference's cufftPlan1d + cufftExecC2C calls
 * (src/headers/cwes2.cuh:139-140,170-182; src/cuOPO.cu:453-454,522-550):
 * unnormalised, exponent sign +1 for CUFFT_INVERSE and -1 for
 * CUFFT_FORWARD, in place or out of place.  One CTA per transform.
 */
#include <cuda_runtime.h>

#include "cuopo.h"
#include "fft.cuh"
#include "internal.h"

using namespace cuopo;

namespace {

template <typename R, int M, int S>
__global__ void __launch_bounds__(M / 16) fft_kernel(const cpx<R> *in, cpx<R> *out, int batch)
{
    using C = cpx<R>;
    constexpr int T = M / 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *bufA = reinterpret_cast<C *>(smem_raw);
    C *bufB = bufA + M;
    C *tab = bufB + M;
    const int t = threadIdx.x;
    fill_twiddle_table<M>(tab, t);
    StageTwiddles<M, C> tw;
    tw.init(t, tab);
    __syncthreads();
    for (int b = blockIdx.x; b < batch; b += gridDim.x) {
        const C *src = in + (size_t)b * M;
        C *dst = out + (size_t)b * M;
        C reg[16];
#pragma unroll
        for (int e = 0; e < 16; e++) reg[e] = src[t + e * T];
        local_transform<S, M, 0, false>(reg, bufA, bufB, tw, t);
#pragma unroll
        for (int e = 0; e < 16; e++) dst[t + e * T] = reg[e];
        __syncthreads();
    }
}

template <typename R, int M, int S>
cudaError_t launch_fft(const void *in, void *out, int batch, cudaStream_t st)
{
    const size_t smem = sizeof(cpx<R>) * (2 * (size_t)M + TwTable<M>::size());
    static cudaError_t attr = cudaFuncSetAttribute(fft_kernel<R, M, S>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return attr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = batch < 8 * sms ? batch : 8 * sms;
    fft_kernel<R, M, S><<<grid, M / 16, smem, st>>>((const cpx<R> *)in, (cpx<R> *)out, batch);
    return cudaGetLastError();
}

template <typename R, int S>
cudaError_t dispatch(int n, const void *in, void *out, int batch, cudaStream_t st)
{
    switch (n) {
    case 512: return launch_fft<R, 512, S>(in, out, batch, st);
    case 1024: return launch_fft<R, 1024, S>(in, out, batch, st);
    case 2048: return launch_fft<R, 2048, S>(in, out, batch, st);
    case 4096: return launch_fft<R, 4096, S>(in, out, batch, st);
    case 8192:
        if constexpr (sizeof(R) == 4) return launch_fft<R, 8192, S>(in, out, batch, st);
        else return cudaErrorInvalidValue;
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

extern "C" cuopo_status cuopo_fft_c2c(const void *in, void *out, int n, int batch, int sign, int precision,
                                      void *stream)
{
    if (!in || !out || batch < 0 || (sign != 1 && sign != -1))
        return cuopo_fail(CUOPO_EINVAL, "fft_c2c: bad argument");
    if (precision != CUOPO_F32 && precision != CUOPO_F64) return cuopo_fail(CUOPO_EINVAL, "fft_c2c: bad precision");
    const int maxn = precision == CUOPO_F32 ? 8192 : 4096;
    if (n < 512 || n > maxn || (n & (n - 1)))
        return cuopo_fail(CUOPO_EUNSUPPORTED, "fft_c2c: n must be a power of 2 in [512, 8192] (F32) or [512, 4096] (F64)");
    if (batch == 0) return CUOPO_OK;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (precision == CUOPO_F32)
        e = sign > 0 ? dispatch<float, 1>(n, in, out, batch, st) : dispatch<float, -1>(n, in, out, batch, st);
    else
        e = sign > 0 ? dispatch<double, 1>(n, in, out, batch, st) : dispatch<double, -1>(n, in, out, batch, st);
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    return CUOPO_OK;
}
