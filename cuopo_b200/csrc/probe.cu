/*
 * probe.cu -- measured FP32 (and FP64) FMA throughput of the device, the
 * denominators of the solver's roofline (the fused SSFM kernels keep every
 * field on chip, so they are bound by FP32 / FP64 issue and shared-memory
 * bandwidth, not by HBM or the tensor cores).
 */
#include <cuda_runtime.h>

#include "cuopo.h"
#include "internal.h"

namespace {

/* 8 independent FMA chains per thread; the result is stored only if it is
 * never taken (x stays finite), so the compiler keeps every FMA. */
__global__ void __launch_bounds__(256) fma_probe(float *sink, int iters, float a, float b)
{
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = fmaf(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.678f) sink[blockIdx.x] = s;
}

/* The same with packed FP32x2 FMAs (two lanes per instruction, sm_100):
 * the FMA pipe's throughput without any limit from instruction issue. */
__global__ void __launch_bounds__(256) fma2_probe(float *sink, int iters, float a, float b)
{
    unsigned long long x[4], A, B;
    asm("mov.b64 %0, {%1, %1};" : "=l"(A) : "f"(a));
    asm("mov.b64 %0, {%1, %1};" : "=l"(B) : "f"(b));
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float u = (float)(threadIdx.x + k) * 1e-3f, v = (float)(threadIdx.x + k + 4) * 1e-3f;
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[k]) : "f"(u), "f"(v));
    }
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int k = 0; k < 4; k++) asm("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(x[k]) : "l"(A), "l"(B));
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        float u, v;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(u), "=f"(v) : "l"(x[k]));
        s += u + v;
    }
    if (s == 12345.678f) sink[blockIdx.x] = s;
}

/* FP64: 8 independent fma.rn.f64 chains per thread (the FP64 solver's
 * kernels are bound by this pipe). */
__global__ void __launch_bounds__(256) dfma_probe(double *sink, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (double)(threadIdx.x + k) * 1e-3;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 12345.678) sink[blockIdx.x] = s;
}

}  // namespace

extern "C" cuopo_status cuopo_probe_fp64_peak(double *tflops, void *stream)
{
    if (!tflops) return cuopo_fail(CUOPO_EINVAL, "probe_fp64_peak: NULL argument");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = (cudaStream_t)stream;
    double *sink = nullptr;
    cudaEvent_t e0, e1;
    cudaError_t e;
    if ((e = cudaMalloc(&sink, sizeof(double) * 64 * sms)) != cudaSuccess)
        return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = 8 * sms, threads = 256, iters = 512;
    dfma_probe<<<blocks, threads, 0, st>>>(sink, 16, 0.999, 1e-4); /* warm-up */
    double best = 0.0;
    for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0, st);
        dfma_probe<<<blocks, threads, 0, st>>>(sink, iters, 0.999, 1e-4);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
        if (ms > 0 && flops / (ms * 1e-3) / 1e12 > best) best = flops / (ms * 1e-3) / 1e12;
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    *tflops = best;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_probe_fp32_peak(double *tflops, void *stream)
{
    if (!tflops) return cuopo_fail(CUOPO_EINVAL, "probe_fp32_peak: NULL argument");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = (cudaStream_t)stream;
    float *sink = nullptr;
    cudaEvent_t e0, e1;
    cudaError_t e;
    if ((e = cudaMalloc(&sink, sizeof(float) * 64 * sms)) != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = 8 * sms, threads = 256, iters = 2048;
    fma_probe<<<blocks, threads, 0, st>>>(sink, 64, 0.999f, 1e-4f); /* warm-up */
    fma2_probe<<<blocks, threads, 0, st>>>(sink, 64, 0.999f, 1e-4f);
    double best = 0.0;
    /* the larger of scalar and packed FMA chains (8 FP32 chains per thread each) */
    for (int rep = 0; rep < 6; rep++) {
        cudaEventRecord(e0, st);
        if (rep % 2 == 0) fma_probe<<<blocks, threads, 0, st>>>(sink, iters, 0.999f, 1e-4f);
        else fma2_probe<<<blocks, threads, 0, st>>>(sink, iters, 0.999f, 1e-4f);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
        if (ms > 0 && flops / (ms * 1e-3) / 1e12 > best) best = flops / (ms * 1e-3) / 1e12;
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    *tflops = best;
    return CUOPO_OK;
}
