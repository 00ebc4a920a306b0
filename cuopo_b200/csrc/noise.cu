/*
 * noise.cu -- seeded complex Gaussian noise for the initial signal/idler.
 *
 * The reference seeds std::normal_distribution<float>(0, 1e-15) from the
 * wall clock (src/headers/functions.cuh:58-71), so its runs are not
 * reproducible.  Here value i of stream (seed, stream_id) is a pure
 * function of its indices: Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC'11) on the counter
 * (i, stream_id) with key seed gives two 32-bit words, which Box-Muller
 * turns into (re, im) ~ N(0, sigma^2) each.  The same code runs on the
 * host and on the device.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "cuopo.h"
#include "internal.h"

namespace {

__host__ __device__ inline void philox_round(uint32_t c[4], const uint32_t k[2])
{
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k[0];
    const uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    uint32_t k[2] = {k0, k1};
    for (int r = 0; r < 10; r++) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
}

__host__ __device__ inline void noise_pair(uint64_t seed, uint64_t stream_id, uint64_t i, double sigma,
                                           float *re, float *im)
{
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), (uint32_t)stream_id, (uint32_t)(stream_id >> 32)};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    /* two uniforms in (0, 1] from 64 bits each */
    const double u1 = ((double)(((uint64_t)c[0] << 21) ^ (uint64_t)c[1]) + 1.0) * (1.0 / 9007199254740992.0);
    const double u2 = ((double)(((uint64_t)c[2] << 21) ^ (uint64_t)c[3]) + 1.0) * (1.0 / 9007199254740992.0);
    const double r = sigma * sqrt(-2.0 * log(u1));
    const double s = sin(6.283185307179586477 * u2);
    const double co = cos(6.283185307179586477 * u2);
    *re = (float)(r * co);
    *im = (float)(r * s);
}

__global__ void noise_kernel(float2 *out, long n, double sigma, uint64_t seed, uint64_t stream_id)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float re, im;
        noise_pair(seed, stream_id, (uint64_t)i, sigma, &re, &im);
        out[i] = make_float2(re, im);
    }
}

}  // namespace

extern "C" void cuopo_noise_pair_host(uint64_t seed, uint64_t stream_id, uint64_t i, double sigma, float *re,
                                      float *im)
{
    noise_pair(seed, stream_id, i, sigma, re, im);
}

extern "C" cuopo_status cuopo_noise_host(float *out, long n, double sigma, uint64_t seed, uint64_t stream_id)
{
    if (!out || n < 0) return cuopo_fail(CUOPO_EINVAL, "noise_host: bad argument");
    for (long i = 0; i < n; i++) noise_pair(seed, stream_id, (uint64_t)i, sigma, &out[2 * i], &out[2 * i + 1]);
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_noise_device(void *out, long n, double sigma, uint64_t seed, uint64_t stream_id,
                                           void *stream)
{
    if (!out || n < 0) return cuopo_fail(CUOPO_EINVAL, "noise_device: bad argument");
    if (n == 0) return CUOPO_OK;
    const int threads = 256;
    long blocks = (n + threads - 1) / threads;
    if (blocks > 148 * 16) blocks = 148 * 16;
    noise_kernel<<<(int)blocks, threads, 0, (cudaStream_t)stream>>>((float2 *)out, n, sigma, seed, stream_id);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ECUDA, cudaGetErrorString(e));
    return CUOPO_OK;
}
