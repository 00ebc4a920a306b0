/*
 * cplx.cuh -- complex arithmetic on float2 / double2 for the solver kernels.
 * Fields are interleaved (re, im), the layout of cufftComplex.
 */
#pragma once
#include <cuda_runtime.h>

namespace cuopo {

template <typename R> struct cpx_of;
template <> struct cpx_of<float> { using type = float2; };
template <> struct cpx_of<double> { using type = double2; };
template <typename R> using cpx = typename cpx_of<R>::type;

template <typename C> struct real_of;
template <> struct real_of<float2> { using type = float; };
template <> struct real_of<double2> { using type = double; };

template <typename C, typename R = typename real_of<C>::type>
__host__ __device__ __forceinline__ C mk(R re, R im) { C c; c.x = re; c.y = im; return c; }

template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b)
{
    return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
/* a * conj(b) */
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b)
{
    return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) { return mk<C>(a.x * s, a.y * s); }
/* a + s*b */
template <typename C, typename R> __host__ __device__ __forceinline__ C caxpy(C a, R s, C b)
{
    return mk<C>(a.x + s * b.x, a.y + s * b.y);
}
/* sign * i * a, sign = +1 or -1 (compile time) */
template <int S, typename C> __host__ __device__ __forceinline__ C cmul_si(C a)
{
    return S > 0 ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x);
}
template <typename C> __host__ __device__ __forceinline__ double cabs2d(C a)
{
    return (double)a.x * (double)a.x + (double)a.y * (double)a.y;
}

}  // namespace cuopo
