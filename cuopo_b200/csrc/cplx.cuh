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

/*
 * float2 on sm_100: the element-wise complex operations issue as one packed
 * FP32x2 instruction (add/sub/mul/fma .f32x2) for both components instead
 * of two scalar ones.  Each lane rounds exactly like the scalar operation
 * (round to nearest, fused multiply-add), so the results are those of the
 * scalar code with the same operation order; what changes is that one issue
 * slot carries two FP32 operations, which is the limit of the SSFM kernels.
 */
#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ >= 1000)
#define CUOPO_F32X2 1
#define CUOPO_F2OP3(OP, A, B)                                                                                 \
    float2 d;                                                                                                 \
    asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n " OP                  \
        " rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}"                                                             \
        : "=f"(d.x), "=f"(d.y)                                                                                \
        : "f"(A.x), "f"(A.y), "f"(B.x), "f"(B.y));                                                            \
    return d;

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { CUOPO_F2OP3("add.rn.f32x2", a, b) }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { CUOPO_F2OP3("sub.rn.f32x2", a, b) }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { CUOPO_F2OP3("mul.rn.f32x2", a, b) }
/* a * b + c, component-wise, fused */
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{\n .reg .b64 ra, rb, rc, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n mov.b64 rc, {%6, %7};\n"
        " fma.rn.f32x2 rd, ra, rb, rc;\n mov.b64 {%0, %1}, rd;\n}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}
#undef CUOPO_F2OP3

template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return f2add(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) { return f2sub(a, b); }
template <> __device__ __forceinline__ float2 cscale<float2, float>(float2 a, float s)
{
    return f2mul(a, make_float2(s, s));
}
template <> __device__ __forceinline__ float2 caxpy<float2, float>(float2 a, float s, float2 b)
{
    return f2fma(make_float2(s, s), b, a);
}
#endif

}  // namespace cuopo
