/*
 * fft.cuh -- register/shared-memory Stockham FFT used inside the fused
 * SSFM kernels.  Replaces the cufftExecC2C calls of the reference
 * (src/headers/cwes2.cuh:170-182, src/headers/cwes3.cuh:175-193,
 * src/cuOPO.cu:522-550): unnormalised C2C, exponent sign S = +1 for
 * CUFFT_INVERSE and S = -1 for CUFFT_FORWARD.
 *
 * Algorithm: Stockham autosort (Cooley-Tukey radix-r stages with the
 * reordering folded into each stage's store), mixed radix: one first
 * stage of radix 2/4/8 when log2(M) is not a multiple of 4, then radix-16
 * stages.  Every thread of the CTA holds E = 16 points of one field in
 * registers; stage outputs go through shared memory to the next stage.
 *
 * Thread t holds points t + e*T (T = M/16 threads, e = 0..15) both before
 * the first stage and after the last one, for any stage plan, so the
 * element-wise work of the solver (RK4, dispersion, cavity map) runs on
 * those registers with no shared-memory exchange or barrier.
 *
 * Twiddles are applied as rotations built from three shears,
 *   x -= t y;  y += s x;  x -= t y,      t = tan(phi/2), s = sin(phi),
 * after an exact quarter-turn step (a multiple of i) that leaves
 * |phi| <= pi/4 (Paeth's three-shear rotation).  Each shear has determinant
 * exactly 1 whatever the float values of t and s, so a rotation never
 * changes the power of a field with random phase to first order; a complex
 * multiplication by float-rounded (cos, sin) does (by |w_f|^2 - 1, a few
 * 1e-8, systematically), and over the ~10^6 transforms of a long cavity run
 * that bias moves the steady-state power by ~1e-4.  A radix-16 stage whose
 * sub-transform length is NS needs W^{r k}, W = exp(2 pi i/(16 NS)),
 * k = t mod NS: with r = b + 4a it applies the rotation by W^{b k} and then
 * a rotations by W^{4k}; the four base angles are all below pi/2.  The
 * last stage keeps its four bases in registers, middle stages read theirs
 * from a small shared-memory table; both are formed in FP64.
 */
#pragma once
#include "cplx.cuh"

namespace cuopo {

/* x * i^m (exact). */
template <int m, typename C>
__device__ __forceinline__ C iq(C x)
{
    constexpr int q = ((m % 4) + 4) % 4;
    if constexpr (q == 0) return x;
    else if constexpr (q == 1) return mk<C>(-x.y, x.x);
    else if constexpr (q == 2) return mk<C>(-x.x, -x.y);
    else return mk<C>(x.y, -x.x);
}

template <typename C>
__device__ __forceinline__ C iq_rt(C x, int m)
{
    using R = typename real_of<C>::type;
    R a = (m & 1) ? -x.y : x.x;
    R b = (m & 1) ? x.x : x.y;
    if (m & 2) {
        a = -a;
        b = -b;
    }
    return mk<C>(a, b);
}

/* Rotation of x by phi given (t, s) = (tan(phi/2), sin(phi)), three shears. */
template <typename C, typename R>
__device__ __forceinline__ C shear_rot(C x, R t, R s)
{
    const R x1 = x.x - t * x.y;
    const R y2 = x.y + s * x1;
    const R x3 = x1 - t * y2;
    return mk<C>(x3, y2);
}

/* exp(S * i * pi * K / 8) * x, K compile-time: quarter turns times a
 * rotation by r pi / 8, |r| <= 2. */
template <int S, int K, typename C>
__device__ __forceinline__ C tw16(C x)
{
    using R = typename real_of<C>::type;
    constexpr int n = S * (((K % 16) + 16) % 16);            /* angle n pi / 8 */
    constexpr int m = n >= 0 ? (n + 1) / 4 : -((-n + 1) / 4); /* nearest quarter turn */
    constexpr int r = n - 4 * m;                               /* -1..2 */
    constexpr double T1 = 0.19891236737965800691;              /* tan(pi/16) */
    constexpr double S1 = 0.38268343236508977173;              /* sin(pi/8) */
    constexpr double T2 = 0.41421356237309504880;              /* tan(pi/8) */
    constexpr double S2 = 0.70710678118654752440;              /* sin(pi/4) */
    const C y = iq<m>(x);
    if constexpr (r == 0) return y;
    else if constexpr (r == 1) return shear_rot(y, (R)T1, (R)S1);
    else if constexpr (r == -1) return shear_rot(y, (R)-T1, (R)-S1);
    else if constexpr (r == 2) return shear_rot(y, (R)T2, (R)S2);
    else return shear_rot(y, (R)-T2, (R)-S2);
}

template <int S, typename C>
__device__ __forceinline__ void dft2(C &x0, C &x1)
{
    const C a = cadd(x0, x1), b = csub(x0, x1);
    x0 = a;
    x1 = b;
}

template <int S, typename C>
__device__ __forceinline__ void dft4(C &x0, C &x1, C &x2, C &x3)
{
    const C a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = csub(x1, x3);
    const C sd = cmul_si<S>(d);
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, sd);
    x3 = csub(b, sd);
}

/* 8 = 2 x 4: n = b + 2a, k = q1 + 4 q2. */
template <int S, typename C>
__device__ __forceinline__ void dft8(C (&v)[8])
{
    dft4<S>(v[0], v[2], v[4], v[6]);
    dft4<S>(v[1], v[3], v[5], v[7]);
    v[3] = tw16<S, 2>(v[3]);
    v[5] = tw16<S, 4>(v[5]);
    v[7] = tw16<S, 6>(v[7]);
    C o[8];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        o[q] = cadd(v[2 * q], v[2 * q + 1]);
        o[q + 4] = csub(v[2 * q], v[2 * q + 1]);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = o[q];
}

/* 16 = 4 x 4: n = b + 4a, k = q1 + 4 q2. */
template <int S, typename C>
__device__ __forceinline__ void dft16(C (&v)[16])
{
#pragma unroll
    for (int b = 0; b < 4; b++) dft4<S>(v[b], v[b + 4], v[b + 8], v[b + 12]);
    /* u_b[q1] = v[b + 4 q1] *= W16^{b q1} */
    v[5] = tw16<S, 1>(v[5]);
    v[9] = tw16<S, 2>(v[9]);
    v[13] = tw16<S, 3>(v[13]);
    v[6] = tw16<S, 2>(v[6]);
    v[10] = tw16<S, 4>(v[10]);
    v[14] = tw16<S, 6>(v[14]);
    v[7] = tw16<S, 3>(v[7]);
    v[11] = tw16<S, 6>(v[11]);
    v[15] = tw16<S, 9>(v[15]);
#pragma unroll
    for (int q = 0; q < 4; q++) dft4<S>(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    /* X[q1 + 4 q2] = v[4 q1 + q2] */
    C o[16];
#pragma unroll
    for (int q1 = 0; q1 < 4; q1++)
#pragma unroll
        for (int q2 = 0; q2 < 4; q2++) o[q1 + 4 * q2] = v[4 * q1 + q2];
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = o[q];
}

template <int S, int RADIX, typename C>
__device__ __forceinline__ void dft(C (&v)[RADIX])
{
    if constexpr (RADIX == 2) dft2<S>(v[0], v[1]);
    else if constexpr (RADIX == 4) dft4<S>(v[0], v[1], v[2], v[3]);
    else if constexpr (RADIX == 8) dft8<S>(v);
    else dft16<S>(v);
}

/* Shared-memory index swizzle: XOR of the low bits with the row number so
 * that the stride-R stores of early stages hit distinct banks.  Rows are
 * 128 bytes (16 float2 or 8 double2). */
template <typename C>
__device__ __forceinline__ int swz(int i)
{
    if constexpr (sizeof(C) == 8) return i ^ ((i >> 4) & 15);
    else return i ^ ((i >> 3) & 7);
}

/* Stage plan of an M-point transform (M = 2^m, 16 <= M). */
template <int M>
struct StagePlan {
    static constexpr int lg(int x) { return x <= 1 ? 0 : 1 + lg(x / 2); }
    static constexpr int m = lg(M);
    static_assert((1 << m) == M && M >= 16, "M must be a power of 2 >= 16");
    static constexpr int R0 = (m % 4 == 0) ? 16 : (1 << (m % 4));
    static constexpr int P = (m % 4 == 0) ? m / 4 : m / 4 + 1;
    static constexpr int T = M / 16;
    static constexpr int radix(int p) { return p == 0 ? R0 : 16; }
    static constexpr int ns(int p)
    {
        int n = 1;
        for (int q = 0; q < p; q++) n *= radix(q);
        return n;
    }
};

/* Shared-memory table of the middle radix-16 stages 1..P-2: for stage p,
 * base j = 1..4 and k < NS_p the rotation (tan(theta/2), sin(theta)),
 * theta = 2 pi j k / (16 NS_p), stored as [p][j][k]. */
template <int M>
struct TwTable {
    using SP = StagePlan<M>;
    static constexpr int offset(int p)
    {
        int o = 0;
        for (int q = 1; q < p; q++) o += 4 * SP::ns(q);
        return o;
    }
    static constexpr int size() { return SP::P > 2 ? offset(SP::P - 1) : 0; }
};

template <typename C>
__device__ __forceinline__ C rot_params(int jk, int den)
{
    using R = typename real_of<C>::type;
    /* theta = 2 pi jk / den in [0, pi/2): t = tan(theta/2), s = sin(theta) */
    double sh, ch, sn, cs;
    sincospi((double)jk / (double)den, &sh, &ch);
    sincospi(2.0 * (double)jk / (double)den, &sn, &cs);
    return mk<C>((R)(sh / ch), (R)sn);
}

/* Fills the table (all threads of the CTA cooperate; caller syncs). */
template <int M, typename C>
__device__ __forceinline__ void fill_twiddle_table(C *tab, int t)
{
    using SP = StagePlan<M>;
#pragma unroll
    for (int p = 1; p + 1 < SP::P; p++) {
        const int ns = SP::ns(p);
        const int off = TwTable<M>::offset(p);
        for (int idx = t; idx < 4 * ns; idx += SP::T) {
            const int j = idx / ns + 1, k = idx % ns;
            tab[off + idx] = rot_params<C>(j * k, 16 * ns);
        }
    }
}

/* The last radix-16 stage's four base rotations of thread t. */
template <int M, typename C>
struct StageTwiddles {
    C b1, b2, b3, b4;  /* (tan(theta/2), sin(theta)) of W^k, W^2k, W^3k, W^4k */
    const C *tab;      /* shared-memory table of the middle stages */
    __device__ __forceinline__ void init(int t, const C *table)
    {
        using SP = StagePlan<M>;
        tab = table;
        if constexpr (SP::P > 1) {
            const int ns = SP::ns(SP::P - 1);
            const int k = t % ns;
            b1 = rot_params<C>(k, 16 * ns);
            b2 = rot_params<C>(2 * k, 16 * ns);
            b3 = rot_params<C>(3 * k, 16 * ns);
            b4 = rot_params<C>(4 * k, 16 * ns);
        }
    }
};

/* v[4a+b] rotated by S (b k + 4 a k) theta: the rotation by W^{bk}, then a
 * rotations by W^{4k}. */
template <int S, typename C>
__device__ __forceinline__ void apply_stage_rotations(C (&v)[16], C b1, C b2, C b3, C b4)
{
    using R = typename real_of<C>::type;
    const R sg = (R)S;
    const C q[4] = {b1, b1, b2, b3};
#pragma unroll
    for (int r = 1; r < 16; r++) {
        const int b = r & 3, a = r >> 2;
        C x = v[r];
        if (b) x = shear_rot(x, sg * q[b].x, sg * q[b].y);
#pragma unroll
        for (int i = 0; i < a; i++) x = shear_rot(x, sg * b4.x, sg * b4.y);
        v[r] = x;
    }
}

template <int S, int M, int P_IDX, typename C>
__device__ __forceinline__ void stage_compute(C (&reg)[16], const StageTwiddles<M, C> &tw)
{
    using SP = StagePlan<M>;
    constexpr int R = SP::radix(P_IDX);
    constexpr int NS = SP::ns(P_IDX);
    constexpr int B = 16 / R;
#pragma unroll
    for (int b = 0; b < B; b++) {
        C v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = reg[b + r * B];
        if constexpr (NS > 1) {
            static_assert(R == 16, "twiddled stages are radix 16");
            if constexpr (P_IDX + 1 == SP::P) {
                apply_stage_rotations<S>(v, tw.b1, tw.b2, tw.b3, tw.b4);
            } else {
                const int k = threadIdx.x % NS;
                const C *row = tw.tab + TwTable<M>::offset(P_IDX) + k;
                apply_stage_rotations<S>(v, row[0], row[NS], row[2 * NS], row[3 * NS]);
            }
        }
        dft<S, R>(v);
#pragma unroll
        for (int r = 0; r < R; r++) reg[b + r * B] = v[r];
    }
}

/* Stage P_IDX output to shared memory at its Stockham positions. */
template <int M, int P_IDX, typename C>
__device__ __forceinline__ void stage_store(C *buf, const C (&reg)[16], int t)
{
    using SP = StagePlan<M>;
    constexpr int R = SP::radix(P_IDX);
    constexpr int NS = SP::ns(P_IDX);
    constexpr int B = 16 / R;
    constexpr int T = SP::T;
#pragma unroll
    for (int b = 0; b < B; b++) {
        const int j = t + b * T;
        const int k = j % NS;
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) buf[swz<C>(base + r * NS)] = reg[b + r * B];
    }
}

template <int M, typename C>
__device__ __forceinline__ void load_own(const C *buf, C (&reg)[16], int t)
{
    constexpr int T = StagePlan<M>::T;
#pragma unroll
    for (int e = 0; e < 16; e++) reg[e] = buf[swz<C>(t + e * T)];
}

template <int M, typename C>
__device__ __forceinline__ void store_own(C *buf, const C (&reg)[16], int t)
{
    constexpr int T = StagePlan<M>::T;
#pragma unroll
    for (int e = 0; e < 16; e++) buf[swz<C>(t + e * T)] = reg[e];
}

/*
 * Local M-point transform of the registers of the CTA (exponent sign S).
 * Exchange x (counted from X0 within the caller's sequence) goes through
 * buffer (x even ? bufA : bufB).  INPLACE: bufA == bufB, and every
 * exchange is bracketed by two barriers instead of one.
 */
template <int S, int M, int X0, bool INPLACE, int P_IDX = 0, typename C>
__device__ __forceinline__ void local_transform(C (&reg)[16], C *bufA, C *bufB,
                                                const StageTwiddles<M, C> &tw, int t)
{
    constexpr int P = StagePlan<M>::P;
    stage_compute<S, M, P_IDX>(reg, tw);
    if constexpr (P_IDX + 1 < P) {
        C *buf = ((X0 + P_IDX) % 2 == 0) ? bufA : bufB;
        if constexpr (INPLACE) __syncthreads();
        stage_store<M, P_IDX>(buf, reg, t);
        __syncthreads();
        load_own<M>(buf, reg, t);
        local_transform<S, M, X0, INPLACE, P_IDX + 1>(reg, bufA, bufB, tw, t);
    }
}

}  // namespace cuopo
