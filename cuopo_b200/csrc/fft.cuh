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
 * Twiddles: a radix-16 stage whose sub-transform length is NS needs
 * W^{r k}, W = exp(2 pi i/(16 NS)), k = t mod NS, r = 1..15, fixed per
 * thread for the whole kernel.  Middle stages (NS <= M/256) read them from
 * a small shared-memory table formed in FP64 when the kernel starts
 * (15 NS entries per stage); the last stage (NS = M/16, one set per
 * thread) keeps the six FP64-rounded powers W^{k}, W^{2k}, W^{3k}, W^{4k},
 * W^{8k}, W^{12k} in registers and forms the others as one product
 * W^{4a k} W^{b k}.  Every twiddle is therefore within two roundings of
 * exact.
 */
#pragma once
#include "cplx.cuh"

namespace cuopo {

/* exp(S * i * pi * K / 8) * x, K compile-time. */
template <int S, int K, typename C>
__device__ __forceinline__ C tw16(C x)
{
    using R = typename real_of<C>::type;
    constexpr int k = ((K % 16) + 16) % 16;
    constexpr double c1 = 0.92387953251128675613;  /* cos(pi/8) */
    constexpr double s1 = 0.38268343236508977173;  /* sin(pi/8) */
    constexpr double h = 0.70710678118654752440;   /* sqrt(1/2) */
    if constexpr (k == 0) return x;
    else if constexpr (k == 4) return cmul_si<S>(x);
    else if constexpr (k == 8) return mk<C>(-x.x, -x.y);
    else if constexpr (k == 12) return cmul_si<-S>(x);
    else if constexpr (k == 2 || k == 6 || k == 10 || k == 14) {
        /* (c + i S s) with |c| = |s| = sqrt(1/2) */
        constexpr double c = (k == 2 || k == 14) ? h : -h;
        constexpr double s = (k == 2 || k == 6) ? h : -h;
        constexpr double ss = S * s;
        /* (a + i b)(c + i ss) */
        return mk<C>((R)c * x.x - (R)ss * x.y, (R)c * x.y + (R)ss * x.x);
    } else {
        constexpr double cs[16] = {1, c1, h, s1, 0, -s1, -h, -c1, -1, -c1, -h, -s1, 0, s1, h, c1};
        constexpr double sn[16] = {0, s1, h, c1, 1, c1, h, s1, 0, -s1, -h, -c1, -1, -c1, -h, -s1};
        constexpr double c = cs[k];
        constexpr double ss = S * sn[k];
        return mk<C>((R)c * x.x - (R)ss * x.y, (R)c * x.y + (R)ss * x.x);
    }
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

/* Shared-memory twiddle table of the middle radix-16 stages 1..P-2:
 * entry (p, r, k) = W_{16 NS_p}^{r k}, r = 1..15, k < NS_p. */
template <int M>
struct TwTable {
    using SP = StagePlan<M>;
    static constexpr int offset(int p)
    {
        int o = 0;
        for (int q = 1; q < p; q++) o += 15 * SP::ns(q);
        return o;
    }
    static constexpr int size() { return SP::P > 2 ? offset(SP::P - 1) : 0; }
};

/* Fills the table (all threads of the CTA cooperate; caller syncs). */
template <int M, typename C>
__device__ __forceinline__ void fill_twiddle_table(C *tab, int t)
{
    using SP = StagePlan<M>;
    using R = typename real_of<C>::type;
#pragma unroll
    for (int p = 1; p + 1 < SP::P; p++) {
        const int ns = SP::ns(p);
        const int off = TwTable<M>::offset(p);
        for (int idx = t; idx < 15 * ns; idx += SP::T) {
            const int r = idx / ns + 1, k = idx % ns;
            double sn, cs;
            sincospi(2.0 * (double)(r * k) / (16.0 * (double)ns), &sn, &cs);
            tab[off + idx] = mk<C>((R)cs, (R)sn);
        }
    }
}

/* The last radix-16 stage's twiddles of thread t (S = +1 form). */
template <int M, typename C>
struct StageTwiddles {
    C w1, w2, w3, w4, w8, w12;
    const C *tab;  /* shared-memory table of the middle stages */
    __device__ __forceinline__ void init(int t, const C *table)
    {
        using R = typename real_of<C>::type;
        using SP = StagePlan<M>;
        tab = table;
        if constexpr (SP::P > 1) {
            const int ns = SP::ns(SP::P - 1);
            const double k = (double)(t % ns);
            const double den = 16.0 * (double)ns;
            double sn, cs;
            sincospi(2.0 * k / den, &sn, &cs);
            w1 = mk<C>((R)cs, (R)sn);
            sincospi(4.0 * k / den, &sn, &cs);
            w2 = mk<C>((R)cs, (R)sn);
            sincospi(6.0 * k / den, &sn, &cs);
            w3 = mk<C>((R)cs, (R)sn);
            sincospi(8.0 * k / den, &sn, &cs);
            w4 = mk<C>((R)cs, (R)sn);
            sincospi(16.0 * k / den, &sn, &cs);
            w8 = mk<C>((R)cs, (R)sn);
            sincospi(24.0 * k / den, &sn, &cs);
            w12 = mk<C>((R)cs, (R)sn);
        }
    }
};

template <int S, typename C>
__device__ __forceinline__ C cj(C a)
{
    return S > 0 ? a : cconj(a);
}

/* v[4a+b] *= W^{(4a+b)k} from the six register powers (last stage). */
template <int S, typename C>
__device__ __forceinline__ void apply_last_twiddles(C (&v)[16], const C &w1, const C &w2, const C &w3,
                                                    const C &w4, const C &w8, const C &w12)
{
    const C b1 = cj<S>(w1), b2 = cj<S>(w2), b3 = cj<S>(w3);
    const C a1 = cj<S>(w4), a2 = cj<S>(w8), a3 = cj<S>(w12);
    v[1] = cmul(v[1], b1);
    v[2] = cmul(v[2], b2);
    v[3] = cmul(v[3], b3);
    v[4] = cmul(v[4], a1);
    v[5] = cmul(v[5], cmul(a1, b1));
    v[6] = cmul(v[6], cmul(a1, b2));
    v[7] = cmul(v[7], cmul(a1, b3));
    v[8] = cmul(v[8], a2);
    v[9] = cmul(v[9], cmul(a2, b1));
    v[10] = cmul(v[10], cmul(a2, b2));
    v[11] = cmul(v[11], cmul(a2, b3));
    v[12] = cmul(v[12], a3);
    v[13] = cmul(v[13], cmul(a3, b1));
    v[14] = cmul(v[14], cmul(a3, b2));
    v[15] = cmul(v[15], cmul(a3, b3));
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
                apply_last_twiddles<S>(v, tw.w1, tw.w2, tw.w3, tw.w4, tw.w8, tw.w12);
            } else {
                const int k = threadIdx.x % NS;
                const C *row = tw.tab + TwTable<M>::offset(P_IDX) + k;
#pragma unroll
                for (int r = 1; r < 16; r++) v[r] = cmul(v[r], cj<S>(row[(r - 1) * NS]));
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
