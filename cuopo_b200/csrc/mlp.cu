/*
 * mlp.cu -- the learned warm start's network: a multilayer perceptron
 * n_in -> width (GELU) x depth -> n_out trained and evaluated with BF16
 * operands on the sm_100a tensor cores (tcgen05.mma, FP32 accumulation in
 * tensor memory), operands staged in shared memory by TMA.  The reference
 * has no counterpart: it always starts a run from noise
 * (src/headers/functions.cuh:58-71).
 *
 * Every contraction of training and inference is one kernel, tc_gemm_kernel:
 * C[M][N] = A[M][K] B[N][K]^T with A and B row-major BF16 ("K-major"), one
 * 128 x BN output tile per CTA, the K loop pipelined through STAGES
 * shared-memory buffers (one TMA producer thread, one MMA issuer thread,
 * mbarriers in between), the accumulator in tensor memory, and a fused
 * epilogue run by 16 warps (TMEM lanes = tile rows, 4 lane quadrants x up
 * to 4 chunks of 32 columns):
 *   forward    z = A W^T + b, h = GELU(z): stores GELU'(z), h and h^T (BF16);
 *   output     y = A W^T + b (FP32);
 *   dX         g_prev = (g W) * GELU'(z_prev) (the stored derivative):
 *              stores g_prev, g_prev^T and adds the column sums of g_prev
 *              into the bias gradient;
 *   dW         grad_W += g^T act over a K slice (split over the batch,
 *              FP32 atomics).
 * Keeping every activation and gradient in both layouts (row-major and
 * transposed, written by the producing epilogue) makes every GEMM of the
 * backward pass a K-major one as well.
 *
 * Device waits on mbarriers are bounded (about 1 s of %globaltimer); a wait
 * that gives up sets the error word and the kernel finishes without storing
 * its tile, freeing its tensor memory (the host turns the word into
 * CUOPO_ETIMEOUT).
 */
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <utility>
#include <vector>

#include "cuopo.h"
#include "internal.h"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int BM = 128;      /* tile rows = TMEM lanes */
constexpr int BK = 64;       /* K per stage: 64 BF16 = one 128-byte swizzle row */
constexpr int STAGES = 4;
constexpr int NTHREADS = 512;   /* 16 warps: 4 TMEM lane quadrants x up to 4 column chunks */
constexpr unsigned long long WAIT_NS = 1000000000ull;

/* ------------------------------------------------------------ PTX helpers */

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* Waits for the phase of parity `parity` of mbarrier b; gives up after
 * WAIT_NS of global time and returns false. */
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity)
{
    if (mbar_try(b, parity)) return true;
    const unsigned long long t0 = gtimer();
    while (!mbar_try(b, parity))
        if (gtimer() - t0 > WAIT_NS) return false;
    return true;
}

/* 2-D tiled TMA load (no multicast) of box {64, rows} at (x, y) into dst,
 * completing on mbarrier bar. */
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

/* Shared-memory matrix descriptor of a K-major tile whose 128-byte rows are
 * stored with the 128-byte swizzle (the TMA's SWIZZLE_128B): 8-row groups
 * 1024 bytes apart (stride byte offset), descriptor version 1 (sm_100),
 * layout type 2 = SWIZZLE_128B. */
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

/* Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
 * N >> 3 at bit 17, M >> 4 at bit 24. */
template <int BN>
__host__ __device__ constexpr uint32_t idesc_bf16()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

/* Programmatic dependent launch: wait for the previous kernel in the stream
 * (a no-op when this grid was launched without the attribute), and let the
 * next one start its prologue early. */
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

/* 32 consecutive FP32 columns of this thread's TMEM lane. */
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

/* -------------------------------------------------------- GELU (erf form) */

/* GELU(z) = z Phi(z) and GELU'(z) = Phi(z) + z phi(z), with
 * Phi(z) = (1 + erf(z / sqrt 2)) / 2 and phi(z) = exp(-z^2 / 2) / sqrt(2 pi).
 * erf(x), x >= 0, by Abramowitz & Stegun 7.1.26 (Handbook of Mathematical
 * Functions, 1964): 1 - (a1 t + ... + a5 t^5) exp(-x^2), t = 1 / (1 + p x),
 * absolute error <= 1.5e-7 -- far below the BF16 rounding of the stored
 * values -- and its exp(-x^2) = exp(-z^2/2) is also phi's. */
__device__ __forceinline__ void gelu_and_grad(float z, float &h, float &gp)
{
    const float x = fabsf(z) * 0.70710678118654752f;
    const float e = __expf(-0.5f * z * z);
    const float t = __fdividef(1.0f, 1.0f + 0.3275911f * x);
    const float poly =
        t * (0.254829592f + t * (-0.284496736f + t * (1.421413741f + t * (-1.453152027f + t * 1.061405429f))));
    const float erf_abs = 1.0f - poly * e;
    const float phi_cdf = 0.5f + 0.5f * copysignf(erf_abs, z);
    h = z * phi_cdf;
    gp = phi_cdf + z * 0.39894228040143268f * e;
}


/* ------------------------------------------------------------ epilogue */

struct Epi {
    int ldo;              /* row stride of the row-major outputs (= N of the GEMM) */
    int ldt;              /* row stride of the transposed output */
    const float *bias;    /* [N] added first, or NULL */
    int act;              /* 0 none, 1 GELU, 2 multiply by gp_in */
    const bf16 *gp_in;    /* GELU'(z) [M][ldo] for act 2 */
    bf16 *gp_out;         /* act 1: GELU'(z) of the pre-activation z [M][ldo], or NULL */
    bf16 *out_bf;         /* [M][ldo], or NULL */
    bf16 *out_bfT;        /* [N][ldt], or NULL */
    float *out_f;         /* [M][ldo], or NULL */
    int atomic;           /* out_f += (split K) instead of = */
    float *colsum;        /* [N] += column sums of the BF16-rounded result, or NULL */
    int *err;             /* bit 0: a bounded wait gave up */
    int hold_done;        /* test hook: the completion barrier is never signalled, so the
                             epilogue's bounded wait runs out (CUOPO_ETIMEOUT path) */
};

__device__ __forceinline__ void store_bf16x32(bf16 *dst, const float (&v)[32])
{
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint4 u;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            __nv_bfloat162 h = __floats2bfloat162_rn(v[8 * q + 2 * j], v[8 * q + 2 * j + 1]);
            w[j] = *reinterpret_cast<uint32_t *>(&h);
        }
        u.x = w[0]; u.y = w[1]; u.z = w[2]; u.w = w[3];
        reinterpret_cast<uint4 *>(dst)[q] = u;
    }
}

__device__ __forceinline__ void load_bf16x32(const bf16 *src, float (&v)[32])
{
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint4 u = reinterpret_cast<const uint4 *>(src)[q];
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int j = 0; j < 4; j++) {
            __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162 *>(&w[j]);
            const float2 f = __bfloat1622float2(h);
            v[8 * q + 2 * j] = f.x;
            v[8 * q + 2 * j + 1] = f.y;
        }
    }
}

/* Row `row`, columns col..col+31 of the tile; lane = this thread's lane. */
__device__ __forceinline__ void epilogue32(const Epi &ep, int row, int col, float (&v)[32], int lane, bool store)
{
    if (ep.bias) {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] += __ldg(ep.bias + col + j);
    }
    const size_t o = (size_t)row * ep.ldo + col;
    if (ep.act == 1) {
        float gp[32];
#pragma unroll
        for (int j = 0; j < 32; j++) gelu_and_grad(v[j], v[j], gp[j]);
        if (ep.gp_out && store) store_bf16x32(ep.gp_out + o, gp);
    } else if (ep.act == 2) {
        float gp[32];
        load_bf16x32(ep.gp_in + o, gp);
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] *= gp[j];
    }
    if (ep.out_f && store) {
        float4 *d = reinterpret_cast<float4 *>(ep.out_f + o);
        if (ep.atomic) {
#pragma unroll
            for (int q = 0; q < 8; q++) {
                atomicAdd(&d[q].x, v[4 * q]);
                atomicAdd(&d[q].y, v[4 * q + 1]);
                atomicAdd(&d[q].z, v[4 * q + 2]);
                atomicAdd(&d[q].w, v[4 * q + 3]);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
    }
    if (ep.out_bf || ep.out_bfT || ep.colsum) {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] = __bfloat162float(__float2bfloat16_rn(v[j]));
    }
    if (ep.out_bf && store) store_bf16x32(ep.out_bf + o, v);
    if (ep.out_bfT && store) {
#pragma unroll
        for (int j = 0; j < 32; j++) ep.out_bfT[(size_t)(col + j) * ep.ldt + row] = __float2bfloat16_rn(v[j]);
    }
    if (ep.colsum) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
            float s = v[j];
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
            if (lane == 0 && store) atomicAdd(ep.colsum + col + j, s);
        }
    }
}

template <int BN>
constexpr size_t gemm_smem_bytes()
{
    return 1024 + (size_t)STAGES * (BM * BK * 2 + BN * BK * 2) + (2 * STAGES + 1) * 8 + 16;
}

/*
 * C tile (blockIdx.x, blockIdx.y) over the K slice blockIdx.z * kb_per ..
 * (+kb_per) blocks of 64.  512 threads: thread 0 issues the TMA loads,
 * thread 32 the MMAs; after the last MMA every warp runs the epilogue of
 * one 32 x 32 block of the tile.
 */
template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const Epi ep,
                   int kb_per)
{
    static_assert(BN == 64 || BN == 128, "tile width: one 32-column chunk per warp and quadrant");
    extern __shared__ uint8_t smem_dyn[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2;
    uint8_t *sA = smem;
    uint8_t *sB = smem + STAGES * A_BYTES;
    uint64_t *full = (uint64_t *)(sB + STAGES * B_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *slot = (uint32_t *)(done + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN, kb0 = blockIdx.z * kb_per;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(slot, BN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *slot;
    /* everything above is this CTA's own set-up; the operands and the
     * epilogue's inputs come from the previous kernel */
    griddep_wait();
    griddep_launch();

    __shared__ int s_err;
    if (threadIdx.x == 0) s_err = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int kb = 0; kb < kb_per; kb++) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(empty + s, ((kb / STAGES) & 1) ^ 1)) {
                atomicOr(&s_err, 1);
                break;
            }
            mbar_expect_tx(full + s, A_BYTES + B_BYTES);
            tma_load_2d(sA + s * A_BYTES, &tmA, (kb0 + kb) * BK, m0, full + s);
            tma_load_2d(sB + s * B_BYTES, &tmB, (kb0 + kb) * BK, n0, full + s);
        }
    } else if (threadIdx.x == 32) {
        constexpr uint32_t idesc = idesc_bf16<BN>();
        for (int kb = 0; kb < kb_per; kb++) {
            const int s = kb % STAGES;
            if (!mbar_wait(full + s, (kb / STAGES) & 1)) {
                atomicOr(&s_err, 1);
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + s * A_BYTES), b0 = smem_u32(sB + s * B_BYTES);
#pragma unroll
            for (int k = 0; k < BK / 16; k++)
                umma_bf16(tmem, sw128_desc(a0 + 32 * k), sw128_desc(b0 + 32 * k), idesc, (kb | k) != 0);
            umma_commit(empty + s);   /* frees the stage once these MMAs have read it */
        }
        if (!ep.hold_done) umma_commit(done);   /* arrives when every MMA above has completed */
    }
    __syncwarp();
    if (!mbar_wait(done, 0)) atomicOr(&s_err, 1);
    /* every role loop and every wait above has ended (all are bounded) */
    __syncthreads();
    tc_fence_after();
    const bool store = s_err == 0;
    /* warp w reads TMEM lane quadrant w % 4 (the lanes it may access) and
     * column chunk w / 4 of 32 */
    const int quad = warp & 3, chunk = warp >> 2;
    if (chunk < BN / 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(chunk * 32), v);
        epilogue32(ep, m0 + quad * 32 + lane, n0 + chunk * 32, v, lane, store);
    }
    if (!store && threadIdx.x == 0 && ep.err) atomicOr(ep.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, BN);
}

/* ------------------------------------------------------- host: TMA maps */

typedef CUresult (*encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                    const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                    CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_fn encoder()
{
    static encode_tiled_fn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (encode_tiled_fn)p;
    }();
    return fn;
}

/* Row-major BF16 matrix [rows][cols] read in boxes of 64 columns x box_rows
 * rows with the 128-byte swizzle. */
cuopo_status encode_bf16(CUtensorMap *m, const void *base, long rows, long cols, int box_rows)
{
    encode_tiled_fn enc = encoder();
    if (!enc) return cuopo_fail(CUOPO_ECUDA, "mlp: cuTensorMapEncodeTiled unavailable");
    if (((uintptr_t)base & 15) || (cols * 2) % 16 || cols % 64 || rows % box_rows)
        return cuopo_fail(CUOPO_EINVAL, "mlp: matrix not aligned for TMA (16-byte base, 64-column multiples)");
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cuopo_fail(CUOPO_ECUDA, "mlp: cuTensorMapEncodeTiled failed");
    return CUOPO_OK;
}

cudaError_t prepare_gemm();

/* Set while a training step is being captured: its kernels are launched with
 * programmatic stream serialization, so each one's launch and set-up overlap
 * the previous one's tail (every kernel waits with griddepcontrol.wait
 * before it reads the previous one's results). */
thread_local int g_pdl = 0; /* 0 off; 1 on from the next launch on; 2 on */

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args &&...args)
{
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = g_pdl == 2 ? 1 : 0;
    if (g_pdl) g_pdl = 2;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int BN>
cudaError_t launch_gemm_bn(const CUtensorMap &a, const CUtensorMap &b, const Epi &ep, int M, int N, int K, int split,
                           cudaStream_t st)
{
    cudaError_t attr = prepare_gemm();
    if (attr != cudaSuccess) return attr;
    dim3 grid((unsigned)(M / BM), (unsigned)(N / BN), (unsigned)split);
    cudaError_t e = launch_k(tc_gemm_kernel<BN>, grid, dim3(NTHREADS), gemm_smem_bytes<BN>(), st, a, b, ep,
                             (K / BK) / split);
    return e != cudaSuccess ? e : cudaGetLastError();
}

/* C = A B^T with tile width bn (64 or 128); K split into `split` slices. */
cudaError_t launch_gemm(const CUtensorMap &a, const CUtensorMap &b, const Epi &ep, int M, int N, int K, int bn,
                        int split, cudaStream_t st)
{
    return bn == 64 ? launch_gemm_bn<64>(a, b, ep, M, N, K, split, st)
                    : launch_gemm_bn<128>(a, b, ep, M, N, K, split, st);
}

/* The largest split of K (in blocks of 64, dividing them) that keeps
 * tiles x split within one wave of the 148 SMs. */
int pick_split(int tiles, int kblocks)
{
    int best = 1;
    for (int s = 1; s <= kblocks; s++) {
        if (kblocks % s) continue;
        if (tiles * s > 148) break;
        best = s;
    }
    return best;
}

/* Shared-memory opt-in of both tile widths, outside any stream capture. */
cudaError_t prepare_gemm()
{
    static cudaError_t st = [] {
        cudaError_t e = cudaFuncSetAttribute(tc_gemm_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)gemm_smem_bytes<64>());
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tc_gemm_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)gemm_smem_bytes<128>());
        return e;
    }();
    return st;
}

Epi epi_none(int ldo, int *err)
{
    Epi e;
    std::memset(&e, 0, sizeof(e));
    e.ldo = ldo;
    e.err = err;
    return e;
}

cuopo_status cuda_err(cudaError_t e, const char *what)
{
    char buf[300];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return cuopo_fail(CUOPO_ECUDA, buf);
}

/* ------------------------------------------------------- small kernels */

/* Training/inference input: x [batch][n_in] FP32 -> xin [rows][64] BF16
 * (zero padded in both directions) and, when xinT != NULL, xin^T [64][ldt];
 * target t [batch][n_out] -> tgt (rows >= batch zero) when t != NULL.
 * Thread (0,0) also advances the Adam step and forms its scalars. */
struct PackArgs {
    const float *x;
    const float *t;
    bf16 *xin;
    bf16 *xinT;
    float *tgt;
    int batch, rows, n_in, n_out, ldt;
    int *step;
    float *adam;      /* [lr, 1 - beta1^t, 1 - beta2^t] */
    float lr, beta1, beta2;
};

__global__ void pack_kernel(const PackArgs a)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (long)a.rows * 64) {
        const int r = (int)(i / 64), c = (int)(i % 64);
        const float v = (r < a.batch && c < a.n_in) ? a.x[(size_t)r * a.n_in + c] : 0.f;
        const bf16 b = __float2bfloat16_rn(v);
        a.xin[i] = b;
        if (a.xinT) a.xinT[(size_t)c * a.ldt + r] = b;
    }
    if (a.t && i < (long)a.rows * a.n_out) {
        const int r = (int)(i / a.n_out);
        a.tgt[i] = r < a.batch ? a.t[i] : 0.f;
    }
    if (i == 0 && a.step) {
        const int t = ++*a.step;
        a.adam[0] = a.lr;
        a.adam[1] = 1.0f - powf(a.beta1, (float)t);
        a.adam[2] = 1.0f - powf(a.beta2, (float)t);
    }
}

/* Mean squared error over batch x n_out and its gradient 2 (y - t) / (batch
 * n_out) (zero on rows >= batch), stored as g [rows][n_out] and g^T
 * [n_out][ldt] (BF16); bias gradient += column sums of the BF16 g; loss +=
 * the batch's mean.  Block: n_out threads x MSE_ROWS rows (each thread
 * writes its column's MSE_ROWS values of g^T as 16-byte stores). */
constexpr int MSE_ROWS = 16;
__global__ void mse_kernel(const float *y, const float *tgt, bf16 *g, bf16 *gT, float *db, float *loss, int batch,
                           int n_out, int ldt)
{
    griddep_wait();
    griddep_launch();
    const int j = threadIdx.x, r0 = blockIdx.x * MSE_ROWS;
    const float scale = 2.0f / ((float)batch * (float)n_out);
    float csum = 0.f, lsum = 0.f;
    uint32_t packed[MSE_ROWS / 2];
#pragma unroll
    for (int q = 0; q < MSE_ROWS; q += 2) {
        float gv[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const int r = r0 + q + u;
            const size_t o = (size_t)r * n_out + j;
            float d = 0.f;
            if (r < batch) d = y[o] - tgt[o];
            lsum += d * d;
            const bf16 b = __float2bfloat16_rn(d * scale);
            g[o] = b;
            gv[u] = __bfloat162float(b);
            csum += gv[u];
        }
        __nv_bfloat162 h = __floats2bfloat162_rn(gv[0], gv[1]);
        packed[q / 2] = *reinterpret_cast<uint32_t *>(&h);
    }
    uint4 *dst = reinterpret_cast<uint4 *>(gT + (size_t)j * ldt + r0);
#pragma unroll
    for (int q = 0; q < MSE_ROWS / 8; q++)
        dst[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
    atomicAdd(db + j, csum);
    __shared__ float part[32];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, d);
    if ((j & 31) == 0) part[j >> 5] = lsum;
    __syncthreads();
    if (j == 0) {
        float s = 0.f;
        for (int w = 0; w < (n_out + 31) / 32; w++) s += part[w];
        atomicAdd(loss, s / ((float)batch * (float)n_out));
    }
}

/* Parameter segments of the flat FP32 buffer: weights [N][Kp] (with a BF16
 * copy and its transpose) or biases [N]. */
struct Seg {
    long off, len;
    int N, Kp;          /* Kp = 0 for a bias */
    bf16 *w, *wT;
};
constexpr int MAX_SEG = 24;
struct AdamArgs {
    float *p, *g, *m, *v;
    const float *adam;  /* [lr, 1 - beta1^t, 1 - beta2^t] */
    float beta1, beta2, eps;
    float gscale;       /* the gradient is multiplied by this (1 / ranks after a sum over ranks) */
    int update;         /* 0: only refresh the BF16 copies */
    int nseg;
    Seg seg[MAX_SEG];
};

__global__ void adam_kernel(const AdamArgs a, long total)
{
    griddep_wait();
    griddep_launch();
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    float p = a.p[i];
    if (a.update) {
        const float g = a.g[i] * a.gscale;
        const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
        const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
        a.m[i] = m;
        a.v[i] = v;
        const float mh = m / a.adam[1], vh = v / a.adam[2];
        p -= a.adam[0] * mh / (sqrtf(vh) + a.eps);
        a.p[i] = p;
    }
    int s = 0;
    while (s + 1 < a.nseg && i >= a.seg[s + 1].off) s++;
    const Seg &sg = a.seg[s];
    if (sg.Kp > 0) sg.w[i - sg.off] = __float2bfloat16_rn(p);
}

/* W^T [Kp][N] from W [N][Kp] (BF16) through 32 x 32 shared-memory tiles, so
 * that both the reads and the writes are coalesced; blockIdx.z = weight
 * segment (a.seg[2 l]). */
__global__ void transpose_weights_kernel(const AdamArgs a)
{
    griddep_wait();
    griddep_launch();
    __shared__ bf16 tile[32][33];
    const Seg &sg = a.seg[2 * blockIdx.z];
    const int n0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
    if (n0 >= sg.N || k0 >= sg.Kp) return;
    const int tx = threadIdx.x, ty = threadIdx.y;   /* 32 x 8 */
    for (int r = ty; r < 32; r += 8) tile[r][tx] = sg.w[(size_t)(n0 + r) * sg.Kp + k0 + tx];
    __syncthreads();
    for (int r = ty; r < 32; r += 8) sg.wT[(size_t)(k0 + r) * sg.N + n0 + tx] = tile[tx][r];
}

}  /* namespace */

/* ====================================================== the MLP object */

struct cuopo_mlp {
    int n_in, width, depth, n_out, max_batch, rows;   /* rows = max_batch rounded up to 128 */
    int L;                                            /* layers = depth + 1 */
    std::vector<int> N, K, Kp;                        /* per layer: outputs, inputs, padded inputs */
    std::vector<long> w_off, b_off;                   /* flat offsets (internal, padded layer 0) */
    long P;                                           /* internal parameter count */
    float *params, *grads, *m, *v, *adam, *loss, *y, *tgt;
    int *err, *step;
    bf16 *xin, *xinT;
    std::vector<bf16 *> w_bf, wT_bf;                  /* per layer [N][Kp], [Kp][N] */
    std::vector<bf16 *> gp, h, hT, g, gT;             /* per hidden layer [rows][width] / [width][rows];
                                                         gp = GELU'(z) */
    bf16 *g_out, *g_outT;
    std::vector<CUtensorMap> mA_fwd, mB_fwd, mA_dW, mB_dW, mA_dX, mB_dX;
    std::vector<void *> allocs;
    AdamArgs adam_args;
    cudaGraphExec_t graph;        /* forward, loss, backward, Adam */
    int graph_batch;
    cudaStream_t graph_stream;
    cudaGraphExec_t grad_graph;   /* forward, loss, backward (data-parallel steps) */
    int grad_graph_batch;
    cudaStream_t grad_graph_stream;
};

namespace {

template <typename T>
cuopo_status dalloc(cuopo_mlp *m, T **p, size_t count)
{
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, sizeof(T) * count);
    if (e != cudaSuccess) return cuopo_fail(CUOPO_ENOMEM, "mlp: cudaMalloc failed");
    m->allocs.push_back(q);
    *p = (T *)q;
    return CUOPO_OK;
}

/* The activation feeding layer l (row-major and transposed). */
bf16 *act_in(cuopo_mlp *m, int l) { return l == 0 ? m->xin : m->h[l - 1]; }
bf16 *act_inT(cuopo_mlp *m, int l) { return l == 0 ? m->xinT : m->hT[l - 1]; }

cuopo_status launch_check(cudaError_t e, const char *what)
{
    return e == cudaSuccess ? CUOPO_OK : cuda_err(e, what);
}

/* Forward pass over `rows_used` rows (a multiple of 128).  train: keep z, h^T. */
cuopo_status forward(cuopo_mlp *m, int rows_used, bool train, cudaStream_t st)
{
    for (int l = 0; l < m->L; l++) {
        Epi ep = epi_none(m->N[l], m->err);
        ep.bias = m->params + m->b_off[l];
        ep.ldt = m->rows;
        if (l < m->L - 1) {
            ep.act = 1;
            ep.out_bf = m->h[l];
            if (train) {
                ep.gp_out = m->gp[l];
                ep.out_bfT = m->hT[l];
            }
        } else {
            ep.out_f = m->y;
        }
        cuopo_status s = launch_check(launch_gemm(m->mA_fwd[l], m->mB_fwd[l], ep, rows_used, m->N[l], m->Kp[l], 128, 1,
                                                  st),
                                      "mlp forward GEMM");
        if (s != CUOPO_OK) return s;
    }
    return CUOPO_OK;
}

cuopo_status zero_grads(cuopo_mlp *m, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(m->grads, 0, sizeof(float) * m->P, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->loss, 0, sizeof(float), st);
    return e != cudaSuccess ? cuda_err(e, "mlp: memset") : CUOPO_OK;
}

/* Loss, gradients (into m->grads) over rows_used rows; `zero`: clear the
 * gradient and loss accumulators first (a captured step clears them before
 * its forward pass, so that its kernels follow one another directly). */
cuopo_status backward(cuopo_mlp *m, int batch, int rows_used, cudaStream_t st, bool zero = true)
{
    cudaError_t e;
    if (zero) {
        cuopo_status z = zero_grads(m, st);
        if (z != CUOPO_OK) return z;
    }
    const int Lo = m->L - 1;
    e = launch_k(mse_kernel, dim3((unsigned)(rows_used / MSE_ROWS)), dim3((unsigned)m->n_out), 0, st,
                 (const float *)m->y, (const float *)m->tgt, m->g_out, m->g_outT, m->grads + m->b_off[Lo], m->loss,
                 batch, m->n_out, m->rows);
    if (e != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "mlp: loss kernel");
    for (int l = Lo; l >= 0; l--) {
        /* dW_l = g_l^T act_{l-1}: M = N_l, N = Kp_l, K = rows_used */
        Epi ew = epi_none(m->Kp[l], m->err);
        ew.out_f = m->grads + m->w_off[l];
        ew.atomic = 1;
        const int bn = (m->Kp[l] % 128 == 0) ? 128 : 64;
        const int tiles = (m->N[l] / BM) * (m->Kp[l] / bn);
        const int split = pick_split(tiles, rows_used / BK);
        cuopo_status s = launch_check(launch_gemm(m->mA_dW[l], m->mB_dW[l], ew, m->N[l], m->Kp[l], rows_used, bn,
                                                  split, st),
                                      "mlp dW GEMM");
        if (s != CUOPO_OK) return s;
        if (l == 0) break;
        /* g_{l-1} = (g_l W_l) * GELU'(z_{l-1}): M = rows_used, N = Kp_l (= width), K = N_l */
        Epi ex = epi_none(m->Kp[l], m->err);
        ex.ldt = m->rows;
        ex.act = 2;
        ex.gp_in = m->gp[l - 1];
        ex.out_bf = m->g[l - 1];
        ex.out_bfT = m->gT[l - 1];
        ex.colsum = m->grads + m->b_off[l - 1];
        s = launch_check(launch_gemm(m->mA_dX[l], m->mB_dX[l], ex, rows_used, m->Kp[l], m->N[l], 128, 1, st),
                         "mlp dX GEMM");
        if (s != CUOPO_OK) return s;
    }
    return CUOPO_OK;
}

cuopo_status run_adam(cuopo_mlp *m, int update, cudaStream_t st, float gscale = 1.0f)
{
    AdamArgs a = m->adam_args;
    a.update = update;
    a.gscale = gscale;
    const int tpb = 256;
    cudaError_t e = launch_k(adam_kernel, dim3((unsigned)((m->P + tpb - 1) / tpb)), dim3(tpb), 0, st, a, m->P);
    cuopo_status s = launch_check(e != cudaSuccess ? e : cudaGetLastError(), "mlp: adam kernel");
    if (s != CUOPO_OK) return s;
    int maxN = 0, maxK = 0;
    for (int l = 0; l < m->L; l++) {
        maxN = m->N[l] > maxN ? m->N[l] : maxN;
        maxK = m->Kp[l] > maxK ? m->Kp[l] : maxK;
    }
    e = launch_k(transpose_weights_kernel, dim3((unsigned)(maxK / 32), (unsigned)(maxN / 32), (unsigned)m->L),
                 dim3(32, 8), 0, st, a);
    return launch_check(e != cudaSuccess ? e : cudaGetLastError(), "mlp: weight transpose kernel");
}

cuopo_status pack(cuopo_mlp *m, const float *x, const float *t, int batch, int rows_used, bool train, float lr,
                  cudaStream_t st)
{
    PackArgs a;
    std::memset(&a, 0, sizeof(a));
    a.x = x;
    a.t = t;
    a.xin = m->xin;
    a.xinT = train ? m->xinT : nullptr;
    a.tgt = m->tgt;
    a.batch = batch;
    a.rows = rows_used;
    a.n_in = m->n_in;
    a.n_out = m->n_out;
    a.ldt = m->rows;
    a.step = (train && lr > 0) ? m->step : nullptr;
    a.adam = m->adam;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    const long n = (long)rows_used * (m->n_out > 64 ? m->n_out : 64);
    pack_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a);
    return launch_check(cudaGetLastError(), "mlp: pack kernel");
}

int round128(int b) { return (b + 127) / 128 * 128; }

cuopo_status check_err(cuopo_mlp *m)
{
    int e = 0;
    cudaError_t ce = cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return cuda_err(ce, "mlp: error word");
    if (e) {
        cudaMemset(m->err, 0, sizeof(int));
        return cuopo_fail(CUOPO_ETIMEOUT, "mlp: a GEMM's bounded wait gave up");
    }
    return CUOPO_OK;
}

}  /* namespace */

extern "C" cuopo_status cuopo_mlp_create(cuopo_mlp **out, int n_in, int width, int depth, int n_out, int max_batch,
                                         uint64_t seed)
{
    if (!out) return cuopo_fail(CUOPO_EINVAL, "mlp_create: NULL argument");
    *out = nullptr;
    if (n_in < 1 || n_in > 64 || width < 128 || width % 128 || n_out < 128 || n_out % 128 || n_out > 1024 ||
        depth < 1 || depth > 10 || max_batch < 1)
        return cuopo_fail(CUOPO_EINVAL, "mlp_create: need 1 <= n_in <= 64, width and n_out multiples of 128 "
                                        "(n_out <= 1024), 1 <= depth <= 10, max_batch >= 1");
    cudaError_t pe = prepare_gemm();
    if (pe != cudaSuccess) return cuda_err(pe, "mlp_create: kernel attributes");
    cuopo_mlp *m = new cuopo_mlp();
    m->n_in = n_in;
    m->width = width;
    m->depth = depth;
    m->n_out = n_out;
    m->max_batch = max_batch;
    m->rows = round128(max_batch);
    m->L = depth + 1;
    m->graph = nullptr;
    m->graph_batch = -1;
    m->graph_stream = nullptr;
    m->grad_graph = nullptr;
    m->grad_graph_batch = -1;
    m->grad_graph_stream = nullptr;
    long off = 0;
    for (int l = 0; l < m->L; l++) {
        m->N.push_back(l == m->L - 1 ? n_out : width);
        m->K.push_back(l == 0 ? n_in : width);
        m->Kp.push_back(l == 0 ? 64 : width);
        m->w_off.push_back(off);
        off += (long)m->N[l] * m->Kp[l];
        m->b_off.push_back(off);
        off += m->N[l];
    }
    m->P = off;
    auto fail = [&](cuopo_status s) {
        cuopo_mlp_destroy(m);
        return s;
    };
    cuopo_status s;
    const size_t R = (size_t)m->rows;
    if ((s = dalloc(m, &m->params, m->P)) || (s = dalloc(m, &m->grads, m->P)) || (s = dalloc(m, &m->m, m->P)) ||
        (s = dalloc(m, &m->v, m->P)) || (s = dalloc(m, &m->adam, 4)) || (s = dalloc(m, &m->loss, 1)) ||
        (s = dalloc(m, &m->y, R * n_out)) || (s = dalloc(m, &m->tgt, R * n_out)) || (s = dalloc(m, &m->err, 1)) ||
        (s = dalloc(m, &m->step, 1)) || (s = dalloc(m, &m->xin, R * 64)) || (s = dalloc(m, &m->xinT, R * 64)) ||
        (s = dalloc(m, &m->g_out, R * n_out)) || (s = dalloc(m, &m->g_outT, R * n_out)))
        return fail(s);
    m->w_bf.resize(m->L);
    m->wT_bf.resize(m->L);
    for (int l = 0; l < m->L; l++)
        if ((s = dalloc(m, &m->w_bf[l], (size_t)m->N[l] * m->Kp[l])) ||
            (s = dalloc(m, &m->wT_bf[l], (size_t)m->N[l] * m->Kp[l])))
            return fail(s);
    m->gp.resize(depth);
    m->h.resize(depth);
    m->hT.resize(depth);
    m->g.resize(depth);
    m->gT.resize(depth);
    for (int l = 0; l < depth; l++)
        if ((s = dalloc(m, &m->gp[l], R * width)) || (s = dalloc(m, &m->h[l], R * width)) ||
            (s = dalloc(m, &m->hT[l], R * width)) || (s = dalloc(m, &m->g[l], R * width)) ||
            (s = dalloc(m, &m->gT[l], R * width)))
            return fail(s);
    cudaError_t e = cudaMemset(m->m, 0, sizeof(float) * m->P);
    if (e == cudaSuccess) e = cudaMemset(m->v, 0, sizeof(float) * m->P);
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->step, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->xin, 0, sizeof(bf16) * R * 64);
    if (e == cudaSuccess) e = cudaMemset(m->xinT, 0, sizeof(bf16) * R * 64);
    if (e != cudaSuccess) return fail(cuda_err(e, "mlp_create: memset"));

    /* tensor maps (every activation buffer has m->rows rows) */
    m->mA_fwd.resize(m->L);
    m->mB_fwd.resize(m->L);
    m->mA_dW.resize(m->L);
    m->mB_dW.resize(m->L);
    m->mA_dX.resize(m->L);
    m->mB_dX.resize(m->L);
    for (int l = 0; l < m->L; l++) {
        const int last = l == m->L - 1;
        if ((s = encode_bf16(&m->mA_fwd[l], act_in(m, l), m->rows, m->Kp[l], BM)) ||
            (s = encode_bf16(&m->mB_fwd[l], m->w_bf[l], m->N[l], m->Kp[l], 128)) ||
            (s = encode_bf16(&m->mA_dW[l], last ? m->g_outT : m->gT[l], m->N[l], m->rows, BM)) ||
            (s = encode_bf16(&m->mB_dW[l], act_inT(m, l), m->Kp[l], m->rows, m->Kp[l] % 128 == 0 ? 128 : 64)))
            return fail(s);
        if (l > 0 && ((s = encode_bf16(&m->mA_dX[l], last ? m->g_out : m->g[l], m->rows, m->N[l], BM)) ||
                      (s = encode_bf16(&m->mB_dX[l], m->wT_bf[l], m->Kp[l], m->N[l], 128))))
            return fail(s);
    }
    /* Adam segments */
    AdamArgs &a = m->adam_args;
    std::memset(&a, 0, sizeof(a));
    a.p = m->params;
    a.g = m->grads;
    a.m = m->m;
    a.v = m->v;
    a.adam = m->adam;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.gscale = 1.0f;
    a.nseg = 2 * m->L;
    for (int l = 0; l < m->L; l++) {
        a.seg[2 * l] = Seg{m->w_off[l], (long)m->N[l] * m->Kp[l], m->N[l], m->Kp[l], m->w_bf[l], m->wT_bf[l]};
        a.seg[2 * l + 1] = Seg{m->b_off[l], m->N[l], m->N[l], 0, nullptr, nullptr};
    }
    /* initial weights: uniform(-sqrt(6/fan_in), +sqrt(6/fan_in)), zero biases (splitmix64 stream of seed) */
    std::vector<float> host((size_t)m->P, 0.f);
    uint64_t st = seed ^ 0x6A09E667F3BCC909ull;
    auto next = [&st]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t x = st;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return (double)((x ^ (x >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < m->L; l++) {
        const double lim = std::sqrt(6.0 / m->K[l]);
        for (int n = 0; n < m->N[l]; n++)
            for (int k = 0; k < m->K[l]; k++)
                host[(size_t)(m->w_off[l] + (long)n * m->Kp[l] + k)] = (float)((2.0 * next() - 1.0) * lim);
    }
    e = cudaMemcpy(m->params, host.data(), sizeof(float) * m->P, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(cuda_err(e, "mlp_create: upload"));
    if ((s = run_adam(m, 0, 0)) != CUOPO_OK) return fail(s);
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(cuda_err(e, "mlp_create"));
    *out = m;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_destroy(cuopo_mlp *m)
{
    if (!m) return CUOPO_OK;
    if (m->graph) cudaGraphExecDestroy(m->graph);
    if (m->grad_graph) cudaGraphExecDestroy(m->grad_graph);
    for (void *p : m->allocs) cudaFree(p);
    delete m;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_param_count(const cuopo_mlp *m, long *n)
{
    if (!m || !n) return cuopo_fail(CUOPO_EINVAL, "mlp_param_count: NULL argument");
    *n = m->P - (long)m->N[0] * (64 - m->n_in);
    return CUOPO_OK;
}

/* User layout: per layer W_l [N_l][K_l] then b_l [N_l] (layer 0 unpadded). */
extern "C" cuopo_status cuopo_mlp_set_params(cuopo_mlp *m, const float *host)
{
    if (!m || !host) return cuopo_fail(CUOPO_EINVAL, "mlp_set_params: NULL argument");
    std::vector<float> in((size_t)m->P, 0.f);
    long u = 0;
    for (int l = 0; l < m->L; l++) {
        for (int n = 0; n < m->N[l]; n++)
            for (int k = 0; k < m->K[l]; k++) in[(size_t)(m->w_off[l] + (long)n * m->Kp[l] + k)] = host[u++];
        for (int n = 0; n < m->N[l]; n++) in[(size_t)(m->b_off[l] + n)] = host[u++];
    }
    cudaError_t e = cudaMemcpy(m->params, in.data(), sizeof(float) * m->P, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(m->m, 0, sizeof(float) * m->P);
    if (e == cudaSuccess) e = cudaMemset(m->v, 0, sizeof(float) * m->P);
    if (e == cudaSuccess) e = cudaMemset(m->step, 0, sizeof(int));
    if (e != cudaSuccess) return cuda_err(e, "mlp_set_params");
    cuopo_status s = run_adam(m, 0, 0);
    if (s != CUOPO_OK) return s;
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? CUOPO_OK : cuda_err(e, "mlp_set_params");
}

static cuopo_status to_user_layout(const cuopo_mlp *m, const float *internal, float *host)
{
    long u = 0;
    for (int l = 0; l < m->L; l++) {
        for (int n = 0; n < m->N[l]; n++)
            for (int k = 0; k < m->K[l]; k++) host[u++] = internal[(size_t)(m->w_off[l] + (long)n * m->Kp[l] + k)];
        for (int n = 0; n < m->N[l]; n++) host[u++] = internal[(size_t)(m->b_off[l] + n)];
    }
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_get_params(cuopo_mlp *m, float *host)
{
    if (!m || !host) return cuopo_fail(CUOPO_EINVAL, "mlp_get_params: NULL argument");
    std::vector<float> in((size_t)m->P);
    cudaError_t e = cudaMemcpy(in.data(), m->params, sizeof(float) * m->P, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_err(e, "mlp_get_params");
    return to_user_layout(m, in.data(), host);
}

extern "C" cuopo_status cuopo_mlp_forward(cuopo_mlp *m, const float *x, float *y, int batch, void *stream)
{
    cuopo::Range range_("cuopo_mlp_forward");
    if (!m || !x || !y) return cuopo_fail(CUOPO_EINVAL, "mlp_forward: NULL argument");
    if (batch < 1 || batch > m->max_batch) return cuopo_fail(CUOPO_EINVAL, "mlp_forward: batch outside [1, max_batch]");
    cudaStream_t st = (cudaStream_t)stream;
    const int rows = round128(batch);
    cuopo_status s = pack(m, x, nullptr, batch, rows, false, 0.f, st);
    if (s == CUOPO_OK) s = forward(m, rows, false, st);
    if (s != CUOPO_OK) return s;
    cudaError_t e = cudaMemcpyAsync(y, m->y, sizeof(float) * (size_t)batch * m->n_out, cudaMemcpyDeviceToDevice, st);
    return e == cudaSuccess ? CUOPO_OK : cuda_err(e, "mlp_forward: copy out");
}

extern "C" cuopo_status cuopo_mlp_gradients(cuopo_mlp *m, const float *x, const float *t, int batch, float *grad,
                                            float *loss, void *stream)
{
    cuopo::Range range_("cuopo_mlp_gradients");
    if (!m || !x || !t) return cuopo_fail(CUOPO_EINVAL, "mlp_gradients: NULL argument");
    if (batch < 1 || batch > m->max_batch) return cuopo_fail(CUOPO_EINVAL, "mlp_gradients: batch outside [1, max_batch]");
    cudaStream_t st = (cudaStream_t)stream;
    const int rows = round128(batch);
    cuopo_status s = pack(m, x, t, batch, rows, true, 0.f, st);
    if (s == CUOPO_OK) s = forward(m, rows, true, st);
    if (s == CUOPO_OK) s = backward(m, batch, rows, st);
    if (s != CUOPO_OK) return s;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(e, "mlp_gradients");
    if ((s = check_err(m)) != CUOPO_OK) return s;
    if (loss) {
        e = cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_err(e, "mlp_gradients: loss");
    }
    if (grad) {
        std::vector<float> in((size_t)m->P);
        e = cudaMemcpy(in.data(), m->grads, sizeof(float) * m->P, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_err(e, "mlp_gradients: copy out");
        to_user_layout(m, in.data(), grad);
    }
    return CUOPO_OK;
}

namespace {

/* Captures forward + loss + backward (+ Adam) for one batch size on a
 * stream into *exec (replacing an earlier graph). */
cuopo_status capture_step(cuopo_mlp *m, int batch, int rows, cudaStream_t st, bool with_adam, cudaGraphExec_t *exec)
{
    if (*exec) {
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    cudaError_t e;
    cudaStream_t cap = st;
    bool own = false;
    if (!cap) {
        if ((e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_err(e, "mlp: capture stream");
        own = true;
        if ((e = cudaStreamSynchronize(0)) != cudaSuccess) {
            cudaStreamDestroy(cap);
            return cuda_err(e, "mlp: capture");
        }
    }
    cudaGraph_t g = nullptr;
    if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        if (own) cudaStreamDestroy(cap);
        return cuda_err(e, "mlp: begin capture");
    }
    cuopo_status s = zero_grads(m, cap);
    g_pdl = 1;
    if (s == CUOPO_OK) s = forward(m, rows, true, cap);
    if (s == CUOPO_OK) s = backward(m, batch, rows, cap, false);
    if (s == CUOPO_OK && with_adam) s = run_adam(m, 1, cap);
    g_pdl = 0;
    e = cudaStreamEndCapture(cap, &g);
    if (s == CUOPO_OK && e != cudaSuccess) s = cuda_err(e, "mlp: end capture");
    if (s == CUOPO_OK) {
        e = cudaGraphInstantiate(exec, g, 0);
        if (e != cudaSuccess) s = cuda_err(e, "mlp: instantiate");
    }
    if (g) cudaGraphDestroy(g);
    if (own) cudaStreamDestroy(cap);
    return s;
}

/* Step counter and Adam scalars for a standalone update. */
__global__ void adam_scalars_kernel(int *step, float *adam, float lr, float beta1, float beta2)
{
    const int t = ++*step;
    adam[0] = lr;
    adam[1] = 1.0f - powf(beta1, (float)t);
    adam[2] = 1.0f - powf(beta2, (float)t);
}

}  /* namespace */

extern "C" cuopo_status cuopo_mlp_train_step(cuopo_mlp *m, const float *x, const float *t, int batch, float lr,
                                             float *loss, void *stream)
{
    cuopo::Range range_("cuopo_mlp_train_step");
    if (!m || !x || !t) return cuopo_fail(CUOPO_EINVAL, "mlp_train_step: NULL argument");
    if (batch < 1 || batch > m->max_batch) return cuopo_fail(CUOPO_EINVAL, "mlp_train_step: batch outside [1, max_batch]");
    if (!(lr > 0)) return cuopo_fail(CUOPO_EINVAL, "mlp_train_step: lr must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    const int rows = round128(batch);
    /* the step's inputs go into the network's own buffers outside the graph */
    cuopo_status s = pack(m, x, t, batch, rows, true, lr, st);
    if (s != CUOPO_OK) return s;
    if (!m->graph || m->graph_batch != batch || m->graph_stream != st) {
        /* forward + loss + backward + Adam, captured once per (batch, stream) */
        if ((s = capture_step(m, batch, rows, st, true, &m->graph)) != CUOPO_OK) return s;
        m->graph_batch = batch;
        m->graph_stream = st;
    }
    cudaError_t e;
    if ((e = cudaGraphLaunch(m->graph, st)) != cudaSuccess) return cuda_err(e, "mlp_train_step: graph launch");
    if (loss && (e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return cuda_err(e, "mlp_train_step: loss");
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_grad_step(cuopo_mlp *m, const float *x, const float *t, int batch, float *loss,
                                            void *stream)
{
    cuopo::Range range_("cuopo_mlp_grad_step");
    if (!m || !x || !t) return cuopo_fail(CUOPO_EINVAL, "mlp_grad_step: NULL argument");
    if (batch < 1 || batch > m->max_batch) return cuopo_fail(CUOPO_EINVAL, "mlp_grad_step: batch outside [1, max_batch]");
    cudaStream_t st = (cudaStream_t)stream;
    const int rows = round128(batch);
    cuopo_status s = pack(m, x, t, batch, rows, true, 0.f, st);
    if (s != CUOPO_OK) return s;
    if (!m->grad_graph || m->grad_graph_batch != batch || m->grad_graph_stream != st) {
        if ((s = capture_step(m, batch, rows, st, false, &m->grad_graph)) != CUOPO_OK) return s;
        m->grad_graph_batch = batch;
        m->grad_graph_stream = st;
    }
    cudaError_t e;
    if ((e = cudaGraphLaunch(m->grad_graph, st)) != cudaSuccess) return cuda_err(e, "mlp_grad_step: graph launch");
    if (loss && (e = cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
        return cuda_err(e, "mlp_grad_step: loss");
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_grad_buffer(cuopo_mlp *m, float **grad_dev, long *count)
{
    if (!m || !grad_dev || !count) return cuopo_fail(CUOPO_EINVAL, "mlp_grad_buffer: NULL argument");
    *grad_dev = m->grads;
    *count = m->P;
    return CUOPO_OK;
}

extern "C" cuopo_status cuopo_mlp_apply_adam(cuopo_mlp *m, float lr, float grad_scale, void *stream)
{
    cuopo::Range range_("cuopo_mlp_apply_adam");
    if (!m) return cuopo_fail(CUOPO_EINVAL, "mlp_apply_adam: NULL argument");
    if (!(lr > 0) || !(grad_scale > 0)) return cuopo_fail(CUOPO_EINVAL, "mlp_apply_adam: lr and grad_scale must be > 0");
    cudaStream_t st = (cudaStream_t)stream;
    adam_scalars_kernel<<<1, 1, 0, st>>>(m->step, m->adam, lr, 0.9f, 0.999f);
    cuopo_status s = launch_check(cudaGetLastError(), "mlp_apply_adam: scalars");
    if (s != CUOPO_OK) return s;
    return run_adam(m, 1, st, grad_scale);
}

extern "C" cuopo_status cuopo_mlp_status(cuopo_mlp *m)
{
    if (!m) return cuopo_fail(CUOPO_EINVAL, "mlp_status: NULL argument");
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_err(e, "mlp_status");
    return check_err(m);
}

/* The tensor-core GEMM alone (tests and roofline): C = A B^T. */
extern "C" cuopo_status cuopo_gemm_bf16(const void *A, const void *B, float *C, int M, int N, int K, int split,
                                        int flags, int *err_dev, void *stream)
{
    if (!A || !B || !C) return cuopo_fail(CUOPO_EINVAL, "gemm_bf16: NULL argument");
    if ((uintptr_t)C & 15) return cuopo_fail(CUOPO_EINVAL, "gemm_bf16: C must be 16-byte aligned");
    if (M < 128 || M % 128 || N < 64 || N % 64 || K < 64 || K % 64 || split < 1 || (K / 64) % split)
        return cuopo_fail(CUOPO_EINVAL, "gemm_bf16: M multiple of 128, N of 64, K of 64, split dividing K/64");
    const int bn = (N % 128 == 0) ? 128 : 64;
    cudaError_t pe = prepare_gemm();
    if (pe != cudaSuccess) return cuda_err(pe, "gemm_bf16: kernel attributes");
    CUtensorMap ma, mb;
    cuopo_status s = encode_bf16(&ma, A, M, K, BM);
    if (s == CUOPO_OK) s = encode_bf16(&mb, B, N, K, bn);
    if (s != CUOPO_OK) return s;
    Epi ep = epi_none(N, err_dev);
    ep.out_f = C;
    ep.atomic = split > 1;
    ep.hold_done = flags & 1;
    cudaStream_t st = (cudaStream_t)stream;
    if (split > 1) {
        cudaError_t e = cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * N, st);
        if (e != cudaSuccess) return cuda_err(e, "gemm_bf16: memset");
    }
    return launch_check(launch_gemm(ma, mb, ep, M, N, K, bn, split, st), "gemm_bf16");
}

/* ============================================ warm-start fields <-> modes */

namespace {

/* Mode k of n_modes (k = 0..n_modes-1) is the Fourier mode q = k - n_modes/2
 * (cycles per round trip).  field[n] = scale sum_q c_q exp(+2 pi i q n / n_t),
 * summed directly for one point per thread (any n_t, the same continuous
 * field sampled on every grid): the phasor of the first mode of each group
 * of 16 comes from sincospif of the exact reduced argument 2 (q n mod n_t) /
 * n_t, the next 15 by rotation with exp(2 pi i n / n_t). */
__global__ void fields_from_modes_kernel(const float *modes, int n_modes, int n_t, float scale, float2 *fields)
{
    extern __shared__ float2 cm[];
    const size_t inst = blockIdx.y;
    for (int k = threadIdx.x; k < n_modes; k += blockDim.x)
        cm[k] = make_float2(modes[inst * 2 * (size_t)n_modes + 2 * k], modes[inst * 2 * (size_t)n_modes + 2 * k + 1]);
    __syncthreads();
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_t) return;
    const unsigned long long mask = (unsigned long long)n_t - 1;
    const float inv = 2.0f / (float)n_t;
    float sr, cr;
    sincospif((float)((unsigned long long)n & mask) * inv, &sr, &cr);
    float ar = 0.f, ai = 0.f;
    for (int k0 = 0; k0 < n_modes; k0 += 16) {
        const long long q = (long long)k0 - n_modes / 2;
        const unsigned long long m = ((unsigned long long)(q + (long long)n_t) * (unsigned long long)n) & mask;
        float s, c;
        sincospif((float)m * inv, &s, &c);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float2 v = cm[k0 + j];
            ar += v.x * c - v.y * s;
            ai += v.x * s + v.y * c;
            const float c2 = c * cr - s * sr;
            s = s * cr + c * sr;
            c = c2;
        }
    }
    fields[inst * n_t + n] = make_float2(scale * ar, scale * ai);
}

/* One block of n_modes threads per instance: c_q = X[q mod n_t] / (n_t
 * scale), then the sign that makes the largest mode's real part >= 0 (the
 * 2-wave equations are invariant under As -> -As). */
__global__ void modes_from_spectrum_kernel(const float2 *spec, int n_t, int n_modes, float inv, float *modes)
{
    extern __shared__ float red[];   /* [n_modes] magnitudes, [n_modes] indices (as float) */
    const size_t inst = blockIdx.x;
    const int k = threadIdx.x;
    const int q = k - n_modes / 2;
    const float2 x = spec[inst * n_t + (size_t)((q + n_t) % n_t)];
    const float re = x.x * inv, im = x.y * inv;
    red[k] = re * re + im * im;
    red[n_modes + k] = (float)k;
    __syncthreads();
    for (int s = n_modes / 2; s > 0; s >>= 1) {
        if (k < s && red[k + s] > red[k]) {
            red[k] = red[k + s];
            red[n_modes + k] = red[n_modes + k + s];
        }
        __syncthreads();
    }
    const int kmax = (int)red[n_modes];
    const float2 xm = spec[inst * n_t + (size_t)((kmax - n_modes / 2 + n_t) % n_t)];
    const float sg = (xm.x < 0.f) ? -1.f : 1.f;
    modes[inst * 2 * (size_t)n_modes + 2 * k] = sg * re;
    modes[inst * 2 * (size_t)n_modes + 2 * k + 1] = sg * im;
}

}  /* namespace */

extern "C" cuopo_status cuopo_fields_from_modes(const float *modes, int count, int n_modes, int n_t, double scale,
                                                void *fields, void *stream)
{
    if (!modes || !fields || count < 1) return cuopo_fail(CUOPO_EINVAL, "fields_from_modes: bad argument");
    if (count > 65535) return cuopo_fail(CUOPO_EINVAL, "fields_from_modes: at most 65535 instances per call");
    if (n_modes < 16 || n_modes % 16 || n_modes > 1024 || n_modes > n_t || n_t < 16 || (n_t & (n_t - 1)))
        return cuopo_fail(CUOPO_EINVAL, "fields_from_modes: n_modes a multiple of 16 in [16, min(n_t, 1024)], "
                                        "n_t a power of 2");
    dim3 grid((unsigned)((n_t + 255) / 256), (unsigned)count);
    fields_from_modes_kernel<<<grid, 256, n_modes * sizeof(float2), (cudaStream_t)stream>>>(
        modes, n_modes, n_t, (float)scale, (float2 *)fields);
    return launch_check(cudaGetLastError(), "fields_from_modes");
}

extern "C" cuopo_status cuopo_modes_from_spectrum(const void *spec, int count, int n_t, int n_modes, double scale,
                                                  float *modes, void *stream)
{
    if (!modes || !spec || count < 1 || !(scale > 0)) return cuopo_fail(CUOPO_EINVAL, "modes_from_spectrum: bad argument");
    if (n_modes < 2 || n_modes > 1024 || (n_modes & (n_modes - 1)) || n_modes > n_t || (n_t & (n_t - 1)))
        return cuopo_fail(CUOPO_EINVAL, "modes_from_spectrum: n_modes a power of 2 <= min(n_t, 1024)");
    modes_from_spectrum_kernel<<<(unsigned)count, (unsigned)n_modes, 2 * n_modes * sizeof(float),
                                 (cudaStream_t)stream>>>((const float2 *)spec, n_t, n_modes,
                                                         (float)(1.0 / ((double)n_t * scale)), modes);
    return launch_check(cudaGetLastError(), "modes_from_spectrum");
}

/* ================================ warm-start fields from a band prediction */

namespace {

/* Layout of one prediction row (n_out = 512) of the band representation:
 * [0, 128) magnitudes of the modes q0-64 .. q0+63, [128, 256) of the modes
 * -q0-64 .. -q0+63, then 64 copies each of cos(Phi), sin(Phi), the band
 * centre as 2 (q0 / (n_t/2))^2 - 1 (q0^2 is close to linear in the cavity
 * detuning) and log10(P) (their means are used). */
constexpr int BAND = 128;
constexpr int BAND_ROW = 512;

__global__ void fields_from_bands_kernel(const float *pred, int n_t, float scale, float2 *fields, int *centres)
{
    __shared__ float row[BAND_ROW];
    __shared__ float2 coef[2 * BAND];
    __shared__ float sc[2];
    __shared__ int q0s;
    const size_t inst = blockIdx.y;
    const int t = threadIdx.x;   /* 256 threads */
    for (int k = t; k < BAND_ROW; k += blockDim.x) row[k] = pred[inst * BAND_ROW + k];
    __syncthreads();
    if (t < 32) {
        /* means of the four scalar groups, and the band power sum(max(a,0)^2) */
        float m[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
        for (int j = t; j < 64; j += 32)
#pragma unroll
            for (int g = 0; g < 4; g++) m[g] += row[2 * BAND + 64 * g + j];
        for (int k = t; k < 2 * BAND; k += 32) {
            const float a = fmaxf(row[k], 0.f);
            m[4] += a * a;
        }
#pragma unroll
        for (int g = 0; g < 5; g++)
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) m[g] += __shfl_xor_sync(0xffffffffu, m[g], d);
        if (t == 0) {
            const float u = fmaxf(0.5f * (m[2] / 64.f + 1.0f), 0.f);
            int q0 = __float2int_rn(sqrtf(u) * (float)(n_t / 2));
            q0 = max(BAND / 2, min(n_t / 2 - BAND / 2, q0));
            q0s = q0;
            const float phi = atan2f(m[1], m[0]);
            const float p = exp10f(m[3] / 64.f);
            const float amp = m[4] > 0.f ? sqrtf(p / m[4]) : 0.f;
            sc[0] = amp * cosf(0.5f * phi);
            sc[1] = amp * sinf(0.5f * phi);
            if (centres) centres[inst] = q0;
        }
    }
    __syncthreads();
    for (int k = t; k < 2 * BAND; k += blockDim.x) {
        const float a = fmaxf(row[k], 0.f);
        coef[k] = make_float2(a * sc[0], a * sc[1]);   /* every pair c_q c_-q has phase Phi */
    }
    __syncthreads();
    const int q0 = q0s;
    const unsigned long long mask = (unsigned long long)n_t - 1;
    const float inv = 2.0f / (float)n_t;
    for (int n = blockIdx.x * blockDim.x + t; n < n_t; n += gridDim.x * blockDim.x) {
        float sr, cr;
        sincospif((float)((unsigned long long)n & mask) * inv, &sr, &cr);
        float ar = 0.f, ai = 0.f;
        for (int k0 = 0; k0 < 2 * BAND; k0 += 16) {
            const long long q = (k0 < BAND) ? (long long)q0 - BAND / 2 + k0 : -(long long)q0 - BAND / 2 + (k0 - BAND);
            const unsigned long long mm = ((unsigned long long)(q + 4LL * n_t) * (unsigned long long)n) & mask;
            float s, c;
            sincospif((float)mm * inv, &s, &c);
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float2 v = coef[k0 + j];
                ar += v.x * c - v.y * s;
                ai += v.x * s + v.y * c;
                const float c2 = c * cr - s * sr;
                s = s * cr + c * sr;
                c = c2;
            }
        }
        fields[inst * n_t + n] = make_float2(scale * ar, scale * ai);
    }
}

}  /* namespace */

extern "C" cuopo_status cuopo_fields_from_bands(const float *pred, int count, int n_t, double scale, void *fields,
                                                int *centres, void *stream)
{
    if (!pred || !fields || count < 1) return cuopo_fail(CUOPO_EINVAL, "fields_from_bands: bad argument");
    if (count > 65535) return cuopo_fail(CUOPO_EINVAL, "fields_from_bands: at most 65535 instances per call");
    if (n_t < 2 * BAND || (n_t & (n_t - 1)))
        return cuopo_fail(CUOPO_EINVAL, "fields_from_bands: n_t must be a power of 2 >= 256");
    dim3 grid((unsigned)((n_t + 255) / 256), (unsigned)count);
    fields_from_bands_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(pred, n_t, (float)scale, (float2 *)fields,
                                                                     centres);
    return launch_check(cudaGetLastError(), "fields_from_bands");
}
