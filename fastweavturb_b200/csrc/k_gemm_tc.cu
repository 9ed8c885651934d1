// k_gemm_tc.cu -- BF16 GEMM on the 5th-generation tensor cores (tcgen05) for the learned
// surrogate: C[M x N] (FP32) = A[M x K] . B[N x K]^T, A and B row-major BF16 (K contiguous).
//
// One CTA of 128 threads computes a 128 x BN tile of C (BN = 16..256, a multiple of 16).
// Per K chunk of 64 the threads stage A and B in shared memory in the no-swizzle K-major
// "core matrix" layout the MMA reads (8 rows x 16 bytes per core matrix, the two core matrices
// of one K=16 step LBO bytes apart, row groups SBO bytes apart); one thread issues four
// tcgen05.mma (M=128, N=BN, K=16, FP32 accumulation in tensor memory) and commits them to an
// mbarrier; after the last chunk the four warps read their 32 accumulator lanes each with
// tcgen05.ld and store C.  Every wait is bounded: on a timeout the CTA sets *err, still frees
// its tensor memory and returns.
//
// The surrogate's matrices are small (width <= 256, batch a few thousand), so the kernel
// favours simplicity over a TMA / multi-stage pipeline.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fwt_internal.h"

namespace fwt {

constexpr int kGemmBM = 128, kGemmBK = 64, kGemmThreads = 128;

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // start address, leading and stride byte offsets in 16-byte units; bits 46-47 = 1 (the
    // sm_100 descriptor version); layout type 0 (no swizzle) in bits 61-63, base offset 0
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t umma_idesc_bf16(int M, int N)
{
    // D F32 (bits 4-5 = 1), A BF16 (bits 7-9 = 1), B BF16 (bits 10-12 = 1), both K-major,
    // N >> 3 in bits 17-22, M >> 4 in bits 24-28
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool gemm_mbar_wait(uint32_t bar, uint32_t phase)
{
    for (int it = 0; it < (1 << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// byte offset of element (row r, k) of a rows x 64 K-major no-swizzle tile
__device__ __forceinline__ uint32_t core_off(int r, int k8, int rows)
{
    return (uint32_t)(k8 * rows * 16 + (r >> 3) * 128 + (r & 7) * 16);
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_tc_kernel(const __nv_bfloat16 *__restrict__ A,
                                                                     const __nv_bfloat16 *__restrict__ B,
                                                                     float *__restrict__ C, int M, int N, int K,
                                                                     int ldc, int *__restrict__ err)
{
    constexpr int kCols = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));   // TMEM columns
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sA = smem;                                  // 128 x 64 bf16 = 16 KB
    unsigned char *sB = smem + kGemmBM * kGemmBK * 2;          // BN x 64 bf16
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(&bar);
    if (warp == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&tmem_base);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t sA_a = (uint32_t)__cvta_generic_to_shared(sA), sB_a = (uint32_t)__cvta_generic_to_shared(sB);
    const uint32_t idesc = umma_idesc_bf16(kGemmBM, BN);
    uint32_t phase = 0;
    bool ok = true;
    const int nk = K / kGemmBK;
    for (int kc = 0; kc < nk && ok; ++kc) {
        // stage A (128 rows) and B (BN rows): one 16-byte core-matrix row per uint4
        for (int i = tid; i < kGemmBM * 8; i += kGemmThreads) {
            const int r = i >> 3, k8 = i & 7;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m0 + r < M) v = *reinterpret_cast<const uint4 *>(A + (size_t)(m0 + r) * K + kc * kGemmBK + k8 * 8);
            *reinterpret_cast<uint4 *>(sA + core_off(r, k8, kGemmBM)) = v;
        }
        for (int i = tid; i < BN * 8; i += kGemmThreads) {
            const int r = i >> 3, k8 = i & 7;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (n0 + r < N) v = *reinterpret_cast<const uint4 *>(B + (size_t)(n0 + r) * K + kc * kGemmBK + k8 * 8);
            *reinterpret_cast<uint4 *>(sB + core_off(r, k8, BN)) = v;
        }
        // the MMA reads shared memory through the async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kGemmBK / 16; ++kk) {
                // K = 16 covers the core matrices 2kk and 2kk+1 along K
                const uint64_t da = umma_smem_desc(sA_a + (uint32_t)(2 * kk * kGemmBM * 16), kGemmBM * 16, 128);
                const uint64_t db = umma_smem_desc(sB_a + (uint32_t)(2 * kk * BN * 16), BN * 16, 128);
                const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar_a)
                         : "memory");
        }
        ok = gemm_mbar_wait(bar_a, phase);
        phase ^= 1u;
        ok = __syncthreads_and(ok) != 0;   // uniform: the next chunk overwrites the staged tiles
    }
    if (!ok) {
        if (tid == 0) atomicOr(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: warp w reads accumulator lanes 32w .. 32w+31 (rows m0 + 32w + lane)
        const int row = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 8) {
            uint32_t v[8];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                           "=r"(v[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (n0 + c0 + j < N) C[(size_t)row * ldc + n0 + c0 + j] = __uint_as_float(v[j]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// C = A . B^T on the tensor cores.  K must be a multiple of 64 (zero-pad), N <= 256 per tile
// column (any N: tiles of BN columns), M any.  ldc >= N.
int gemm_bf16_tc(const void *A, const void *B, float *C, int M, int N, int K, int ldc, int *d_err, cudaStream_t st)
{
    if (M < 1 || N < 1 || K < kGemmBK || K % kGemmBK) return fail(FWT_E_ARG, "gemm: K must be a positive multiple of 64");
    if (((uintptr_t)A | (uintptr_t)B) & 15) return fail(FWT_E_ARG, "gemm: operands must be 16-byte aligned");
    const int BN = N > 128 ? 256 : (N > 64 ? 128 : 64);
    const dim3 grid((unsigned)((M + kGemmBM - 1) / kGemmBM), (unsigned)((N + BN - 1) / BN));
    const size_t smem = (size_t)(kGemmBM + BN) * kGemmBK * 2;
#define FWT_GEMM(BNV)                                                                                         \
    do {                                                                                                      \
        FWT_CUDA(cudaFuncSetAttribute(gemm_bf16_tc_kernel<BNV>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                      (int)smem));                                                            \
        gemm_bf16_tc_kernel<BNV><<<grid, kGemmThreads, smem, st>>>((const __nv_bfloat16 *)A,                 \
                                                                     (const __nv_bfloat16 *)B, C, M, N, K, ldc, \
                                                                     d_err);                                  \
    } while (0)
    if (BN == 256) FWT_GEMM(256);
    else if (BN == 128) FWT_GEMM(128);
    else FWT_GEMM(64);
#undef FWT_GEMM
    FWT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace fwt
