// k_pdf_noalloc.cu -- fwt_pdf_noalloc: the PDF of a device field with no memory allocation.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or allocator hook
// that must not re-enter the allocator, code between the capture of a fixed memory plan and
// its replay, or embedders whose device memory is owned by someone else and budgeted to the
// byte.  For them this entry point keeps all of its scratch -- the value range, the bin edges
// and the bin counts -- in one file-scope static device array of fixed size
// (kPdfNoAllocMaxBins bins, about 128 KB), which every GPU that loads the library holds until
// the process exits.  The caller passes the input field (device memory) and host output
// arrays; nothing is allocated, by this code or by any library it calls.
//
// Sharing: every call uses the same array and it keeps the last call's contents, so the
// counts and the range are cleared at the start of each call.  Calls that overlap on the GPU
// (two streams, two host threads on one device) race on the array and give wrong results;
// serialise them.
//
// Set-up: the array's host-side name is only a stand-in, not a device address.  Every call,
// with the caller's device current, looks the address up with cudaGetSymbolAddress (a lookup in
// the already loaded module, so a context made anew after cudaDeviceReset gets its own array).
// The first call in each CUDA context also loads every kernel of this entry point (CUDA loads
// kernels lazily, and a load allocates device memory) and sets their shared-memory limit once,
// so that later calls -- FP32 or FP64, any bin count -- allocate nothing; that first call
// should come before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <algorithm>
#include <mutex>

#include "k_common.cuh"

namespace fwt {

constexpr int kPdfNoAllocMaxBins = 8192;

struct PdfScratch {
    uint32_t mm[2];                                // ordered-int min, max of the scaled values
    float vmin, vmax, bsz, pad[3];
    float lo[kPdfNoAllocMaxBins];                  // bin lower edges (REAL(4) layout)
    float hi[kPdfNoAllocMaxBins];                  // bin upper edges
    unsigned long long cnt[kPdfNoAllocMaxBins];    // bin counts
};

static __device__ __align__(256) PdfScratch g_pdf_scratch;

template <typename Real>
__global__ void na_clear_minmax_kernel(const Real *__restrict__ a, size_t n, double s, int nbins,
                                       PdfScratch *__restrict__ S)
{
    // block 0 clears the counts; every block reduces its share of the range
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < nbins; i += blockDim.x) S->cnt[i] = 0ull;
    float mn = 3.4e38f, mx = -3.4e38f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = (float)((double)a[i] * s);
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&S->mm[0], f2ord(mn));
        atomicMax(&S->mm[1], f2ord(mx));
    }
}

__global__ void na_init_kernel(PdfScratch *__restrict__ S)
{
    if (threadIdx.x == 0) {
        S->mm[0] = 0xffffffffu;
        S->mm[1] = 0u;
    }
}

// bin edges of the reference's REAL(4) layout (subroutine.f90:12-20), no contracted arithmetic
__global__ void na_edges_kernel(int nbins, PdfScratch *__restrict__ S)
{
    const float vmin = ord2f(S->mm[0]), vmax = ord2f(S->mm[1]);
    const float bsz = __fdiv_rn(__fsub_rn(vmax, vmin), (float)nbins);
    const float half = __fmul_rn(0.5f, bsz);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->vmin = vmin;
        S->vmax = vmax;
        S->bsz = bsz;
    }
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nbins; l += gridDim.x * blockDim.x) {
        const float prod = __fmul_rn((float)l, bsz);
        const float val = (float)__dadd_rn(__dadd_rn((double)vmin, __dmul_rn(0.5, (double)bsz)), (double)prod);
        S->lo[l] = __fsub_rn(val, half);
        S->hi[l] = __fadd_rn(val, half);
    }
}

template <typename Real>
__global__ void __launch_bounds__(256) na_hist_kernel(const Real *__restrict__ a, size_t n, double s, int nbins,
                                                      PdfScratch *__restrict__ S)
{
    extern __shared__ unsigned char smem[];
    float *s_hi = (float *)smem;
    float *s_lo = s_hi + nbins;
    uint32_t *s_cnt = (uint32_t *)(s_lo + nbins);
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
        s_hi[i] = S->hi[i];
        s_lo[i] = S->lo[i];
        s_cnt[i] = 0;
    }
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = (float)((double)a[i] * s);
        int lo_i = 0, hi_i = nbins;   // first l with v < hi[l]
        while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i) >> 1;
            if (v < s_hi[mid]) hi_i = mid;
            else lo_i = mid + 1;
        }
        if (lo_i < nbins && s_lo[lo_i] <= v) atomicAdd(s_cnt + lo_i, 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (s_cnt[i]) atomicAdd(S->cnt + i, (unsigned long long)s_cnt[i]);
}

constexpr int kPdfNoAllocShmem = (int)(sizeof(float) * 2 + sizeof(uint32_t)) * kPdfNoAllocMaxBins;   // 96 KB

// The current CUDA context (the driver's cuCtxGetCurrent, reached through the runtime so that
// the library needs no link to libcuda); null if it cannot be had.
static void *current_context()
{
    using GetCtx = int (*)(void **);
    static GetCtx fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (GetCtx)f;
        cudaGetLastError();
    });
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// Load every kernel of the entry point and set the histogram kernels' shared-memory limit to
// the fixed maximum, once per context.
static int prepare_context()
{
    static std::mutex mu;
    static void *done[64] = {nullptr};
    static int ndone = 0;
    void *ctx = current_context();
    std::lock_guard<std::mutex> lk(mu);
    for (int i = 0; i < ndone; ++i)
        if (ctx && done[i] == ctx) return 0;
    cudaFuncAttributes fa;
    FWT_CUDA(cudaFuncGetAttributes(&fa, na_init_kernel));
    FWT_CUDA(cudaFuncGetAttributes(&fa, na_edges_kernel));
    FWT_CUDA(cudaFuncGetAttributes(&fa, na_clear_minmax_kernel<float>));
    FWT_CUDA(cudaFuncGetAttributes(&fa, na_clear_minmax_kernel<double>));
    FWT_CUDA(cudaFuncSetAttribute(na_hist_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPdfNoAllocShmem));
    FWT_CUDA(cudaFuncSetAttribute(na_hist_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPdfNoAllocShmem));
    if (ctx && ndone < 64) done[ndone++] = ctx;
    return 0;
}

// device address of g_pdf_scratch in the current context
static PdfScratch *scratch_addr(int *rc)
{
    *rc = prepare_context();
    if (*rc) return nullptr;
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_pdf_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        *rc = fail(FWT_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return nullptr;
    }
    return (PdfScratch *)p;
}

}  // namespace fwt

using namespace fwt;

extern "C" int fwt_pdf_noalloc(const void *d_data, int precision, int nx, int ny, int nz, double scale, int nbins,
                               void *stream, float *val, float *pdf, uint64_t *counts)
{
    if (!d_data || (!val && !pdf && !counts)) return fail(FWT_E_ARG, "pdf_noalloc: null argument");
    if (precision != 32 && precision != 64) return fail(FWT_E_ARG, "pdf_noalloc: precision must be 32 or 64");
    if (nx < 1 || ny < 1 || nz < 1) return fail(FWT_E_ARG, "pdf_noalloc: field dimensions must be positive");
    if (nbins < 1 || nbins > kPdfNoAllocMaxBins)
        return fail(FWT_E_RANGE, "pdf_noalloc: nbins must be 1.." + std::to_string(kPdfNoAllocMaxBins) +
                                     " (the size of its static scratch)");
    if (!(scale > 0)) return fail(FWT_E_ARG, "pdf_noalloc: scale must be positive");
    int dev = 0;
    FWT_CUDA(cudaGetDevice(&dev));
    int rc = 0;
    PdfScratch *S = scratch_addr(&rc);
    if (!S) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t n = (size_t)nx * ny * nz;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * 4));
    const size_t shb = sizeof(float) * 2 * nbins + sizeof(uint32_t) * nbins;
    na_init_kernel<<<1, 32, 0, st>>>(S);
    if (precision == 64) {
        na_clear_minmax_kernel<double><<<blocks, 256, 0, st>>>((const double *)d_data, n, scale, nbins, S);
        na_edges_kernel<<<(nbins + 255) / 256, 256, 0, st>>>(nbins, S);
        na_hist_kernel<double><<<blocks, 256, shb, st>>>((const double *)d_data, n, scale, nbins, S);
    } else {
        na_clear_minmax_kernel<float><<<blocks, 256, 0, st>>>((const float *)d_data, n, scale, nbins, S);
        na_edges_kernel<<<(nbins + 255) / 256, 256, 0, st>>>(nbins, S);
        na_hist_kernel<float><<<blocks, 256, shb, st>>>((const float *)d_data, n, scale, nbins, S);
    }
    FWT_CUDA(cudaGetLastError());
    // results to the caller's host arrays (plain copies, no staging buffers of ours)
    float rng[3];
    FWT_CUDA(cudaMemcpyAsync(rng, &S->vmin, sizeof(rng), cudaMemcpyDeviceToHost, st));
    if (counts) FWT_CUDA(cudaMemcpyAsync(counts, S->cnt, sizeof(uint64_t) * nbins, cudaMemcpyDeviceToHost, st));
    FWT_CUDA(cudaStreamSynchronize(st));
    // val and pdf in the reference's REAL(4) arithmetic (subroutine.f90:19,38)
    const float vmin = rng[0], bsz = rng[2];
    float den = bsz;
    den = (float)(den * (float)nx);
    den = (float)(den * (float)ny);
    den = (float)(den * (float)nz);
    if (val)
        for (int l = 0; l < nbins; ++l) {
            const float prod = (float)((float)l * bsz);
            val[l] = (float)((double)vmin + 0.5 * (double)bsz + (double)prod);
        }
    if (pdf) {
        // the counts pass through a small stack chunk when the caller wants no count array
        constexpr int kChunk = 256;
        uint64_t chunk[kChunk];
        for (int l0 = 0; l0 < nbins; l0 += kChunk) {
            const int m = std::min(kChunk, nbins - l0);
            const uint64_t *hc = counts ? counts + l0 : chunk;
            if (!counts) {
                FWT_CUDA(cudaMemcpyAsync(chunk, S->cnt + l0, sizeof(uint64_t) * m, cudaMemcpyDeviceToHost, st));
                FWT_CUDA(cudaStreamSynchronize(st));
            }
            for (int i = 0; i < m; ++i) pdf[l0 + i] = (float)((float)hc[i] / den);
        }
    }
    return 0;
}
