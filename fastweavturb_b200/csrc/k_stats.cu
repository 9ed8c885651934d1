// k_stats.cu -- statistics of the woven field:
//   minmax_kernel      component ranges, bit-exact (order-preserving integer atomics)
//   pdf_kernel         REAL(4) bin search of subroutine.f90:22-34 as a binary search on
//                      the bins' upper edges, integer shared-memory histograms
//   sp_kernel          longitudinal increments at separations r, moments p = 1..pmax
//                      accumulated in FP64 (subroutine.f90:64-129); lines staged in shared
//                      memory so each velocity component is read from HBM once
//   field_wh_kernel    downsampled |omega| and omega.u (tube.f90:1055-1071)
#include "k_common.cuh"

#include <cmath>

namespace fwt {

// Component range, exact in the field's precision: FP32 values through order-preserving
// 32-bit atomics, FP64 values through 64-bit ones (mm: two words of the value's width).
template <typename Real>
__global__ void minmax_kernel(const Real *__restrict__ a, size_t n, void *__restrict__ mm)
{
    Real mn = (Real)3.4e38f, mx = (Real)-3.4e38f;
    if (sizeof(Real) == 8) {
        mn = (Real)1.7e308;
        mx = (Real)-1.7e308;
    }
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const Real v = a[i];
        mn = fmin(mn, v);
        mx = fmax(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if constexpr (sizeof(Real) == 8) {
            unsigned long long *m = (unsigned long long *)mm;
            atomicMin(m, d2ord((double)mn));
            atomicMax(m + 1, d2ord((double)mx));
        } else {
            uint32_t *m = (uint32_t *)mm;
            atomicMin(m, f2ord((float)mn));
            atomicMax(m + 1, f2ord((float)mx));
        }
    }
}

// v = (float)((double)x * s); bin = first l with v < hi[l], counted if lo[l] <= v
template <typename Real>
__global__ void __launch_bounds__(256) pdf_kernel(const Real *__restrict__ a, size_t n, double s,
                                                  const float *__restrict__ lo, const float *__restrict__ hi, int nbins,
                                                  unsigned long long *__restrict__ counts)
{
    extern __shared__ unsigned char smem[];
    float *s_hi = (float *)smem;
    float *s_lo = s_hi + nbins;
    uint32_t *s_cnt = (uint32_t *)(s_lo + nbins);
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
        s_hi[i] = hi[i];
        s_lo[i] = lo[i];
        s_cnt[i] = 0;
    }
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float v = (float)((double)a[i] * s);
        int lo_i = 0, hi_i = nbins;   // first l in [0, nbins) with v < s_hi[l]
        while (lo_i < hi_i) {
            const int mid = (lo_i + hi_i) >> 1;
            if (v < s_hi[mid]) hi_i = mid;
            else lo_i = mid + 1;
        }
        if (lo_i < nbins && s_lo[lo_i] <= v) atomicAdd(s_cnt + lo_i, 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (s_cnt[i]) atomicAdd(counts + i, (unsigned long long)s_cnt[i]);
}

// Structure functions along one axis.  A block stages W lines of length N in shared memory
// as [pos][line] (padded), in the field's own precision, then warp w accumulates, for its
// separations, sum (du * s)^p for p = 1..PMAX in registers.  W = 32 lines for FP32 fields and
// 16 for FP64 (a 1024-point FP64 group still fits one block's shared memory); groups at the end
// of an axis may hold fewer lines, so any N works.  axis 0: u_x along x; 1: u_y along y;
// 2: u_z along z.
template <typename Real>
__host__ __device__ constexpr int sp_lines(int N)
{
    return N < (sizeof(Real) == 8 ? 16 : 32) ? N : (sizeof(Real) == 8 ? 16 : 32);
}

// The field is a box n0 x n1 x n2 (x fastest) whose extent along `axis` is the line length N:
// the whole grid, or a z-slab (axes 0, 1) or y-pencil (axis 2) of a grid split over GPUs.
template <typename Real, int PMAX, int MPW>
__global__ void __launch_bounds__(256) sp_kernel(const Real *__restrict__ u, int N, int n0, int n1, int n2, int axis,
                                                 double s, const int *__restrict__ rs, int nr,
                                                 double *__restrict__ Sp)
{
    extern __shared__ __align__(16) unsigned char sp_smem[];
    Real *tile = reinterpret_cast<Real *>(sp_smem);   // N x (W + 1)
    const int W = sp_lines<Real>(N);
    const int ld = W + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double acc[MPW][PMAX];
#pragma unroll
    for (int a = 0; a < MPW; ++a)
#pragma unroll
        for (int p = 0; p < PMAX; ++p) acc[a][p] = 0.0;
    int rr[MPW];
#pragma unroll
    for (int a = 0; a < MPW; ++a) {
        const int m = warp + a * nwarps;
        rr[a] = m < nr ? rs[m] % N : -1;
    }
    // axis 0: groups of W consecutive x-rows (row = y + n1 z); axes 1, 2: groups of W
    // consecutive x at fixed z (axis 1) or fixed y (axis 2)
    const int xgroups = (n0 + W - 1) / W;
    const int64_t nrows = (int64_t)n1 * n2;
    const int64_t ngroups = axis == 0 ? (nrows + W - 1) / W : (int64_t)xgroups * (axis == 1 ? n2 : n1);
    for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        __syncthreads();
        int nl;   // lines of this group
        if (axis == 0) {
            const int64_t row0 = g * W;
            nl = (int)min((int64_t)W, nrows - row0);
            for (int e = threadIdx.x; e < N * nl; e += blockDim.x) {
                const int x = e % N, l = e / N;
                tile[x * ld + l] = u[(size_t)(row0 + l) * n0 + x];
            }
        } else {
            const int xg = (int)(g % xgroups), o = (int)(g / xgroups);
            const int x0 = xg * W;
            nl = min(W, n0 - x0);
            for (int e = threadIdx.x; e < N * W; e += blockDim.x) {
                const int l = e % W, pos = e / W;
                if (l >= nl) continue;
                size_t gi;
                if (axis == 1) gi = (size_t)(x0 + l) + (size_t)n0 * ((size_t)pos + (size_t)n1 * o);
                else gi = (size_t)(x0 + l) + (size_t)n0 * ((size_t)o + (size_t)n1 * pos);
                tile[pos * ld + l] = u[gi];
            }
        }
        __syncthreads();
        if (lane < nl) {
#pragma unroll
            for (int a = 0; a < MPW; ++a) {
                const int r = rr[a];
                if (r < 0) continue;
                for (int pos = 0; pos < N; ++pos) {
                    int q = pos + r;
                    if (q >= N) q -= N;
                    const double du = ((double)tile[q * ld + lane] - (double)tile[pos * ld + lane]) * s;
                    double pw = du;
#pragma unroll
                    for (int p = 0; p < PMAX; ++p) {
                        acc[a][p] += pw;
                        pw *= du;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < MPW; ++a) {
        const int m = warp + a * nwarps;
        if (m >= nr) continue;
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
            const double v = warp_sum(acc[a][p]);
            if (lane == 0) atomicAdd(Sp + p * nr + m, v);
        }
    }
}

template <typename Real>
__global__ void field_wh_kernel(const Real *__restrict__ w, const Real *__restrict__ u, int N, int nd, double s,
                                float *__restrict__ out)
{
    const size_t n3 = (size_t)N * N * N;
    const int rd = N / nd;
    const size_t m3 = (size_t)nd * nd * nd;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m3; q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % nd), j = (int)((q / nd) % nd), k = (int)(q / ((size_t)nd * nd));
        // data_box(i, j, k) = field(i*r_d, j*r_d, k*r_d), 1-based
        const size_t g = (size_t)((i + 1) * rd - 1) + (size_t)N * ((size_t)((j + 1) * rd - 1) + (size_t)N * ((k + 1) * rd - 1));
        const double wx = (double)w[g] * s, wy = (double)w[g + n3] * s, wz = (double)w[g + 2 * n3] * s;
        const double ux = (double)u[g] * s, uy = (double)u[g + n3] * s, uz = (double)u[g + 2 * n3] * s;
        out[q] = (float)sqrt(wx * wx + wy * wy + wz * wz);
        out[q + m3] = (float)(wx * ux + wy * uy + wz * uz);
    }
}

__global__ void mm_init2(void *mm, int n, int wide)
{
    const int i = threadIdx.x;
    if (i >= n) return;
    if (wide) ((unsigned long long *)mm)[i] = (i & 1) ? 0ull : ~0ull;
    else ((uint32_t *)mm)[i] = (i & 1) ? 0u : 0xffffffffu;
}

static unsigned grid_for(Ctx *c, size_t n, int per_sm = 8)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * per_sm));
}

// raw component ranges of u (which = 1) or omega (which = 0), exact in the field's precision
int stats_minmax(Ctx *c, int which)
{
    const size_t n3 = field_elems(c);
    void *f = which ? c->b_u.p : c->b_w.p;
    const bool wide = c->p.precision == 64;
    FWT_TRY(buf_reserve(c, c->scratch[19], 128));
    char *mm = (char *)c->scratch[19].p + 16;
    const int km = kt_begin(c, KT_STATS);
    mm_init2<<<1, 32, 0, c->stream>>>(mm, 6, wide ? 1 : 0);
    for (int d = 0; d < 3; ++d) {
        if (wide)
            minmax_kernel<double><<<grid_for(c, n3), 256, 0, c->stream>>>((const double *)f + d * n3, n3, mm + 16 * d);
        else
            minmax_kernel<float><<<grid_for(c, n3), 256, 0, c->stream>>>((const float *)f + d * n3, n3, mm + 8 * d);
    }
    kt_end(c, km);
    c->launches += 4;
    FWT_CUDA(cudaGetLastError());
    unsigned long long h[6];
    FWT_CUDA(cudaMemcpyAsync(h, mm, wide ? 48 : 24, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    std::vector<double> &mn = which ? c->umin : c->wmin, &mx = which ? c->umax : c->wmax;
    mn.assign(3, 0.0);
    mx.assign(3, 0.0);
    const uint32_t *h32 = (const uint32_t *)h;
    for (int d = 0; d < 3; ++d) {
        mn[d] = wide ? ord2d(h[2 * d]) : (double)ord2f(h32[2 * d]);
        mx[d] = wide ? ord2d(h[2 * d + 1]) : (double)ord2f(h32[2 * d + 1]);
    }
    if (which) c->umm_valid = true;
    else c->wmm_valid = true;
    return 0;
}

int stats_normalise(Ctx *c)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "normalise: not available on a z-slab context");
    if (!c->have_u) return fail(FWT_E_STATE, "normalise before Biot-Savart");
    // Etot = sum u.u dv / 2 / (2pi)^3 = 1/2 <u^2>; up = sqrt(2 Etot / 3) (tube.f90:1028-1030)
    c->Etot = c->Etot_raw;
    c->up = std::sqrt(2 * c->Etot / 3);
    c->enstrophy = c->enstrophy_raw / (c->up * c->up);
    c->normalised = true;
    return 0;
}

// host-side REAL(4) bin layout, identical to the reference's (subroutine.f90:12-20)
static void pdf_layout(float vmin, float vmax, int nbins, std::vector<float> &val, std::vector<float> &lo,
                       std::vector<float> &hi, float &bsz)
{
    bsz = (float)((float)(vmax - vmin) / (float)nbins);
    val.resize(nbins);
    lo.resize(nbins);
    hi.resize(nbins);
    const float half = (float)(0.5f * bsz);
    for (int l = 0; l < nbins; ++l) {
        const float prod = (float)((float)l * bsz);
        val[l] = (float)((double)vmin + 0.5 * (double)bsz + (double)prod);
        lo[l] = (float)(val[l] - half);
        hi[l] = (float)(val[l] + half);
    }
}

int stats_pdf(Ctx *c, int which, int comp, int nbins, float *val, float *pdf, uint64_t *counts)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "pdf: not available on a z-slab context");
    if (which != 0 && which != 1) return fail(FWT_E_ARG, "pdf: which must be 0 (u) or 1 (omega)");
    if (comp < -1 || comp > 2) return fail(FWT_E_ARG, "pdf: component must be -1..2");
    if (nbins < 1 || nbins > 8192) return fail(FWT_E_ARG, "pdf: nbins must be 1..8192");
    if (!c->normalised) return fail(FWT_E_STATE, "pdf before normalisation");
    const bool is_u = which == 0;
    if (is_u && !c->umm_valid) FWT_TRY(stats_minmax(c, 1));
    if (!is_u && !c->wmm_valid) FWT_TRY(stats_minmax(c, 0));
    const std::vector<double> &mn = is_u ? c->umin : c->wmin, &mx = is_u ? c->umax : c->wmax;
    const double s = 1.0 / c->up;
    double rmin = 1.7e308, rmax = -1.7e308;
    for (int d = 0; d < 3; ++d) {
        if (comp >= 0 && d != comp) continue;
        rmin = std::min(rmin, mn[d]);
        rmax = std::max(rmax, mx[d]);
    }
    // range of the scaled REAL(4) values (float)(x s): rounding is monotone, so it is the
    // rounded scaled range of the exact raw values
    const float vmin = (float)(rmin * s), vmax = (float)(rmax * s);
    std::vector<float> hval, hlo, hhi;
    float bsz;
    pdf_layout(vmin, vmax, nbins, hval, hlo, hhi, bsz);
    FWT_TRY(buf_reserve(c, c->scratch[10], sizeof(float) * 2 * nbins + sizeof(unsigned long long) * nbins + 64));
    float *d_lo = (float *)c->scratch[10].p, *d_hi = d_lo + nbins;
    unsigned long long *d_cnt = (unsigned long long *)(((uintptr_t)(d_hi + nbins) + 15) & ~(uintptr_t)15);
    FWT_CUDA(cudaMemcpyAsync(d_lo, hlo.data(), sizeof(float) * nbins, cudaMemcpyHostToDevice, c->stream));
    FWT_CUDA(cudaMemcpyAsync(d_hi, hhi.data(), sizeof(float) * nbins, cudaMemcpyHostToDevice, c->stream));
    FWT_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * nbins, c->stream));
    const size_t n3 = field_elems(c);
    const void *f = is_u ? c->b_u.p : c->b_w.p;
    const size_t shb = sizeof(float) * 2 * nbins + sizeof(uint32_t) * nbins;
    // 8192 bins take 96 KB of shared memory, above the default 48 KB: the limit is raised to
    // the device's opt-in maximum, the same value for every context (the attribute belongs to
    // the kernel, for the whole process)
    int optin = 0;
    FWT_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    if (shb > (size_t)optin) return fail(FWT_E_RANGE, "pdf: bins exceed one block's shared memory");
    if (c->p.precision == 64)
        FWT_CUDA(cudaFuncSetAttribute(pdf_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    else
        FWT_CUDA(cudaFuncSetAttribute(pdf_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
    const int km = kt_begin(c, KT_STATS);
    for (int d = 0; d < 3; ++d) {
        if (comp >= 0 && d != comp) continue;
        if (c->p.precision == 64)
            pdf_kernel<double><<<grid_for(c, n3, 4), 256, shb, c->stream>>>((const double *)f + d * n3, n3, s, d_lo,
                                                                            d_hi, nbins, d_cnt);
        else
            pdf_kernel<float><<<grid_for(c, n3, 4), 256, shb, c->stream>>>((const float *)f + d * n3, n3, s, d_lo,
                                                                           d_hi, nbins, d_cnt);
        c->launches += 1;
    }
    kt_end(c, km);
    FWT_CUDA(cudaGetLastError());
    std::vector<unsigned long long> hc(nbins);
    FWT_CUDA(cudaMemcpyAsync(hc.data(), d_cnt, sizeof(unsigned long long) * nbins, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    // pdf_v(l)/(bin_size*nx*ny*nzp*nproc), left to right in REAL(4) (subroutine.f90:38)
    const int N = c->p.N;
    const int nz_eff = comp < 0 ? 3 * N : N;
    float den = bsz;
    den = (float)(den * (float)N);
    den = (float)(den * (float)N);
    den = (float)(den * (float)nz_eff);
    for (int l = 0; l < nbins; ++l) {
        if (val) val[l] = hval[l];
        if (pdf) pdf[l] = (float)((float)hc[l] / den);
        if (counts) counts[l] = hc[l];
    }
    return 0;
}

int stats_sp(Ctx *c, int pmax, const int *r, int nr, double *Sp)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "S_p: not available on a z-slab context");
    if (!c->normalised) return fail(FWT_E_STATE, "structure functions before normalisation");
    if (pmax < 1 || pmax > 10) return fail(FWT_E_ARG, "Sp: pmax must be 1..10");
    if (nr < 1 || nr > 64) return fail(FWT_E_ARG, "Sp: nr must be 1..64");
    const int N = c->p.N;
    const bool f64 = c->p.precision == 64;
    const int W = f64 ? sp_lines<double>(N) : sp_lines<float>(N);
    for (int m = 0; m < nr; ++m)
        if (r[m] < 0) return fail(FWT_E_ARG, "Sp: negative separation");
    FWT_TRY(buf_reserve(c, c->scratch[9], sizeof(int) * 64 + sizeof(double) * 10 * 64 + 64));
    int *d_r = (int *)c->scratch[9].p;
    double *d_sp = (double *)((char *)c->scratch[9].p + 256);
    FWT_CUDA(cudaMemcpyAsync(d_r, r, sizeof(int) * nr, cudaMemcpyHostToDevice, c->stream));
    FWT_CUDA(cudaMemsetAsync(d_sp, 0, sizeof(double) * 10 * nr, c->stream));
    const size_t n3 = field_elems(c);
    const double s = 1.0 / c->up;
    const size_t shb = (f64 ? sizeof(double) : sizeof(float)) * (size_t)N * (W + 1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int64_t groups = ((int64_t)N * N + W - 1) / W;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(groups, (int64_t)sms * 4));
    const int mpw = (nr + 7) / 8;
    // The dynamic shared-memory limit is a property of the kernel for the whole process: every
    // context sets the same value, the device's opt-in maximum, so that contexts of different N
    // on concurrent host threads never lower it under another's launch.
    int optin = 0;
    FWT_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    if (shb > (size_t)optin) return fail(FWT_E_RANGE, "Sp: N too large for one block's shared memory");
    const int km = kt_begin(c, KT_STATS);
#define FWT_SP(REAL, MPW)                                                                                        \
    do {                                                                                                         \
        auto k = sp_kernel<REAL, 10, MPW>;                                                                       \
        FWT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));                  \
        for (int ax = 0; ax < 3; ++ax)                                                                           \
            k<<<blocks, 256, shb, c->stream>>>((const REAL *)c->b_u.p + ax * n3, N, N, N, N, ax, s, d_r, nr, d_sp); \
    } while (0)
    if (c->p.precision == 64) {
        if (mpw <= 1) FWT_SP(double, 1); else if (mpw <= 2) FWT_SP(double, 2); else if (mpw <= 4) FWT_SP(double, 4);
        else FWT_SP(double, 8);
    } else {
        if (mpw <= 1) FWT_SP(float, 1); else if (mpw <= 2) FWT_SP(float, 2); else if (mpw <= 4) FWT_SP(float, 4);
        else FWT_SP(float, 8);
    }
#undef FWT_SP
    kt_end(c, km);
    c->launches += 3;
    FWT_CUDA(cudaGetLastError());
    std::vector<double> h(10 * nr);
    FWT_CUDA(cudaMemcpyAsync(h.data(), d_sp, sizeof(double) * 10 * nr, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    const double inv = 1.0 / ((double)N * N * N * 3.0);
    for (int p = 0; p < pmax; ++p)
        for (int m = 0; m < nr; ++m) Sp[p * nr + m] = h[p * nr + m] * inv;
    return 0;
}

int stats_field_wh(Ctx *c, float *host_out)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "field output: not available on a z-slab context");
    if (!c->normalised) return fail(FWT_E_STATE, "field output before normalisation");
    const int N = c->p.N, nd = c->p.N_downsample;
    if (nd < 1 || N % nd) return fail(FWT_E_ARG, "N_downsample must divide N");
    const size_t m3 = (size_t)nd * nd * nd, n3 = field_elems(c);
    FWT_TRY(buf_reserve(c, c->scratch[8], sizeof(float) * 2 * m3));
    float *d = (float *)c->scratch[8].p;
    const double s = 1.0 / c->up;
    const int km = kt_begin(c, KT_STATS);
    if (c->p.precision == 64)
        field_wh_kernel<double><<<grid_for(c, m3), 256, 0, c->stream>>>((const double *)c->b_w.p,
                                                                        (const double *)c->b_u.p, N, nd, s, d);
    else
        field_wh_kernel<float><<<grid_for(c, m3), 256, 0, c->stream>>>((const float *)c->b_w.p, (const float *)c->b_u.p,
                                                                       N, nd, s, d);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    (void)n3;
    if (host_out) {
        FWT_CUDA(cudaMemcpyAsync(host_out, d, sizeof(float) * 2 * m3, cudaMemcpyDeviceToHost, c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
    }
    return 0;
}

int stats_copy_field(Ctx *c, int which, int comp, double *host)
{
    if (which != 0 && which != 1) return fail(FWT_E_ARG, "copy_field: which must be 0 (omega) or 1 (u)");
    if (comp < 0 || comp > 2) return fail(FWT_E_ARG, "copy_field: component must be 0..2");
    if (which == 0 && !c->have_w) return fail(FWT_E_STATE, "omega not built");
    if (which == 1 && !c->have_u) return fail(FWT_E_STATE, "u not built");
    const size_t n3 = field_elems(c);
    const double s = c->normalised ? 1.0 / c->up : 1.0;
    const void *f = which ? c->b_u.p : c->b_w.p;
    if (c->p.precision == 64) {
        FWT_CUDA(cudaMemcpyAsync(host, (const double *)f + comp * n3, sizeof(double) * n3, cudaMemcpyDeviceToHost,
                                 c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
        if (s != 1.0)
            for (size_t i = 0; i < n3; ++i) host[i] = host[i] * s;
    } else {
        std::vector<float> tmp(n3);
        FWT_CUDA(cudaMemcpyAsync(tmp.data(), (const float *)f + comp * n3, sizeof(float) * n3, cudaMemcpyDeviceToHost,
                                 c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < n3; ++i) host[i] = (double)tmp[i] * s;
    }
    return 0;
}

// S_p sums of one velocity component on a box (a z-slab or y-pencil of a grid split over GPUs):
// sums[p * nr + m] = sum over the box's lines along `axis` of (du s)^(p+1), du the increment at
// separation r[m]; the line axis must span the grid (extent N).  Not normalised: the caller adds
// the three components' sums over all boxes and divides by 3 N^3, as stats_sp does.
int stats_sp_block(Ctx *c, const void *u, int n0, int n1, int n2, int axis, double s, const int *r, int nr,
                   double *sums)
{
    const int N = c->p.N;
    if (axis < 0 || axis > 2) return fail(FWT_E_ARG, "sp_block: axis must be 0..2");
    const int ext[3] = {n0, n1, n2};
    if (ext[axis] != N || n0 < 1 || n1 < 1 || n2 < 1) return fail(FWT_E_ARG, "sp_block: the line axis must span N");
    if (nr < 1 || nr > 64) return fail(FWT_E_ARG, "sp_block: nr must be 1..64");
    for (int m = 0; m < nr; ++m)
        if (r[m] < 0) return fail(FWT_E_ARG, "sp_block: negative separation");
    const bool f64 = c->p.precision == 64;
    const int W = f64 ? sp_lines<double>(N) : sp_lines<float>(N);
    FWT_TRY(buf_reserve(c, c->scratch[9], sizeof(int) * 64 + sizeof(double) * 10 * 64 + 64));
    int *d_r = (int *)c->scratch[9].p;
    double *d_sp = (double *)((char *)c->scratch[9].p + 256);
    FWT_CUDA(cudaMemcpyAsync(d_r, r, sizeof(int) * nr, cudaMemcpyHostToDevice, c->stream));
    FWT_CUDA(cudaMemsetAsync(d_sp, 0, sizeof(double) * 10 * nr, c->stream));
    const size_t shb = (f64 ? sizeof(double) : sizeof(float)) * (size_t)N * (W + 1);
    int optin = 0;
    FWT_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev));
    if (shb > (size_t)optin) return fail(FWT_E_RANGE, "sp_block: N too large for one block's shared memory");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((int64_t)n0 * n1 * n2 / N / W + 1,
                                                                             (int64_t)sms * 4));
    const int mpw = (nr + 7) / 8;
    const int km = kt_begin(c, KT_STATS);
#define FWT_SPB(REAL, MPW)                                                                                       \
    do {                                                                                                         \
        auto k = sp_kernel<REAL, 10, MPW>;                                                                       \
        FWT_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin));                  \
        k<<<blocks, 256, shb, c->stream>>>((const REAL *)u, N, n0, n1, n2, axis, s, d_r, nr, d_sp);              \
    } while (0)
    if (f64) {
        if (mpw <= 1) FWT_SPB(double, 1); else if (mpw <= 2) FWT_SPB(double, 2); else if (mpw <= 4) FWT_SPB(double, 4);
        else FWT_SPB(double, 8);
    } else {
        if (mpw <= 1) FWT_SPB(float, 1); else if (mpw <= 2) FWT_SPB(float, 2); else if (mpw <= 4) FWT_SPB(float, 4);
        else FWT_SPB(float, 8);
    }
#undef FWT_SPB
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    FWT_CUDA(cudaMemcpyAsync(sums, d_sp, sizeof(double) * 10 * nr, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

}  // namespace fwt
