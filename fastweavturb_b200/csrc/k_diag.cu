// k_diag.cu -- the reference's field diagnostics that its main program keeps switched off
// (tube.f90:1027, 1050-1053, 1201-1202: the calls are commented out there):
//   vsf_phi_kernel        the scalar field phi = |omega| ("VSF deviation of vorticity
//                         magnitude", tube.f90:1201), when the caller gives none
//   vsf_deviation_kernel  cal_deviation (subroutine.f90:1519-1546): the mean over the grid of
//                         |omega . grad phi| / (|omega| |grad phi| + 1e-11), grad phi by the
//                         sixth-order central differences of the reference on the periodic
//                         grid (the ghost layers that wall_phiv, subroutine.f90:1575-1601,
//                         fills are the periodic images, read here by wrapped indices)
//   helicity_kernel       cal_helicity of (omega, u) (subroutine.f90:1550-1569): sum of
//                         omega . u times the cell volume
// Both reductions accumulate in FP64: per thread, per warp by shuffles, one atomic per warp.
#include "k_common.cuh"

namespace fwt {

namespace {

template <typename Real>
__global__ void vsf_phi_kernel(const Real *__restrict__ w, size_t n3, Real *__restrict__ phi)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
        const double a = (double)w[i], b = (double)w[i + n3], c = (double)w[i + 2 * n3];
        phi[i] = (Real)sqrt(a * a + b * b + c * c);
    }
}

// (9 f(-2) - f(-3) - 45 f(-1) + 45 f(1) - 9 f(2) + f(3)) / 60 / dx along one axis, in the
// reference's order of terms (subroutine.f90:1532-1534)
template <typename Real>
__device__ __forceinline__ double d6(const Real *__restrict__ f, size_t base, size_t stride, int i, int N, double dx)
{
    auto at = [&](int o) {
        int k = i + o;
        if (k < 0) k += N;
        if (k >= N) k -= N;
        return (double)f[base + (size_t)k * stride];
    };
    return (9.0 * at(-2) - at(-3) - 45.0 * at(-1) + 45.0 * at(1) - 9.0 * at(2) + at(3)) / 60.0 / dx;
}

template <typename Real>
__global__ void __launch_bounds__(256) vsf_deviation_kernel(const Real *__restrict__ w, const Real *__restrict__ phi,
                                                            int N, double dx, double *__restrict__ sum)
{
    const size_t n3 = (size_t)N * N * N, NN = (size_t)N * N;
    double acc = 0.0;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n3; g += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(g % N), j = (int)((g / N) % N), k = (int)(g / NN);
        const double gx = d6(phi, g - i, 1, i, N, dx);
        const double gy = d6(phi, g - (size_t)j * N, (size_t)N, j, N, dx);
        const double gz = d6(phi, g - (size_t)k * NN, NN, k, N, dx);
        const double graph = sqrt(gx * gx + gy * gy + gz * gz);
        const double a = (double)w[g], b = (double)w[g + n3], c = (double)w[g + 2 * n3];
        const double vorti = sqrt(a * a + b * b + c * c);
        const double dot = a * gx + b * gy + c * gz;
        acc += fabs(dot) / (vorti * graph + 1.0e-11);
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}

template <typename Real>
__global__ void helicity_kernel(const Real *__restrict__ w, const Real *__restrict__ u, size_t n3,
                                double *__restrict__ sum)
{
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x)
        acc += (double)w[i] * (double)u[i] + (double)w[i + n3] * (double)u[i + n3] +
               (double)w[i + 2 * n3] * (double)u[i + 2 * n3];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) atomicAdd(sum, acc);
}

unsigned diag_grid(const Ctx *c, size_t n)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)sms * 8));
}

}  // namespace

int diag_vsf_deviation(Ctx *c, const void *d_phi, double *deviation)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "VSF deviation: not available on a z-slab context");
    if (!c->have_w) return fail(FWT_E_STATE, "vsf_deviation: omega not built");
    const int N = c->p.N;
    const size_t n3 = field_elems(c);
    const bool f64 = c->p.precision == 64;
    FWT_TRY(buf_reserve(c, c->scratch[9], 64));
    double *d_sum = (double *)c->scratch[9].p;
    FWT_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(double), c->stream));
    const void *phi = d_phi;
    const unsigned g = diag_grid(c, n3);
    const int km = kt_begin(c, KT_STATS);
    if (!phi) {
        FWT_TRY(buf_reserve(c, c->scratch[8], n3 * real_bytes(c)));
        if (f64) vsf_phi_kernel<double><<<g, 256, 0, c->stream>>>((const double *)c->b_w.p, n3, (double *)c->scratch[8].p);
        else vsf_phi_kernel<float><<<g, 256, 0, c->stream>>>((const float *)c->b_w.p, n3, (float *)c->scratch[8].p);
        phi = c->scratch[8].p;
        c->launches += 1;
    }
    const double dx = kPi2 / N;
    if (f64)
        vsf_deviation_kernel<double><<<g, 256, 0, c->stream>>>((const double *)c->b_w.p, (const double *)phi, N, dx,
                                                               d_sum);
    else
        vsf_deviation_kernel<float><<<g, 256, 0, c->stream>>>((const float *)c->b_w.p, (const float *)phi, N, dx,
                                                              d_sum);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    double h = 0.0;
    FWT_CUDA(cudaMemcpyAsync(&h, d_sum, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    *deviation = h / ((double)N * N * N);
    return 0;
}

int diag_helicity(Ctx *c, double *helicity)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "helicity: not available on a z-slab context");
    if (!c->have_u) return fail(FWT_E_STATE, "helicity: u not built");
    const int N = c->p.N;
    const size_t n3 = field_elems(c);
    FWT_TRY(buf_reserve(c, c->scratch[9], 64));
    double *d_sum = (double *)c->scratch[9].p;
    FWT_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(double), c->stream));
    const unsigned g = diag_grid(c, n3);
    const int km = kt_begin(c, KT_STATS);
    if (c->p.precision == 64)
        helicity_kernel<double><<<g, 256, 0, c->stream>>>((const double *)c->b_w.p, (const double *)c->b_u.p, n3,
                                                          d_sum);
    else
        helicity_kernel<float><<<g, 256, 0, c->stream>>>((const float *)c->b_w.p, (const float *)c->b_u.p, n3, d_sum);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    double h = 0.0;
    FWT_CUDA(cudaMemcpyAsync(&h, d_sum, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    // dv = (2 pi / N)^3 (tube.f90:1024); the fields are divided by u' once normalised
    const double dx = kPi2 / N;
    const double s = c->normalised ? 1.0 / (c->up * c->up) : 1.0;
    *helicity = h * dx * dx * dx * s;
    return 0;
}

}  // namespace fwt
