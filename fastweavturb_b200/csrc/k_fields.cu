// k_fields.cu -- the reference's optional field outputs (tube.f90:1075-1120), switched off there
// by the compile-time flags u_out and d_out (tube.f90:55) and here by fwt_set_outputs:
//   field_uw.dat   ux, uy, uz, wx, wy, wz at the downsampled points
//   field_wd.dat   |omega| and the dissipation S_ij S_ij (dissipation_field,
//                  subroutine.f90:1086-1126), S_ij = (du_i/dx_j + du_j/dx_i) / 2
//
// The reference differentiates spectrally: one complex FFT per velocity component and
// direction, multiplication by i k_j, the unscaled backward transform and its real part
// (dx_dy_dz_dp_dm, subroutine.f90:1128-1163), nine gradient fields in all.  Here one batched
// R2C of u gives u^, and two batched C2R passes give the six distinct S_ij directly, formed in
// the spectrum as i (k_j u^_i + k_i u^_j) / 2: the diagonal (S_11, S_22, S_33), then
// S_12, S_13, S_23.  Each pass adds its squares, at the downsampled points only, into an FP64
// sum.  Nyquist planes: the real part of the reference's backward transform is the C2R of the
// Hermitian part of i k u^, which has the Nyquist component of k set to 0 (the same rule as
// the Biot-Savart kernel).
#include "k_common.cuh"

namespace fwt {

namespace {

// data_box(i, j, k, :) = field(i*r_d, j*r_d, k*r_d, :), 1-based (tube.f90:1076-1087)
__device__ __forceinline__ size_t box_point(size_t q, int N, int nd)
{
    const int rd = N / nd;
    const int i = (int)(q % nd), j = (int)((q / nd) % nd), k = (int)(q / ((size_t)nd * nd));
    return (size_t)((i + 1) * rd - 1) + (size_t)N * ((size_t)((j + 1) * rd - 1) + (size_t)N * ((k + 1) * rd - 1));
}

template <typename Real>
__global__ void field_uw_kernel(const Real *__restrict__ w, const Real *__restrict__ u, int N, int nd, double s,
                                float *__restrict__ out)
{
    const size_t n3 = (size_t)N * N * N, m3 = (size_t)nd * nd * nd;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m3; q += (size_t)gridDim.x * blockDim.x) {
        const size_t g = box_point(q, N, nd);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            out[q + c * m3] = (float)((double)u[g + c * n3] * s);
            out[q + (3 + c) * m3] = (float)((double)w[g + c * n3] * s);
        }
    }
}

// pass 0: o_c = i k_c u^_c (S_11, S_22, S_33); pass 1: S_12, S_13, S_23 = i (k_j u^_i + k_i u^_j) / 2;
// u^ is the unscaled R2C output, so every mode is also scaled by 1 / N^3
template <typename Real>
__global__ void strain_spec_kernel(const typename Cplx<Real>::T *__restrict__ ux,
                                   const typename Cplx<Real>::T *__restrict__ uy,
                                   const typename Cplx<Real>::T *__restrict__ uz, typename Cplx<Real>::T *__restrict__ o0,
                                   typename Cplx<Real>::T *__restrict__ o1, typename Cplx<Real>::T *__restrict__ o2,
                                   int N, int pass)
{
    const int nh = N / 2 + 1;
    const size_t total = (size_t)N * N * nh;
    const double inv = 1.0 / ((double)N * N * N);
    for (size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (size_t)gridDim.x * blockDim.x) {
        const int jx = (int)(id % nh);
        const size_t row = id / nh;
        const int jy = (int)(row % N), jz = (int)(row / N);
        const Real kx = (jx == N / 2) ? (Real)0 : (Real)jx;
        const Real ky = (jy == N / 2) ? (Real)0 : (Real)((jy + N / 2) % N - N / 2);
        const Real kz = (jz == N / 2) ? (Real)0 : (Real)((jz + N / 2) % N - N / 2);
        const typename Cplx<Real>::T a = ux[id], b = uy[id], c = uz[id];
        // i k (p + i q) = -k q + i k p
        typename Cplx<Real>::T r0, r1, r2;
        if (pass == 0) {
            r0.x = -kx * a.y; r0.y = kx * a.x;
            r1.x = -ky * b.y; r1.y = ky * b.x;
            r2.x = -kz * c.y; r2.y = kz * c.x;
        } else {
            const Real h = (Real)0.5;
            r0.x = -h * (ky * a.y + kx * b.y); r0.y = h * (ky * a.x + kx * b.x);   // S_12
            r1.x = -h * (kz * a.y + kx * c.y); r1.y = h * (kz * a.x + kx * c.x);   // S_13
            r2.x = -h * (kz * b.y + ky * c.y); r2.y = h * (kz * b.x + ky * c.x);   // S_23
        }
        const Real sc = (Real)inv;
        r0.x *= sc; r0.y *= sc; r1.x *= sc; r1.y *= sc; r2.x *= sc; r2.y *= sc;
        o0[id] = r0;
        o1[id] = r1;
        o2[id] = r2;
    }
}

// acc[q] += wgt (S_a^2 + S_b^2 + S_c^2) at the downsampled points
template <typename Real>
__global__ void strain_acc_kernel(const Real *__restrict__ S, int N, int nd, double wgt, double *__restrict__ acc)
{
    const size_t n3 = (size_t)N * N * N, m3 = (size_t)nd * nd * nd;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m3; q += (size_t)gridDim.x * blockDim.x) {
        const size_t g = box_point(q, N, nd);
        const double a = S[g], b = S[g + n3], c = S[g + 2 * n3];
        acc[q] += wgt * (a * a + b * b + c * c);
    }
}

// (|omega|, S_ij S_ij) of the normalised fields: omega and u scale by s = 1/u', S_ij S_ij by s^2
template <typename Real>
__global__ void field_wd_kernel(const Real *__restrict__ w, const double *__restrict__ acc, int N, int nd, double s,
                                float *__restrict__ out)
{
    const size_t n3 = (size_t)N * N * N, m3 = (size_t)nd * nd * nd;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < m3; q += (size_t)gridDim.x * blockDim.x) {
        const size_t g = box_point(q, N, nd);
        const double wx = (double)w[g] * s, wy = (double)w[g + n3] * s, wz = (double)w[g + 2 * n3] * s;
        out[q] = (float)sqrt(wx * wx + wy * wy + wz * wz);
        out[q + m3] = (float)(acc[q] * s * s);
    }
}

unsigned grid_of(size_t n)
{
    return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)148 * 16));
}

int check_box(Ctx *c)
{
    if (!c->normalised) return fail(FWT_E_STATE, "field output before normalisation");
    const int N = c->p.N, nd = c->p.N_downsample;
    if (nd < 1 || N % nd) return fail(FWT_E_ARG, "N_downsample must divide N");
    return 0;
}

template <typename Real>
int field_wd_impl(Ctx *c, float *d_out)
{
    using C = typename Cplx<Real>::T;
    const int N = c->p.N, nd = c->p.N_downsample;
    const size_t nh = (size_t)N * N * (N / 2 + 1), n3 = (size_t)N * N * N, m3 = (size_t)nd * nd * nd;
    FWT_TRY(spectral_init(c));
    FWT_TRY(buf_reserve(c, c->b_spec, 3 * nh * sizeof(C)));
    FWT_TRY(buf_reserve(c, c->b_aux_spec, 3 * nh * sizeof(C)));
    FWT_TRY(buf_reserve(c, c->b_aux_real, 3 * n3 * sizeof(Real)));
    FWT_TRY(buf_reserve(c, c->b_aux_acc, m3 * sizeof(double)));
    C *uh = (C *)c->b_spec.p, *sh = (C *)c->b_aux_spec.p;
    Real *S = (Real *)c->b_aux_real.p;
    double *acc = (double *)c->b_aux_acc.p;
    FWT_CUDA(cudaMemsetAsync(acc, 0, m3 * sizeof(double), c->stream));
    int km = kt_begin(c, KT_FFT);
    // u^ = R2C(u); the R2C is out of place and leaves u as it is
    if (sizeof(Real) == 8) FWT_CUFFT(cufftExecD2Z(c->plan_r2c, (cufftDoubleReal *)c->b_u.p, (cufftDoubleComplex *)uh));
    else FWT_CUFFT(cufftExecR2C(c->plan_r2c, (cufftReal *)c->b_u.p, (cufftComplex *)uh));
    kt_end(c, km);
    for (int pass = 0; pass < 2; ++pass) {
        km = kt_begin(c, KT_STATS);
        strain_spec_kernel<Real><<<grid_of(nh), 256, 0, c->stream>>>(uh, uh + nh, uh + 2 * nh, sh, sh + nh, sh + 2 * nh,
                                                                     N, pass);
        kt_end(c, km);
        km = kt_begin(c, KT_FFT);
        // the C2R overwrites its input: each pass forms its spectra from u^ again
        if (sizeof(Real) == 8) FWT_CUFFT(cufftExecZ2D(c->plan_c2r, (cufftDoubleComplex *)sh, (cufftDoubleReal *)S));
        else FWT_CUFFT(cufftExecC2R(c->plan_c2r, (cufftComplex *)sh, (cufftReal *)S));
        kt_end(c, km);
        km = kt_begin(c, KT_STATS);
        strain_acc_kernel<Real><<<grid_of(m3), 256, 0, c->stream>>>(S, N, nd, pass == 0 ? 1.0 : 2.0, acc);
        kt_end(c, km);
    }
    km = kt_begin(c, KT_STATS);
    field_wd_kernel<Real><<<grid_of(m3), 256, 0, c->stream>>>((const Real *)c->b_w.p, acc, N, nd, 1.0 / c->up, d_out);
    kt_end(c, km);
    c->launches += 5;
    FWT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace

int stats_field_uw(Ctx *c, float *host_out)
{
    FWT_TRY(check_box(c));
    const int N = c->p.N, nd = c->p.N_downsample;
    const size_t m3 = (size_t)nd * nd * nd;
    FWT_TRY(buf_reserve(c, c->b_aux_out, sizeof(float) * 6 * m3));
    float *d = (float *)c->b_aux_out.p;
    const int km = kt_begin(c, KT_STATS);
    if (c->p.precision == 64)
        field_uw_kernel<double><<<grid_of(m3), 256, 0, c->stream>>>((const double *)c->b_w.p, (const double *)c->b_u.p,
                                                                    N, nd, 1.0 / c->up, d);
    else
        field_uw_kernel<float><<<grid_of(m3), 256, 0, c->stream>>>((const float *)c->b_w.p, (const float *)c->b_u.p, N,
                                                                   nd, 1.0 / c->up, d);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    FWT_CUDA(cudaMemcpyAsync(host_out, d, sizeof(float) * 6 * m3, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

int stats_field_wd(Ctx *c, float *host_out)
{
    FWT_TRY(check_box(c));
    const int nd = c->p.N_downsample;
    const size_t m3 = (size_t)nd * nd * nd;
    FWT_TRY(buf_reserve(c, c->b_aux_out, sizeof(float) * 2 * m3));
    float *d = (float *)c->b_aux_out.p;
    if (c->p.precision == 64) FWT_TRY(field_wd_impl<double>(c, d));
    else FWT_TRY(field_wd_impl<float>(c, d));
    FWT_CUDA(cudaMemcpyAsync(host_out, d, sizeof(float) * 2 * m3, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

}  // namespace fwt
