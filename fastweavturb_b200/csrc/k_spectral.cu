// k_spectral.cu -- spectral Biot-Savart and filter around cuFFT (the only library call).
//
//   omega --R2C--> w^ --[biot_savart_kernel]--> u^ --C2R--> u
//
// biot_savart_kernel fuses, per mode of the half spectrum: the forward 1/N^3 scaling
// (subroutine.f90:1002,1010,1018), the shell sums of 1/2|w^|^2 (spectrum_vor_temp.dat,
// subroutine.f90:1604-1638), u^ = i k x w^ / |k|^2 with u^(0) = 0 (tube.f90:994-1007), the shell
// sums of 1/2|u^|^2 (spectrum.dat, scaled by 1/u'^2 afterwards) and the total energy and
// enstrophy (tube.f90:1026-1044 by Parseval).
//
// Nyquist planes: the reference transforms with a full complex FFT and wavenumber -N/2 at
// index N/2 (subroutine.f90:903-911), then keeps the real part of the backward transform
// (subroutine.f90:1083).  The real part equals the C2R of the Hermitian part of its u^, which
// is i (k' x w^)/|k|^2 with every Nyquist component of k' set to 0 and |k|^2 unchanged; this
// kernel writes exactly that, so C2R reproduces the reference's velocity.
#include "k_common.cuh"

namespace fwt {

// segmented warp reduction of (shell, value) pairs whose shells are non-decreasing across
// lanes; the last lane of each run adds the run total into sh[shell]
__device__ __forceinline__ void shell_add(double *sh, int nek, int s, double v, bool valid)
{
    const int lane = threadIdx.x & 31;
    if (!valid) s = -1 - lane;   // unique, never equal to a neighbour's shell
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double vv = __shfl_up_sync(0xffffffffu, v, o);
        const int ss = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o && ss == s) v += vv;
    }
    const int sn = __shfl_down_sync(0xffffffffu, s, 1);
    const bool tail = (lane == 31) || (sn != s);
    if (tail && valid && s >= 1 && s <= nek) atomicAdd(sh + s, v);
}

// mode = 0: Biot-Savart; mode = 1: low-pass filter (zero |k|^2 > kc2) and scale
// The spectrum is a block of the half spectrum: all kz, the ky indices y0 .. y0 + ny - 1, all
// kx, stored [kz][ky - y0][kx] (the whole half spectrum: y0 = 0, ny = N; one y-pencil of a grid
// split over GPUs: its ky range).
template <typename Real>
__global__ void __launch_bounds__(256) biot_savart_kernel(typename Cplx<Real>::T *__restrict__ sx,
                                                          typename Cplx<Real>::T *__restrict__ sy,
                                                          typename Cplx<Real>::T *__restrict__ sz, int N, int y0,
                                                          int ny, int mode, double kc2, double *__restrict__ g_shw,
                                                          double *__restrict__ g_shu, double *__restrict__ g_tot)
{
    extern __shared__ double sh[];   // 2 * (nek + 1)
    const int nek = N / 2;
    const int nh = N / 2 + 1;
    double *shw = sh, *shu = sh + (nek + 1);
    for (int i = threadIdx.x; i < 2 * (nek + 1); i += blockDim.x) sh[i] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const Real inv = (Real)(1.0 / ((double)N * N * N));
    double tot_u = 0.0, tot_w = 0.0;
    for (int64_t row = warp0; row < (int64_t)N * ny; row += nwarps) {
        const int jy = y0 + (int)(row % ny), jz = (int)(row / ny);
        const int ky = (jy + N / 2) % N - N / 2, kz = (jz + N / 2) % N - N / 2;
        const Real kye = (jy == N / 2) ? (Real)0 : (Real)ky;
        const Real kze = (jz == N / 2) ? (Real)0 : (Real)kz;
        const int64_t base = row * nh;
        for (int x0 = 0; x0 < nh; x0 += 32) {
            const int jx = x0 + lane;
            const bool valid = jx < nh;
            double ew = 0.0, eu = 0.0;
            int shell = 0;
            if (valid) {
                const int64_t id = base + jx;
                const double k2 = (double)jx * jx + (double)ky * ky + (double)kz * kz;
                shell = (int)(sqrt(k2 + 0.00000001) + 0.5);
                const double wgt = (jx == 0 || jx == N / 2) ? 1.0 : 2.0;
                typename Cplx<Real>::T a = sx[id], b = sy[id], c = sz[id];
                a.x *= inv; a.y *= inv; b.x *= inv; b.y *= inv; c.x *= inv; c.y *= inv;
                if (mode == 1) {
                    if (k2 > kc2) {
                        a.x = a.y = b.x = b.y = c.x = c.y = (Real)0;
                    }
                    sx[id] = a; sy[id] = b; sz[id] = c;
                    continue;
                }
                ew = 0.5 * wgt * ((double)a.x * a.x + (double)a.y * a.y + (double)b.x * b.x + (double)b.y * b.y +
                                  (double)c.x * c.x + (double)c.y * c.y);
                const Real kxe = (jx == N / 2) ? (Real)0 : (Real)jx;
                const Real ik2 = k2 > 0.0 ? (Real)(1.0 / k2) : (Real)0;
                // u^ = i (k x w^) / k2 ; i (p + i q) = -q + i p
                const Real px = kye * c.x - kze * b.x, qx = kye * c.y - kze * b.y;
                const Real py = kze * a.x - kxe * c.x, qy = kze * a.y - kxe * c.y;
                const Real pz = kxe * b.x - kye * a.x, qz = kxe * b.y - kye * a.y;
                a.x = -qx * ik2; a.y = px * ik2;
                b.x = -qy * ik2; b.y = py * ik2;
                c.x = -qz * ik2; c.y = pz * ik2;
                sx[id] = a; sy[id] = b; sz[id] = c;
                eu = 0.5 * wgt * ((double)a.x * a.x + (double)a.y * a.y + (double)b.x * b.x + (double)b.y * b.y +
                                  (double)c.x * c.x + (double)c.y * c.y);
                tot_u += eu;
                tot_w += ew;
            }
            if (mode == 0) {
                shell_add(shw, nek, shell, ew, valid);
                shell_add(shu, nek, shell, eu, valid);
            }
        }
    }
    if (mode == 1) return;
    tot_u = warp_sum(tot_u);
    tot_w = warp_sum(tot_w);
    if (lane == 0) {
        atomicAdd(g_tot + 0, tot_u);
        atomicAdd(g_tot + 1, tot_w);
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= nek; i += blockDim.x) {
        if (shw[i] != 0.0) atomicAdd(g_shw + i, shw[i]);
        if (shu[i] != 0.0) atomicAdd(g_shu + i, shu[i]);
    }
}

int spectral_init(Ctx *c)
{
    if (c->plans) return 0;
    const int N = c->p.N;
    int n[3] = {N, N, N};
    const bool dbl = c->p.precision == 64;
    FWT_CUFFT(cufftCreate(&c->plan_r2c));
    FWT_CUFFT(cufftCreate(&c->plan_c2r));
    // the two plans run one after the other on the context's stream: one work area serves
    // both (at 1024^3 in FP64 each would otherwise hold tens of GB of its own)
    FWT_CUFFT(cufftSetAutoAllocation(c->plan_r2c, 0));
    FWT_CUFFT(cufftSetAutoAllocation(c->plan_c2r, 0));
    size_t ws1 = 0, ws2 = 0;
    const long long nh = (long long)N * N * (N / 2 + 1), n3 = (long long)N * N * N;
    FWT_CUFFT(cufftMakePlanMany(c->plan_r2c, 3, n, nullptr, 1, (int)0, nullptr, 1, 0,
                                dbl ? CUFFT_D2Z : CUFFT_R2C, 3, &ws1));
    FWT_CUFFT(cufftMakePlanMany(c->plan_c2r, 3, n, nullptr, 1, 0, nullptr, 1, 0, dbl ? CUFFT_Z2D : CUFFT_C2R, 3,
                                &ws2));
    (void)nh;
    (void)n3;
    FWT_CUFFT(cufftSetStream(c->plan_r2c, c->stream));
    FWT_CUFFT(cufftSetStream(c->plan_c2r, c->stream));
    c->fft_ws_bytes = std::max(ws1, ws2);
    FWT_TRY(buf_reserve(c, c->b_fftws, c->fft_ws_bytes));
    FWT_CUFFT(cufftSetWorkArea(c->plan_r2c, c->b_fftws.p));
    FWT_CUFFT(cufftSetWorkArea(c->plan_c2r, c->b_fftws.p));
    c->plans = true;
    return 0;
}

static int spec_buffers(Ctx *c)
{
    const int N = c->p.N;
    const size_t nh = (size_t)N * N * (N / 2 + 1);
    FWT_TRY(buf_reserve(c, c->b_spec, 3 * nh * 2 * real_bytes(c)));
    return 0;
}

static int run_r2c(Ctx *c, void *in, void *out)
{
    const int km = kt_begin(c, KT_FFT);
    if (c->p.precision == 64) FWT_CUFFT(cufftExecD2Z(c->plan_r2c, (cufftDoubleReal *)in, (cufftDoubleComplex *)out));
    else FWT_CUFFT(cufftExecR2C(c->plan_r2c, (cufftReal *)in, (cufftComplex *)out));
    kt_end(c, km);
    return 0;
}

static int run_c2r(Ctx *c, void *in, void *out)
{
    const int km = kt_begin(c, KT_FFT);
    if (c->p.precision == 64) FWT_CUFFT(cufftExecZ2D(c->plan_c2r, (cufftDoubleComplex *)in, (cufftDoubleReal *)out));
    else FWT_CUFFT(cufftExecC2R(c->plan_c2r, (cufftComplex *)in, (cufftReal *)out));
    kt_end(c, km);
    return 0;
}

static int launch_bs(Ctx *c, int mode, double kc2, double *d_shw, double *d_shu, double *d_tot)
{
    const int N = c->p.N;
    const size_t nh = (size_t)N * N * (N / 2 + 1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int64_t rows = (int64_t)N * N;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8, (int64_t)sms * 8));
    const size_t shb = sizeof(double) * 2 * (N / 2 + 1);
    const int km = kt_begin(c, KT_SPECTRAL);
    if (c->p.precision == 64) {
        cufftDoubleComplex *s = (cufftDoubleComplex *)c->b_spec.p;
        biot_savart_kernel<double><<<blocks, 256, shb, c->stream>>>(s, s + nh, s + 2 * nh, N, 0, N, mode, kc2, d_shw,
                                                                    d_shu, d_tot);
    } else {
        cufftComplex *s = (cufftComplex *)c->b_spec.p;
        biot_savart_kernel<float><<<blocks, 256, shb, c->stream>>>(s, s + nh, s + 2 * nh, N, 0, N, mode, kc2, d_shw,
                                                                   d_shu, d_tot);
    }
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    return 0;
}

int spectral_filter(Ctx *c, double k_c)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "spectral filter: not available on a z-slab context");
    if (!c->have_w) return fail(FWT_E_STATE, "filter before deposition");
    FWT_TRY(spectral_init(c));
    FWT_TRY(spec_buffers(c));
    FWT_TRY(run_r2c(c, c->b_w.p, c->b_spec.p));
    FWT_TRY(launch_bs(c, 1, k_c * k_c, nullptr, nullptr, nullptr));
    FWT_TRY(run_c2r(c, c->b_spec.p, c->b_w.p));
    c->wmm_valid = false;
    return 0;
}

int spectral_biot_savart(Ctx *c)
{
    if (c->slab_nz) return fail(FWT_E_STATE, "Biot-Savart: not available on a z-slab context");
    if (!c->have_w) return fail(FWT_E_STATE, "Biot-Savart before deposition");
    const int N = c->p.N;
    const int nek = N / 2;
    FWT_TRY(spectral_init(c));
    FWT_TRY(spec_buffers(c));
    const size_t n3 = field_elems(c);
    FWT_TRY(buf_reserve(c, c->b_u, 3 * n3 * real_bytes(c)));
    FWT_TRY(buf_reserve(c, c->scratch[11], sizeof(double) * (2 * (nek + 1) + 4)));
    double *d_shw = (double *)c->scratch[11].p, *d_shu = d_shw + (nek + 1), *d_tot = d_shu + (nek + 1);
    FWT_CUDA(cudaMemsetAsync(d_shw, 0, sizeof(double) * (2 * (nek + 1) + 4), c->stream));
    FWT_TRY(run_r2c(c, c->b_w.p, c->b_spec.p));
    FWT_TRY(launch_bs(c, 0, 0.0, d_shw, d_shu, d_tot));
    FWT_TRY(run_c2r(c, c->b_spec.p, c->b_u.p));
    std::vector<double> h(2 * (nek + 1) + 2);
    FWT_CUDA(cudaMemcpyAsync(h.data(), d_shw, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    c->spec_w.assign(h.begin() + 1, h.begin() + 1 + nek);
    c->spec_u.assign(h.begin() + (nek + 1) + 1, h.begin() + (nek + 1) + 1 + nek);
    c->Etot_raw = h[2 * (nek + 1)];
    c->enstrophy_raw = h[2 * (nek + 1) + 1];
    c->have_u = true;
    c->normalised = false;
    c->umm_valid = false;
    return 0;
}

// Biot-Savart on one y-pencil of the half spectrum (a grid split over GPUs): spec holds the
// three components, each [N kz][ny ky][N/2 + 1 kx] from ky = y0, unscaled forward transforms
// of omega; in place it becomes u^ as in spectral_biot_savart.  host_sums receives the pencil's
// shell sums of 1/2 |w^|^2 and 1/2 |u^|^2 (shells 1..N/2) and its total energy and enstrophy
// (2 (N/2 + 1) + 2 values: [0] and [N/2 + 1] unused), to be summed over the pencils.
int spectral_block(Ctx *c, void *spec, int y0, int ny, double *host_sums)
{
    const int N = c->p.N;
    const int nek = N / 2;
    if (y0 < 0 || ny < 1 || y0 + ny > N) return fail(FWT_E_ARG, "biot_savart_block: ky range outside 0..N-1");
    FWT_TRY(buf_reserve(c, c->scratch[11], sizeof(double) * (2 * (nek + 1) + 4)));
    double *d_shw = (double *)c->scratch[11].p, *d_shu = d_shw + (nek + 1), *d_tot = d_shu + (nek + 1);
    FWT_CUDA(cudaMemsetAsync(d_shw, 0, sizeof(double) * (2 * (nek + 1) + 4), c->stream));
    const size_t nb = (size_t)N * ny * (N / 2 + 1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int64_t rows = (int64_t)N * ny;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows + 7) / 8, (int64_t)sms * 8));
    const size_t shb = sizeof(double) * 2 * (N / 2 + 1);
    const int km = kt_begin(c, KT_SPECTRAL);
    if (c->p.precision == 64) {
        cufftDoubleComplex *s = (cufftDoubleComplex *)spec;
        biot_savart_kernel<double><<<blocks, 256, shb, c->stream>>>(s, s + nb, s + 2 * nb, N, y0, ny, 0, 0.0, d_shw,
                                                                    d_shu, d_tot);
    } else {
        cufftComplex *s = (cufftComplex *)spec;
        biot_savart_kernel<float><<<blocks, 256, shb, c->stream>>>(s, s + nb, s + 2 * nb, N, y0, ny, 0, 0.0, d_shw,
                                                                   d_shu, d_tot);
    }
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    FWT_CUDA(cudaMemcpyAsync(host_sums, d_shw, sizeof(double) * (2 * (nek + 1) + 2), cudaMemcpyDeviceToHost,
                             c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

}  // namespace fwt
