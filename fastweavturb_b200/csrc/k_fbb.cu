// k_fbb.cu -- fractional-Brownian-bridge centerlines on the device (FBB_with_parameters.m:76-126).
//
// The reference draws fBm with MATLAB's wfbm (closed, Wavelet Toolbox).  Here fBm comes from
// the Davies-Harte circulant embedding (Davies & Harte 1987; Wood & Chan 1994), a published
// exact method: with lambda = FFT of the 2M circulant row of the fGn autocovariance
// gamma(k) = (|k+1|^2H - 2|k|^2H + |k-1|^2H)/2, the real part of FFT(sqrt(lambda/2M) (Za + i Zb))
// over the first M entries is fGn, and its FP64 prefix sum is fBm.  Random numbers: Philox4x32-10
// (Salmon et al., SC'11) with counter {index, tube, stream, 0} and key = seed, Gaussians by
// Box-Muller on 53-bit uniforms.  Then, per tube: bridge f(j) (m:92-102), rms-step
// normalisation to dB (m:104-112), uniform shift and wrap mod 2pi - pi (m:117-120).
#include <cufft.h>

#include <cmath>
#include <map>

#include "k_common.cuh"

namespace fwt {

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__host__ __device__ __forceinline__ double u53(uint32_t hi, uint32_t lo)
{
    return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6) + 0.5) * (1.0 / 9007199254740992.0);
}

// circulant first row of the fGn autocovariance, size 2M
__global__ void fbb_row_kernel(int M, double H, cufftDoubleComplex *row)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 2 * M) return;
    const int kk = k <= M ? k : 2 * M - k;
    const double a = (double)kk;
    const double g = 0.5 * (pow(fabs(a + 1.0), 2 * H) - 2.0 * pow(fabs(a), 2 * H) + pow(fabs(a - 1.0), 2 * H));
    row[k].x = g;
    row[k].y = 0.0;
}

__global__ void fbb_sqrt_kernel(int n2, const cufftDoubleComplex *lam, double *sq)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n2) return;
    sq[k] = sqrt(fmax(lam[k].x, 0.0) / n2);
}

// Z[b][k] = sq[k] (Za + i Zb), b = 3*(tube - t0) + coord
__global__ void fbb_fill_kernel(uint64_t seed, int t0, int nb, int n2, const double *__restrict__ sq,
                                cufftDoubleComplex *__restrict__ Z)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)nb * n2) return;
    const int b = (int)(i / n2), k = (int)(i % n2);
    const uint32_t tube = (uint32_t)(t0 + b / 3), co = (uint32_t)(b % 3);
    uint32_t c[4] = {(uint32_t)k, tube, co, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double a = u53(c[0], c[1]), bb = u53(c[2], c[3]);
    const double r = sqrt(-2.0 * log(a));
    double sn, cs;
    sincos(6.28318530717958647692 * bb, &sn, &cs);
    Z[i].x = sq[k] * (r * cs);
    Z[i].y = sq[k] * (r * sn);
}

// fBm = FP64 inclusive prefix sum of Re W[0..M-1]; one block per (tube, coord)
__global__ void fbb_scan_kernel(const cufftDoubleComplex *__restrict__ W, int n2, int M, double *__restrict__ fbm)
{
    const int b = blockIdx.x;
    const cufftDoubleComplex *w = W + (int64_t)b * n2;
    double *o = fbm + (int64_t)b * M;
    __shared__ double part[32];
    __shared__ double carry;
    if (threadIdx.x == 0) carry = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = 0; base < M; base += blockDim.x) {
        const int j = base + threadIdx.x;
        double v = j < M ? w[j].x : 0.0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += t;
        }
        if (lane == 31) part[wp] = v;
        __syncthreads();
        if (wp == 0) {
            double y = lane < nw ? part[lane] : 0.0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const double t = __shfl_up_sync(0xffffffffu, y, off);
                if (lane >= off) y += t;
            }
            if (lane < nw) part[lane] = y;
        }
        __syncthreads();
        const double incl = v + (wp > 0 ? part[wp - 1] : 0.0) + carry;
        if (j < M) o[j] = incl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
}

// per tube: subsample (Np < 128), bridge, rms normalisation, shift, wrap
__global__ void fbb_bridge_kernel(uint64_t seed, int t0, int Np, int M, double H, double dB,
                                  const double *__restrict__ fbm, double *__restrict__ X, double *__restrict__ Y,
                                  double *__restrict__ Z, int64_t node0)
{
    const int tl = blockIdx.x;
    const uint32_t tube = (uint32_t)(t0 + tl);
    const double *f[3] = {fbm + (int64_t)(3 * tl) * M, fbm + (int64_t)(3 * tl + 1) * M, fbm + (int64_t)(3 * tl + 2) * M};
    auto src = [&](int co, int j) -> double {   // FBM(co, j), j = 0..Np-1
        if (Np < 128) {
            const int r_t = 128 / Np;
            const int idx = (int)ceil((double)(j + 1) * r_t) - 1;
            return f[co][idx];
        }
        return f[co][j];
    };
    auto fb = [&](int j) -> double {   // f_bridge(j+1)
        const double x = (double)(j + 1) / Np;
        return 0.5 * (pow(x, 2.0 * H) + 1.0 - pow(1.0 - x, 2.0 * H));
    };
    double end[3];
    for (int co = 0; co < 3; ++co) end[co] = src(co, Np - 1);
    // rms of steps over the three coordinates
    double acc = 0.0;
    for (int j = threadIdx.x; j < Np - 1; j += blockDim.x) {
        const double f0 = fb(j), f1 = fb(j + 1);
        for (int co = 0; co < 3; ++co) {
            const double d = (src(co, j + 1) - f1 * end[co]) - (src(co, j) - f0 * end[co]);
            acc += d * d / (Np - 1);
        }
    }
    __shared__ double red[32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    __shared__ double s_scale;
    __shared__ double s_shift[3];
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += red[w];
        s_scale = dB / sqrt(r);
        for (int co = 0; co < 3; ++co) {
            uint32_t c[4] = {(uint32_t)co, tube, 3u, 0u};
            philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
            const double u = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6)) * (1.0 / 9007199254740992.0);
            s_shift[co] = (u - 0.5) * 2.0 * dev_pi();
        }
    }
    __syncthreads();
    double *out[3] = {X, Y, Z};
    const int64_t o = node0 + (int64_t)tl * Np;
    for (int j = threadIdx.x; j < Np; j += blockDim.x) {
        const double fj = fb(j);
        for (int co = 0; co < 3; ++co) {
            double v = (src(co, j) - fj * end[co]) * s_scale + s_shift[co];
            // mod(v, 2pi) - pi with MATLAB's floored modulo
            double m = v - floor(v / (2.0 * dev_pi())) * (2.0 * dev_pi());
            out[co][o + j] = m - dev_pi();
        }
    }
}

// A Z2Z plan of length n2 over `batch` contiguous rows, made once per context and shape (at
// most eight are kept; the oldest is dropped).
static int fbb_plan(Ctx *c, int n2, int batch, cufftHandle *out)
{
    for (const auto &p : c->fbb_plans) {
        if (p.n2 == n2 && p.batch == batch) {
            *out = p.h;
            return 0;
        }
    }
    if (c->fbb_plans.size() >= 8) {
        cufftDestroy(c->fbb_plans.front().h);
        c->fbb_plans.erase(c->fbb_plans.begin());
    }
    cufftHandle h = 0;
    int n[1] = {n2};
    FWT_CUFFT(cufftPlanMany(&h, 1, n, nullptr, 1, n2, nullptr, 1, n2, CUFFT_Z2Z, batch));
    c->fbb_plans.push_back({n2, batch, h});
    *out = h;
    return 0;
}

int fbb_generate(Ctx *c, uint64_t seed, int nlev, const int *tubes, const int *nodes, const double *H,
                 const double *dB, double *d_x, double *d_y, double *d_z)
{
    int64_t node0 = 0;
    int t0 = 0;
    for (int lv = 0; lv < nlev; ++lv) {
        const int T = tubes[lv], Np = nodes[lv];
        if (T < 0 || Np < 2) return fail(FWT_E_ARG, "generator: tubes >= 0 and nodes >= 2 required");
        if (!(H[lv] > 0 && H[lv] < 1)) return fail(FWT_E_ARG, "generator: H must be in (0,1)");
        if (Np < 128 && 128 % Np) return fail(FWT_E_ARG, "generator: nodes below 128 must divide 128");
        const int M = Np < 128 ? 128 : Np, n2 = 2 * M;
        // eigenvalues of the circulant embedding
        FWT_TRY(buf_reserve(c, c->scratch[2], sizeof(cufftDoubleComplex) * n2 + sizeof(double) * n2));
        cufftDoubleComplex *row = (cufftDoubleComplex *)c->scratch[2].p;
        double *sq = (double *)(row + n2);
        fbb_row_kernel<<<(n2 + 255) / 256, 256, 0, c->stream>>>(M, H[lv], row);
        cufftHandle p1;
        FWT_TRY(fbb_plan(c, n2, 1, &p1));
        FWT_CUFFT(cufftSetStream(p1, c->stream));
        FWT_CUFFT(cufftExecZ2Z(p1, row, row, CUFFT_FORWARD));
        fbb_sqrt_kernel<<<(n2 + 255) / 256, 256, 0, c->stream>>>(n2, row, sq);
        c->launches += 3;
        // batches of tubes: 3 complex rows of n2 per tube, ~1 GB per batch
        const int per = std::max(1, (int)std::min<int64_t>(T, ((int64_t)1 << 30) / ((int64_t)3 * n2 * 16)));
        cufftHandle pb = 0;
        for (int tb = 0; tb < T; tb += per) {
            const int nt = std::min(per, T - tb), nb = 3 * nt;
            FWT_TRY(buf_reserve(c, c->scratch[3], sizeof(cufftDoubleComplex) * (size_t)nb * n2));
            FWT_TRY(buf_reserve(c, c->scratch[4], sizeof(double) * (size_t)nb * M));
            cufftDoubleComplex *Zb = (cufftDoubleComplex *)c->scratch[3].p;
            double *fbm = (double *)c->scratch[4].p;
            const int64_t tot = (int64_t)nb * n2;
            fbb_fill_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(seed, t0 + tb, nb, n2, sq, Zb);
            FWT_TRY(fbb_plan(c, n2, nb, &pb));
            FWT_CUFFT(cufftSetStream(pb, c->stream));
            FWT_CUFFT(cufftExecZ2Z(pb, Zb, Zb, CUFFT_FORWARD));
            fbb_scan_kernel<<<nb, 256, 0, c->stream>>>(Zb, n2, M, fbm);
            fbb_bridge_kernel<<<nt, 256, 0, c->stream>>>(seed, t0 + tb, Np, M, H[lv], dB[lv], fbm, d_x, d_y, d_z,
                                                         node0 + (int64_t)tb * Np);
            c->launches += 4;
            FWT_CUDA(cudaGetLastError());
        }
        node0 += (int64_t)T * Np;
        t0 += T;
    }
    // the arrays are complete when the call returns
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

}  // namespace fwt

extern "C" int fwt_fbb_signs(uint64_t seed, int ntubes, int *signs)
{
    if (ntubes < 0 || (!signs && ntubes)) return fwt::fail(FWT_E_ARG, "bad arguments");
    for (int t = 0; t < ntubes; ++t) {
        uint32_t c[4] = {0u, (uint32_t)t, 4u, 0u};
        fwt::philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        signs[t] = (c[0] & 1u) ? -1 : 1;
    }
    return 0;
}
