// k_centerline.cu -- centerline set-up on the device, all FP64 (one B200 runs FP64 at half
// the FP32 rate, and the integer sub-segment counts must follow the reference):
//   line_prep_kernel   periodic arc length cze, Len_Disc, c', c''       tube.f90:392-515
//   section_coe_kernel quintic coefficients                              subroutine.f90:440-488
//   section_kernel     turning-angle sum, one warp per section           tube.f90:625-657
//   section_ntf_kernel ntf/dtf, FP64 recompute list near a step of ceil  tube.f90:655-657
//   sample_kernel      sample points ci with the endpoint copy          tube.f90:706-723
//   chord_kernel       chords dci, |dci|, unit chords tci               tube.f90:740-751
//   subseg_kernel      sub-segment records (unwrap, Rtube, box)          tube.f90:766-798
#include "k_deposit.cuh"
#include "k_tile_common.cuh"

namespace fwt {

// Slot -> batch-local line: block i fills line i's n_sec + 1 section slots.
__global__ void slot_line_kernel(const LineParam *__restrict__ lp, int nlines, int *__restrict__ slot_line)
{
    const int i = blockIdx.x;
    if (i >= nlines) return;
    const LineParam &P = lp[i];
    for (int t = threadIdx.x; t < P.n_sec + 1; t += blockDim.x) slot_line[P.slot_off + t] = i;
}

// ------------------------------------------------------------------ a2: line preprocessing
// One block per line.  cze is an FP64 block scan of the wrapped node distances.
__global__ void line_prep_kernel(const LineParam *__restrict__ lp, int nlines, const double *__restrict__ X,
                                 const double *__restrict__ Y, const double *__restrict__ Z,
                                 double *__restrict__ cze, double *__restrict__ ck, double *__restrict__ ckk,
                                 double *__restrict__ Len_out, int64_t node_base)
{
    const int l = blockIdx.x;
    if (l >= nlines) return;
    const int np = lp[l].n_sec;
    const int64_t g0 = lp[l].node_off;            // global node index of node 0
    const int64_t o = g0 - node_base;              // batch-local node index
    const double *c[3] = {X + g0, Y + g0, Z + g0};
    __shared__ double s_part[32];
    __shared__ double s_carry;
    if (threadIdx.x == 0) s_carry = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // pass 1: cze(i) = cze(i-1) + dist(i-1, i), inclusive scan over i = 1..np-1
    for (int base = 0; base < np; base += blockDim.x) {
        const int i = base + threadIdx.x;
        double d = 0.0;
        if (i >= 1 && i < np) {
            double cd[3];
            for (int k = 0; k < 3; ++k) {
                double v = fabs(c[k][i] - c[k][i - 1]);
                if (v > dev_pi()) v = v - dev_pi2();
                cd[k] = v;
            }
            d = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
        }
        // warp inclusive scan
        double v = d;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            double t = __shfl_up_sync(0xffffffffu, v, off);
            if (lane >= off) v += t;
        }
        if (lane == 31) s_part[warp] = v;
        __syncthreads();
        if (warp == 0) {
            double w = (lane < nw) ? s_part[lane] : 0.0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                double t = __shfl_up_sync(0xffffffffu, w, off);
                if (lane >= off) w += t;
            }
            if (lane < nw) s_part[lane] = w;
        }
        __syncthreads();
        const double pre = (warp > 0 ? s_part[warp - 1] : 0.0) + s_carry;
        if (i < np) cze[o + i] = pre + v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry = pre + v;
        __syncthreads();
    }
    __shared__ double s_total;
    if (threadIdx.x == 0) {
        double cd[3];
        for (int k = 0; k < 3; ++k) {
            double v = fabs(c[k][0] - c[k][np - 1]);
            if (v > dev_pi()) v = v - dev_pi2();
            cd[k] = v;
        }
        const double dist = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
        s_total = cze[o + np - 1] + dist;
        Len_out[l] = s_total / dev_pi2();
    }
    __syncthreads();
    const double total = s_total, L = total / dev_pi2();
    for (int i = threadIdx.x; i < np; i += blockDim.x) cze[o + i] = cze[o + i] * dev_pi2() / total;
    __syncthreads();
    // first derivative (tube.f90:440-466)
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        int ip, im;
        double dz;
        if (i == 0) { ip = 1; im = np - 1; dz = cze[o + 1] - cze[o + np - 1] + dev_pi2(); }
        else if (i == np - 1) { ip = 0; im = np - 2; dz = cze[o] - cze[o + np - 2] + dev_pi2(); }
        else { ip = i + 1; im = i - 1; dz = cze[o + i + 1] - cze[o + i - 1]; }
        for (int k = 0; k < 3; ++k) {
            double v = c[k][ip] - c[k][im];
            if (v > dev_pi()) v = v - dev_pi2();
            if (v < -dev_pi()) v = v + dev_pi2();
            ck[3 * (o + i) + k] = v / (dz * L);
        }
    }
    __syncthreads();
    // second derivative (tube.f90:469-489)
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        int ip, im;
        double dz;
        if (i == 0) { ip = 1; im = np - 1; dz = cze[o + 1] - cze[o + np - 1] + dev_pi2(); }
        else if (i == np - 1) { ip = 0; im = np - 2; dz = cze[o] - cze[o + np - 2] + dev_pi2(); }
        else { ip = i + 1; im = i - 1; dz = cze[o + i + 1] - cze[o + i - 1]; }
        for (int k = 0; k < 3; ++k) ckk[3 * (o + i) + k] = (ck[3 * (o + ip) + k] - ck[3 * (o + im) + k]) / (dz * L);
    }
}


// ------------------------------------------------------------------ a3/a5: sections
// |c' x c''| / |c'|^2 at z of the quintic whose derivative coefficients are d1 ([coord][5]:
// a1, 2 a2, 3 a3, 4 a4, 5 a5) and d2 ([coord][4]: 2 a2, 6 a3, 12 a4, 20 a5), FP32
// (tube.f90:633-647), added to th
__device__ __forceinline__ void turning_integrand(const float (&d1)[3][5], const float (&d2)[3][4], float z, float &th)
{
    float dc[3], dd[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        dc[d] = fmaf(fmaf(fmaf(fmaf(d1[d][4], z, d1[d][3]), z, d1[d][2]), z, d1[d][1]), z, d1[d][0]);
        dd[d] = fmaf(fmaf(fmaf(d2[d][3], z, d2[d][2]), z, d2[d][1]), z, d2[d][0]);
    }
    const float x0 = dc[1] * dd[2] - dc[2] * dd[1];
    const float x1 = dc[2] * dd[0] - dc[0] * dd[2];
    const float x2 = dc[0] * dd[1] - dc[1] * dd[0];
    const float ndc2 = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2];
    // hardware square root and reciprocal (a few ulp): the sum only has to land within 1e-4 of
    // the reference's, and sections closer than that to a step of ceil() are redone in FP64
    float nx, rn;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(nx) : "f"(x0 * x0 + x1 * x1 + x2 * x2));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rn) : "f"(ndc2));
    th = fmaf(nx, rn, th);
}

// Sections in three passes (n_sec + 1 slots per line; slot n_sec is the periodic copy): the
// quintic coefficients and the sample step, one thread per slot (section_coe_kernel); the
// turning-angle sum, one warp per slot (section_kernel); ntf and dtf, one thread per slot
// (section_ntf_kernel).  The FP64 arithmetic of the first and last pass runs on every lane
// instead of three lanes of the summing warp.

// get_spline_5th_coe (subroutine.f90:440-461) for the three coordinates of slot s, and the FP32
// sample step dtf_pre * Len of the turning-angle sum.
__global__ void section_coe_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                                   const double *__restrict__ X, const double *__restrict__ Y,
                                   const double *__restrict__ Z, const double *__restrict__ cze,
                                   const double *__restrict__ ck, const double *__restrict__ ckk,
                                   const double *__restrict__ Len, int64_t node_base, int ntf_pre,
                                   double *__restrict__ coe_out, float *__restrict__ zstep_out)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int l = slot_line[s];
    const LineParam P = lp[l];
    const int t = (int)(s - P.slot_off);
    const int np = P.n_sec;
    const int64_t o = P.node_off - node_base;
    const double L = Len[l];
    const double *cz_line = cze + o;
    // nodes of the left/right ends of the section (periodic extension, tube.f90:574-596)
    const int il = t < np ? t : t - np;
    const int ir = (t + 1) < np ? (t + 1) : (t + 1 - np);
    const double zl = cze_pl_at(cz_line, np, t), zr_ = cze_pl_at(cz_line, np, t + 1);
    // spline argument is cze_pl*Len (tube.f90:598)
    const double zr = zr_ * L - zl * L;
    const double z2 = zr * zr, z3 = z2 * zr, z4 = z3 * zr, z5 = z4 * zr;
#pragma unroll 1
    for (int d = 0; d < 3; ++d) {
        const double *cd = (d == 0 ? X : (d == 1 ? Y : Z)) + P.node_off;
        const double xl = cd[il], xr = cd[ir];
        const double vl = ck[3 * (o + il) + d], vr = ck[3 * (o + ir) + d];
        const double al = ckk[3 * (o + il) + d], ar = ckk[3 * (o + ir) + d];
        double xpl = xl, xpr = xr;
        if (xl - xr > dev_pi()) xpr = xr + dev_pi2();
        else if (xl - xr < -dev_pi()) xpl = xl + dev_pi2();
        double *a6 = coe_out + 18 * s + 6 * d;
        a6[0] = xl;
        a6[1] = vl;
        a6[2] = al / 2.0;
        a6[3] = (20.0 * (xpr - xpl) - (12.0 * vl + 8.0 * vr) * zr - (3.0 * al - ar) * z2) / (2.0 * z3);
        a6[4] = (-30.0 * (xpr - xpl) + (16.0 * vl + 14.0 * vr) * zr + (3.0 * al - 2.0 * ar) * z2) / (2.0 * z4);
        a6[5] = (12.0 * (xpr - xpl) - 6.0 * (vl + vr) * zr - (al - ar) * z2) / (2.0 * z5);
    }
    const double dtfp = (zr_ - zl) / (1.0 * ntf_pre);
    zstep_out[s] = (float)(dtfp * L);
}

// The turning-angle sum of slot `warp` (tube.f90:625-657): sum |c' x c''| / |c'|^2 over
// ntf_pre + 1 samples, the integrand in FP32 from the FP32 coefficients, the sum in FP64
// (without the factor dtf_pre * Len, applied by section_ntf_kernel).
__global__ void section_kernel(int64_t nslots, int ntf_pre, const double *__restrict__ coe,
                               const float *__restrict__ zstep_in, double *__restrict__ tsum_out)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    // lane m < 18 loads coefficient m; every lane takes the FP32 derivative coefficients by
    // shuffles, scaled once (1, 2, 3, 4, 5 for c' and 2, 6, 12, 20 for c'')
    const float mine = lane < 18 ? (float)coe[18 * warp + lane] : 0.0f;
    float d1[3][5], d2[3][4];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
#pragma unroll
        for (int m = 1; m <= 5; ++m) d1[d][m - 1] = (float)m * __shfl_sync(0xffffffffu, mine, 6 * d + m);
#pragma unroll
        for (int m = 2; m <= 5; ++m) d2[d][m - 2] = (float)(m * (m - 1)) * __shfl_sync(0xffffffffu, mine, 6 * d + m);
    }
    const float zstep = zstep_in[warp], z64 = 64.0f * zstep;
    float th0 = 0.0f, th1 = 0.0f;
    int tj = lane;
    float za = zstep * (float)lane, zb = zstep * (float)(lane + 32);
    for (; tj + 32 <= ntf_pre; tj += 64) {   // two independent samples per step
        turning_integrand(d1, d2, za, th0);
        turning_integrand(d1, d2, zb, th1);
        za += z64;
        zb += z64;
    }
    if (tj <= ntf_pre) turning_integrand(d1, d2, za, th0);
    const double sum = warp_sum((double)th0 + (double)th1);
    if (lane == 0) tsum_out[warp] = sum;
}

// ntf = ceil(ntf_times theta / 2 pi) + 1 and dtf of slot s, theta = sum * dtf_pre * Len.  The
// integrand was evaluated in FP32; a result that falls near a step of ceil is marked (ntf = 0)
// and recomputed in FP64 by section_fp64_kernel.
__global__ void section_ntf_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                                   const double *__restrict__ cze, const double *__restrict__ Len, int64_t node_base,
                                   int ntf_times, int ntf_pre, const double *__restrict__ tsum,
                                   int *__restrict__ ntf_out, double *__restrict__ dtf_out,
                                   unsigned *__restrict__ near)   // near[0]: count, near[4 + i]: marked slots
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const int l = slot_line[s];
    const LineParam P = lp[l];
    const int t = (int)(s - P.slot_off);
    const int np = P.n_sec;
    const double L = Len[l];
    const double *cz_line = cze + (P.node_off - node_base);
    const double zl = cze_pl_at(cz_line, np, t), zr_ = cze_pl_at(cz_line, np, t + 1);
    const double dtfp = (zr_ - zl) / (1.0 * ntf_pre);
    const double th32 = tsum[s] * dtfp * L;
    const double xr = ntf_times * th32 / dev_pi2();
    const double fr = xr - floor(xr);
    const bool near_step = fmin(fr, 1.0 - fr) < 1e-4 * (xr + 1.0) || !(xr == xr);
    const int ntf = near_step ? 0 : (int)ceil(xr) + 1;
    if (near_step) near[4 + atomicAdd(near, 1u)] = (unsigned)s;
    ntf_out[s] = ntf;
    dtf_out[s] = near_step ? 0.0 : (zr_ - zl) / (1.0 * ntf);
}

// FP64 turning angle of the sections section_kernel marked (ntf = 0), taken from its list of
// them (a few per thousand): a fixed grid of warps strides over the list, one section per warp
// at a time, with the reference's integrand (tube.f90:625-657) in FP64 from the stored
// coefficients.
__global__ void section_fp64_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line,
                                    const double *__restrict__ cze, const double *__restrict__ Len,
                                    int64_t node_base, int ntf_times, int ntf_pre, const double *__restrict__ coe_all,
                                    const unsigned *__restrict__ near, int *__restrict__ ntf_out,
                                    double *__restrict__ dtf_out)
{
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned count = near[0];
    const int lane = threadIdx.x & 31;
    for (unsigned i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += nwarps) {
        const int64_t warp = near[4 + i];
        const int l = slot_line[warp];
        const LineParam P = lp[l];
        const int t = (int)(warp - P.slot_off);
        const int np = P.n_sec;
        const double L = Len[l];
        const double *cz_line = cze + (P.node_off - node_base);
        const double zl = cze_pl_at(cz_line, np, t), zr_ = cze_pl_at(cz_line, np, t + 1);
        const double dtfp = (zr_ - zl) / (1.0 * ntf_pre);
        const double *coe = coe_all + 18 * (size_t)warp;
        double th = 0.0;
        for (int tj = lane; tj <= ntf_pre; tj += 32) {
            const double s = zl + dtfp * tj;
            const double z = (s - zl) * L;
            double dc[3], dd[3];
    #pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double *a = coe + 6 * d;
                dc[d] = (((5.0 * a[5] * z + 4.0 * a[4]) * z + 3.0 * a[3]) * z + 2.0 * a[2]) * z + a[1];
                dd[d] = ((20.0 * a[5] * z + 12.0 * a[4]) * z + 6.0 * a[3]) * z + 2.0 * a[2];
            }
            const double x0 = dc[1] * dd[2] - dc[2] * dd[1];
            const double x1 = dc[2] * dd[0] - dc[0] * dd[2];
            const double x2 = dc[0] * dd[1] - dc[1] * dd[0];
            const double ndc2 = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2];
            th += sqrt(x0 * x0 + x1 * x1 + x2 * x2) / ndc2 * dtfp * L;
        }
        th = warp_sum(th);
        if (lane == 0) {
            const int ntf = (int)ceil(ntf_times * th / dev_pi2()) + 1;
            ntf_out[warp] = ntf;
            dtf_out[warp] = (zr_ - zl) / (1.0 * ntf);
        }
    }
}

// per-slot counts for the scans: samples (ntf+1) and sub-segments (ntf for real sections)
__global__ void slot_counts_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line,
                                   int64_t nslots, const int *__restrict__ ntf, int64_t *__restrict__ nsamp,
                                   int64_t *__restrict__ nsub)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const LineParam P = lp[slot_line[s]];
    const int t = (int)(s - P.slot_off);
    nsamp[s] = ntf[s] + 1;
    nsub[s] = t < P.n_sec ? ntf[s] : 0;
}

// per-line ntf sum (over all n_sec+1 slots) and max, for test_data.dat (tube.f90:672-676)
__global__ void line_ntf_stats_kernel(const LineParam *__restrict__ lp, int nlines, const int *__restrict__ ntf,
                                      int64_t *__restrict__ out)
{
    const int l = blockIdx.x;
    if (l >= nlines) return;
    const LineParam P = lp[l];
    int64_t sum = 0;
    int mx = 0;
    for (int t = threadIdx.x; t < P.n_sec + 1; t += blockDim.x) {
        const int v = ntf[P.slot_off + t];
        sum += v;
        mx = max(mx, v);
    }
    __shared__ int64_t ssum[32];
    __shared__ int smax[32];
    sum = warp_sum(sum);
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o2));
    if ((threadIdx.x & 31) == 0) { ssum[threadIdx.x >> 5] = sum; smax[threadIdx.x >> 5] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t s = 0;
        int m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s += ssum[w]; m = max(m, smax[w]); }
        out[2 * l] = s;
        out[2 * l + 1] = m;
    }
}

// ------------------------------------------------------------------ sample points
// One warp per slot; samples t_j = 0..ntf at s = cze_pl(t) + dtf*t_j (tube.f90:706-713),
// with ci(t, ntf) replaced by ci(t+1, 1) for real sections (tube.f90:721-723).
__global__ void sample_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                              const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
                              const double *__restrict__ cze, const double *__restrict__ Len, int64_t node_base,
                              const double *__restrict__ coe, const int *__restrict__ ntf,
                              const double *__restrict__ dtf, const int64_t *__restrict__ soff,
                              double *__restrict__ s_out, double *__restrict__ ci_out)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    const int l = slot_line[warp];
    const LineParam P = lp[l];
    const int t = (int)(warp - P.slot_off);
    const int np = P.n_sec;
    const double L = Len[l];
    const double zl = cze_pl_at(cze + (P.node_off - node_base), np, t);
    double cf[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) cf[k] = coe[18 * warp + k];
    const int n = ntf[warp];
    const double d = dtf[warp];
    const int64_t base = soff[warp];
    for (int tj = lane; tj <= n; tj += 32) {
        const double s = zl + d * tj;
        s_out[base + tj] = s;
        double c3[3];
        if (tj == n && t < np) {
            // endpoint copy: ci(t+1, 1) is the spline of slot t+1 at 0, i.e. node t+1
            const int inext = (t + 1 < np) ? t + 1 : 0;
            c3[0] = X[P.node_off + inext];
            c3[1] = Y[P.node_off + inext];
            c3[2] = Z[P.node_off + inext];
        } else {
            spl_pos(cf, (s - zl) * L, c3);
        }
        ci_out[3 * (base + tj) + 0] = c3[0];
        ci_out[3 * (base + tj) + 1] = c3[1];
        ci_out[3 * (base + tj) + 2] = c3[2];
    }
}


// ------------------------------------------------------------------ chords
// One warp per real section; tci(t, t_j) for t_j = 0..ntf; t_j = ntf uses the first
// chord of the next slot (tube.f90:740-751).
__global__ void chord_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                             const int *__restrict__ ntf, const int64_t *__restrict__ soff,
                             const double *__restrict__ ci, double *__restrict__ tci, double *__restrict__ ndci)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    const LineParam P = lp[slot_line[warp]];
    const int t = (int)(warp - P.slot_off);
    if (t >= P.n_sec) return;
    const int n = ntf[warp];
    const int64_t base = soff[warp], nbase = soff[warp + 1];
    for (int tj = lane; tj <= n; tj += 32) {
        const int64_t a = tj < n ? base + tj : nbase;
        const int64_t b = tj < n ? base + tj + 1 : nbase + 1;
        double dc[3];
        cminus3(ci + 3 * b, ci + 3 * a, dc);
        const double nn = sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
        ndci[base + tj] = nn;
        tci[3 * (base + tj) + 0] = dc[0] / nn;
        tci[3 * (base + tj) + 1] = dc[1] / nn;
        tci[3 * (base + tj) + 2] = dc[2] / nn;
    }
}

// ------------------------------------------------------------------ sub-segment records
__global__ void subseg_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                              const int *__restrict__ ntf, const int64_t *__restrict__ soff,
                              const int64_t *__restrict__ qoff, const double *__restrict__ s_in,
                              const double *__restrict__ ci, const double *__restrict__ tci,
                              const double *__restrict__ ndci, int line_base, int N, double Rtube_ratio,
                              SubSeg *__restrict__ out, SegRec *__restrict__ rec, const double *__restrict__ coe,
                              const double *__restrict__ dtf, double dzeta_sup, double eta)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    const int l = slot_line[warp];
    const LineParam P = lp[l];
    const int t = (int)(warp - P.slot_off);
    if (t >= P.n_sec) return;
    const int n = ntf[warp];
    const int64_t base = soff[warp], q0 = qoff[warp];
    const double dx = dev_pi2() / N, xstart = -dev_pi();
    for (int tj = lane; tj < n; tj += 32) {
        SubSeg S;
        const double s0 = s_in[base + tj], s1 = s_in[base + tj + 1];
        double c0[3], c1[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            c0[d] = ci[3 * (base + tj) + d];
            c1[d] = ci[3 * (base + tj + 1) + d];
            // mark1 unwrap (tube.f90:779-785)
            if (c1[d] - c0[d] > dev_pi()) c0[d] = c0[d] + dev_pi2();
            else if (c1[d] - c0[d] < -dev_pi()) c1[d] = c1[d] + dev_pi2();
            S.ci0[d] = c0[d];
            S.ci1[d] = c1[d];
            S.tci0[d] = tci[3 * (base + tj) + d];
            S.tci1[d] = tci[3 * (base + tj + 1) + d];
        }
        S.s0 = s0;
        S.s1 = s1;
        S.ndci0 = ndci[base + tj];
        S.ssec = s_in[base];
        S.zs0 = s0 - s_in[base];
        double Rt = Rtube_ratio * sigma_func(s0, P.length, P.sigma_max, P.sigma_min, P.n_T);
        const double r1 = Rtube_ratio * sigma_func(s1, P.length, P.sigma_max, P.sigma_min, P.n_T);
        Rt = fmax(Rt, r1);
        S.Rt = Rt;
        S.slot = (int)warp;
        S.line = l + line_base;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double mn = fmin(c0[d], c1[d]), mx = fmax(c0[d], c1[d]);
            // i_min = floor((min - xstart - Rtube)/dx + 1), i_max = ceiling((max - xstart + Rtube)/dx + 1)
            S.box_lo[d] = (int)floor(dadd(__ddiv_rn(dsub(dsub(mn, xstart), Rt), dx), 1.0));
            S.box_hi[d] = (int)ceil(dadd(__ddiv_rn(dadd(dsub(mx, xstart), Rt), dx), 1.0));
        }
        if (out) out[q0 + tj] = S;
        if (rec) {
            SegF G;
            seg_setup_f32(S, P, coe, dtf[warp], dzeta_sup, eta, N, S.box_lo[0], S.box_lo[1], S.box_lo[2], G);
            SegRec R;
            segrec_from(G, S, R);
            rec[q0 + tj] = R;
        }
    }
}

// ------------------------------------------------------------------ fused sub-segment records
// Sub-segment records straight from the spline coefficients, one thread per sub-segment
// (tube.f90:706-798): each thread evaluates the three sample points it needs (ci_j, ci_j+1,
// ci_j+2), the two chords and the FP32 record, with no sample arrays in global memory.
// Extended samples of section t: ci_j (j < ntf) on the spline, ci_ntf = node t+1 (the endpoint
// copy, tube.f90:721-723) and ci_{ntf+1} = the first sample of section t+1, so that
// chord_j = cminus(ci_{j+1}, ci_j) covers j = 0..ntf (tube.f90:740-751).

// slot of every sub-segment of the batch (one warp per section)
__global__ void subseg_map_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                                  const int *__restrict__ ntf, const int64_t *__restrict__ qoff, int *__restrict__ map)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    const LineParam &P = lp[slot_line[warp]];
    if ((int)(warp - P.slot_off) >= P.n_sec) return;
    const int n = ntf[warp];
    const int64_t q0 = qoff[warp];
    for (int j = lane; j < n; j += 32) map[q0 + j] = (int)warp;
}

__global__ void __launch_bounds__(256) subseg_fused_kernel(
    const LineParam *__restrict__ lp, const int *__restrict__ slot_line, const int *__restrict__ map, int64_t nsub,
    const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
    const double *__restrict__ cze, int64_t node_base, const double *__restrict__ coe, const int *__restrict__ ntf,
    const double *__restrict__ dtf, const int64_t *__restrict__ qoff, int line_base, int N, double Rtube_ratio,
    double dzeta_sup, double eta, SegRec *__restrict__ rec)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub) return;
    const int slot = map[q];
    const int l = slot_line[slot];
    const LineParam P = lp[l];
    const int t = slot - (int)P.slot_off;
    const int np = P.n_sec;
    const int j = (int)(q - qoff[slot]);
    const int n = ntf[slot];
    const double L = P.Len;
    const double *czl = cze + (P.node_off - node_base);
    const double zl = cze_pl_at(czl, np, t), zl1 = cze_pl_at(czl, np, t + 1);
    const double d = dtf[slot];
    const double *cf = coe + 18 * (size_t)slot;
    const int inext = (t + 1 < np) ? t + 1 : 0;
    // extended sample k of this section (k = j, j+1, j+2)
    auto sample = [&](int k, double *c3) {
        if (k < n) {
            spl_pos_fma(cf, (zl + d * k - zl) * L, c3);
        } else if (k == n) {
            c3[0] = X[P.node_off + inext];
            c3[1] = Y[P.node_off + inext];
            c3[2] = Z[P.node_off + inext];
        } else {
            spl_pos_fma(coe + 18 * (size_t)(slot + 1), (zl1 + dtf[slot + 1] * 1 - zl1) * L, c3);
        }
    };
    double c0[3], c1[3], c2[3];
    sample(j, c0);
    sample(j + 1, c1);
    sample(j + 2, c2);
    double ch0[3], ch1[3];
    cminus3(c1, c0, ch0);
    cminus3(c2, c1, ch1);
    const double n0 = sqrt(ch0[0] * ch0[0] + ch0[1] * ch0[1] + ch0[2] * ch0[2]);
    const double n1 = sqrt(ch1[0] * ch1[0] + ch1[1] * ch1[1] + ch1[2] * ch1[2]);
    const double i0 = 1.0 / n0, i1 = 1.0 / n1;
    SubSeg S;
    const double s0 = zl + d * j, s1 = zl + d * (j + 1);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double a = c0[k], b = c1[k];
        if (b - a > dev_pi()) a = a + dev_pi2();   // mark1, tube.f90:779-785
        else if (b - a < -dev_pi()) b = b + dev_pi2();
        S.ci0[k] = a;
        S.ci1[k] = b;
        S.tci0[k] = ch0[k] * i0;
        S.tci1[k] = ch1[k] * i1;
    }
    S.s0 = s0;
    S.s1 = s1;
    S.ndci0 = n0;
    S.ssec = zl;
    S.zs0 = s0 - zl;
    double Rt;
    if (P.sigma_max == P.sigma_min) {
        Rt = Rtube_ratio * P.sigma_min;   // sigma_func is exactly sigma_min when sigma_max = sigma_min
    } else {
        Rt = Rtube_ratio * sigma_func(s0, P.length, P.sigma_max, P.sigma_min, P.n_T);
        Rt = fmax(Rt, Rtube_ratio * sigma_func(s1, P.length, P.sigma_max, P.sigma_min, P.n_T));
    }
    S.Rt = Rt;
    S.slot = slot;
    S.line = l + line_base;
    const double inv_dx = (double)N / dev_pi2(), xstart = -dev_pi();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double mn = fmin(S.ci0[k], S.ci1[k]), mx = fmax(S.ci0[k], S.ci1[k]);
        // i_min = floor((min - xstart - Rtube)/dx + 1), i_max = ceiling((max - xstart + Rtube)/dx + 1)
        S.box_lo[k] = (int)floor((mn - xstart - Rt) * inv_dx + 1.0);
        S.box_hi[k] = (int)ceil((mx - xstart + Rt) * inv_dx + 1.0);
    }
    SegF G;
    seg_setup_f32(S, P, coe, d, dzeta_sup, eta, N, S.box_lo[0], S.box_lo[1], S.box_lo[2], G);
    SegRec R;
    segrec_from(G, S, R);
    rec[q] = R;
}


// FP64 sub-segment records of the FP64 tile path, one thread per sub-segment, built by the same
// device code as the records of the FP64 redo (redo_subseg): the tile kernels decide their
// candidate points in FP32 with a margin and then test and evaluate them in FP64 from these.
__global__ void __launch_bounds__(256) subseg64_kernel(const RedoCtx R, const int *__restrict__ map,
                                                       const int64_t *__restrict__ qoff, int64_t nsub, int line_base,
                                                       SubSeg *__restrict__ out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub) return;
    const int slot = map[q];
    SubSeg S;
    LineParam P;
    redo_subseg(R, slot, (int)(q - qoff[slot]), S, P);
    S.line = R.slot_line[slot] + line_base;
    out[q] = S;
}

// ------------------------------------------------------------------ scan
// Exclusive scan of n int64 values in place; out[n] receives the total.  Three launches:
// block sums, a single-block scan of the block sums, and the per-block scan.
constexpr int kScanBlock = 1024;

__global__ void scan_block_sums(const int64_t *__restrict__ in, int64_t n, int64_t *__restrict__ sums)
{
    const int64_t i0 = (int64_t)blockIdx.x * kScanBlock;
    int64_t v = 0;
    for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x) {
        const int64_t i = i0 + k;
        if (i < n) v += in[i];
    }
    __shared__ int64_t s[32];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void scan_sums_serial(int64_t *__restrict__ sums, int64_t nb, int64_t *__restrict__ total)
{
    // single block; chunked scan with carry
    __shared__ int64_t carry;
    __shared__ int64_t part[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int64_t i = b0 + threadIdx.x;
        const int64_t x = i < nb ? sums[i] : 0;
        int64_t v = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) part[w] = v;
        __syncthreads();
        if (w == 0) {
            int64_t y = lane < nw ? part[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int64_t t = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += t;
            }
            if (lane < nw) part[lane] = y;
        }
        __syncthreads();
        const int64_t incl = v + (w > 0 ? part[w - 1] : 0) + carry;
        if (i < nb) sums[i] = incl - x;  // exclusive
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_apply(int64_t *__restrict__ data, int64_t n, const int64_t *__restrict__ sums)
{
    __shared__ int64_t part[32];
    __shared__ int64_t carry;
    const int64_t i0 = (int64_t)blockIdx.x * kScanBlock;
    if (threadIdx.x == 0) carry = sums[blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k0 = 0; k0 < kScanBlock; k0 += blockDim.x) {
        const int64_t i = i0 + k0 + threadIdx.x;
        const int64_t x = i < n ? data[i] : 0;
        int64_t v = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) part[w] = v;
        __syncthreads();
        if (w == 0) {
            int64_t y = lane < nw ? part[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int64_t t = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += t;
            }
            if (lane < nw) part[lane] = y;
        }
        __syncthreads();
        const int64_t incl = v + (w > 0 ? part[w - 1] : 0) + carry;
        if (i < n) data[i] = incl - x;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
}

int scan_exclusive_i64(Ctx *c, int64_t *d_data, int64_t n, int64_t *d_total, DevBuf &tmp)
{
    const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    FWT_TRY(buf_reserve(c, tmp, sizeof(int64_t) * (size_t)(nb + 1)));
    int64_t *sums = (int64_t *)tmp.p;
    if (nb > 0) {
        scan_block_sums<<<(unsigned)nb, 256, 0, c->stream>>>(d_data, n, sums);
        scan_sums_serial<<<1, 1024, 0, c->stream>>>(sums, nb, d_total);
        scan_apply<<<(unsigned)nb, 256, 0, c->stream>>>(d_data, n, sums);
        c->launches += 3;
    } else {
        FWT_CUDA(cudaMemsetAsync(d_total, 0, sizeof(int64_t), c->stream));
    }
    FWT_CUDA(cudaGetLastError());
    return 0;
}

// ------------------------------------------------------------------ driver
// FP64 sub-segment records of every sub-segment of the batch (the FP64 tile path), after the
// FP32 records: the sub-segment -> section map (built here for a piece batch), then the records.
int subseg64_setup(Ctx *c, CenterlineBatch &B)
{
    Ctx &C = *c;
    const int64_t nsub = std::max<int64_t>(B.nsub, 1);
    const int *map = nullptr;
    const unsigned wblocks = (unsigned)((B.nslots * 32 + 255) / 256);
    int km = kt_begin(c, KT_CENTERLINE);
    if (B.rec) {
        map = B.rec_map;   // the sub-segment batch's own map
    } else {
        FWT_TRY(buf_reserve(c, C.scratch[16], sizeof(int) * (size_t)nsub));
        int *m = (int *)C.scratch[16].p;
        subseg_map_kernel<<<wblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, B.nslots, B.ntf, B.qoff, m);
        c->launches += 1;
        map = m;
    }
    FWT_TRY(buf_reserve(c, C.scratch[17], sizeof(SubSeg) * (size_t)nsub));
    B.seg = (SubSeg *)C.scratch[17].p;
    const RedoCtx R = redo_ctx(c, B, 1.0, B.rec == nullptr);
    if (B.nsub > 0)
        subseg64_kernel<<<(unsigned)((B.nsub + 255) / 256), 256, 0, c->stream>>>(R, map, B.qoff, B.nsub, B.la, B.seg);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    return 0;
}

int centerline_setup(Ctx *c, int la, int lb, CenterlineBatch &B, BatchRecords mode)
{
    // la..lb-1: 0-based lines of this batch
    const int nl = lb - la;
    B.la = la;
    B.nl = nl;
    B.node_base = c->node_off[la];
    int64_t nodes = 0, slots = 0;
    std::vector<LineParam> hp(nl);
    for (int i = 0; i < nl; ++i) {
        const int l = la + i;
        LineParam &P = hp[i];
        P.n_sec = (int)c->npoint[l];
        P.node_off = c->node_off[l];
        P.slot_off = slots;
        P.sigma_min = c->sigma[l];
        P.sigma_max = c->p.sigma_ratio * c->sigma[l];
        P.Gamma = c->Gamma[l];
        P.n_T = c->n_T[l];
        P.length = 0;
        P.Len = 0;
        nodes += P.n_sec;
        slots += P.n_sec + 1;
    }
    B.nodes = nodes;
    B.nslots = slots;

    // buffers
    Ctx &C = *c;
    FWT_TRY(buf_reserve(c, C.scratch[0], sizeof(LineParam) * nl));
    FWT_TRY(buf_reserve(c, C.scratch[1], sizeof(int) * (size_t)slots));
    FWT_TRY(buf_reserve(c, C.scratch[2], sizeof(double) * (size_t)nodes));       // cze
    FWT_TRY(buf_reserve(c, C.scratch[3], sizeof(double) * 3 * (size_t)nodes));   // ck
    FWT_TRY(buf_reserve(c, C.scratch[4], sizeof(double) * 3 * (size_t)nodes));   // ckk
    FWT_TRY(buf_reserve(c, C.scratch[5], sizeof(double) * (size_t)nl));          // Len
    FWT_TRY(buf_reserve(c, C.scratch[6], sizeof(double) * 18 * (size_t)slots));  // coe
    FWT_TRY(buf_reserve(c, C.scratch[7], sizeof(int) * (size_t)slots));          // ntf
    FWT_TRY(buf_reserve(c, C.scratch[8], sizeof(double) * (size_t)slots));       // dtf
    FWT_TRY(buf_reserve(c, C.scratch[9], sizeof(int64_t) * (size_t)(slots + 1)));   // soff
    FWT_TRY(buf_reserve(c, C.scratch[10], sizeof(int64_t) * (size_t)(slots + 1)));  // qoff
    FWT_TRY(buf_reserve(c, C.scratch[11], sizeof(int64_t) * (size_t)(2 * nl + 4))); // line stats + totals
    B.lp = (LineParam *)C.scratch[0].p;
    B.slot_line = (int *)C.scratch[1].p;
    B.cze = (double *)C.scratch[2].p;
    B.ck = (double *)C.scratch[3].p;
    B.ckk = (double *)C.scratch[4].p;
    B.Len = (double *)C.scratch[5].p;
    B.coe = (double *)C.scratch[6].p;
    B.ntf = (int *)C.scratch[7].p;
    B.dtf = (double *)C.scratch[8].p;
    B.soff = (int64_t *)C.scratch[9].p;
    B.qoff = (int64_t *)C.scratch[10].p;
    int64_t *d_misc = (int64_t *)C.scratch[11].p;
    FWT_CUDA(cudaMemcpyAsync(B.lp, hp.data(), sizeof(LineParam) * nl, cudaMemcpyHostToDevice, c->stream));

    int km = kt_begin(c, KT_CENTERLINE);
    // slot -> line on the device (a host table of one int per slot, copied from pageable
    // memory, cost milliseconds per batch)
    slot_line_kernel<<<nl, 256, 0, c->stream>>>(B.lp, nl, B.slot_line);
    line_prep_kernel<<<nl, 256, 0, c->stream>>>(B.lp, nl, c->d_x, c->d_y, c->d_z, B.cze, B.ck, B.ckk, B.Len,
                                                B.node_base);
    c->launches += 1;
    kt_end(c, km);
    const unsigned wblocks = (unsigned)((slots * 32 + 255) / 256);
    km = kt_begin(c, KT_SECTION);
    FWT_TRY(buf_reserve(c, C.scratch[24], sizeof(unsigned) * (size_t)(slots + 4)));   // near-step list
    unsigned *d_near = (unsigned *)C.scratch[24].p;
    FWT_CUDA(cudaMemsetAsync(d_near, 0, sizeof(unsigned), c->stream));
    FWT_TRY(buf_reserve(c, C.scratch[28], (sizeof(double) + sizeof(float)) * (size_t)std::max<int64_t>(slots, 1)));
    double *d_tsum = (double *)C.scratch[28].p;
    float *d_zstep = (float *)(d_tsum + slots);
    const unsigned tblocks = (unsigned)((slots + 255) / 256);
    section_coe_kernel<<<tblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, c->d_x, c->d_y, c->d_z, B.cze, B.ck,
                                                      B.ckk, B.Len, B.node_base, c->p.ntf_pre, B.coe, d_zstep);
    section_kernel<<<wblocks, 256, 0, c->stream>>>(slots, c->p.ntf_pre, B.coe, d_zstep, d_tsum);
    section_ntf_kernel<<<tblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.cze, B.Len, B.node_base,
                                                      c->p.ntf_times, c->p.ntf_pre, d_tsum, B.ntf, B.dtf, d_near);
    // a fixed grid: the list holds a few sections per thousand
    section_fp64_kernel<<<4 * 148, 256, 0, c->stream>>>(B.lp, B.slot_line, B.cze, B.Len, B.node_base,
                                                        c->p.ntf_times, c->p.ntf_pre, B.coe, d_near, B.ntf, B.dtf);
    c->launches += 4;
    kt_end(c, km);
    km = kt_begin(c, KT_CENTERLINE);
    slot_counts_kernel<<<(unsigned)((slots + 255) / 256), 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf,
                                                                               B.soff, B.qoff);
    line_ntf_stats_kernel<<<nl, 256, 0, c->stream>>>(B.lp, nl, B.ntf, d_misc);
    c->launches += 4;
    FWT_CUDA(cudaGetLastError());
    FWT_TRY(scan_exclusive_i64(c, B.soff, slots, d_misc + 2 * nl, C.scratch[12]));
    FWT_TRY(scan_exclusive_i64(c, B.qoff, slots, d_misc + 2 * nl + 1, C.scratch[13]));
    kt_end(c, km);
    // per-line Len and ntf statistics + totals to the host
    std::vector<int64_t> hmisc((size_t)(2 * nl + 2));
    std::vector<double> hLen((size_t)nl);
    FWT_CUDA(cudaMemcpyAsync(hmisc.data(), d_misc, sizeof(int64_t) * (2 * nl + 2), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(hLen.data(), B.Len, sizeof(double) * nl, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    B.nsamples = hmisc[2 * nl];
    B.nsub = hmisc[2 * nl + 1];
    B.line_ntf_sum.assign(hmisc.begin(), hmisc.begin() + 2 * nl);
    B.Lens = hLen;
    // fill line length (needed by sigma_func) and re-upload the line table
    for (int i = 0; i < nl; ++i) {
        hp[i].Len = hLen[i];
        hp[i].length = hLen[i] * kPi2;
    }
    FWT_CUDA(cudaMemcpyAsync(B.lp, hp.data(), sizeof(LineParam) * nl, cudaMemcpyHostToDevice, c->stream));
    // the scans wrote the totals at [n]: set soff[slots], qoff[slots]
    FWT_CUDA(cudaMemcpyAsync(B.soff + slots, &B.nsamples, sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
    FWT_CUDA(cudaMemcpyAsync(B.qoff + slots, &B.nsub, sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));

    if (mode == BatchRecords::Pieces) {
        FWT_TRY(piece_setup(c, B));
        return c->p.precision == 64 ? subseg64_setup(c, B) : 0;
    }
    // the tile-owned FP32 kernel reads compact FP32 records built by one fused kernel; the box
    // walk reads FP64 records built from sample arrays
    const bool tile_mode = mode == BatchRecords::SubSeg;
    const size_t rec_bytes = tile_mode ? sizeof(SegRec) : sizeof(SubSeg);
    FWT_TRY(buf_reserve(c, C.scratch[18], rec_bytes * (size_t)std::max<int64_t>(B.nsub, 1)));
    if (tile_mode) {
        B.rec = (SegRec *)C.scratch[18].p;
        FWT_TRY(buf_reserve(c, C.scratch[14], sizeof(int) * (size_t)std::max<int64_t>(B.nsub, 1)));
        int *d_map = (int *)C.scratch[14].p;
        B.rec_map = d_map;
        B.rec_first = B.qoff;
        km = kt_begin(c, KT_CENTERLINE);
        subseg_map_kernel<<<wblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf, B.qoff, d_map);
        if (B.nsub > 0)
            subseg_fused_kernel<<<(unsigned)((B.nsub + 255) / 256), 256, 0, c->stream>>>(
                B.lp, B.slot_line, d_map, B.nsub, c->d_x, c->d_y, c->d_z, B.cze, B.node_base, B.coe, B.ntf, B.dtf,
                B.qoff, la, c->p.N, c->p.Rtube_ratio, c->p.dzeta_sup, c->p.eta_t, B.rec);
        kt_end(c, km);
        c->launches += 2;
        FWT_CUDA(cudaGetLastError());
        return c->p.precision == 64 ? subseg64_setup(c, B) : 0;
    }
    FWT_TRY(buf_reserve(c, C.scratch[14], sizeof(double) * (size_t)B.nsamples));        // s
    FWT_TRY(buf_reserve(c, C.scratch[15], sizeof(double) * 3 * (size_t)B.nsamples));    // ci
    FWT_TRY(buf_reserve(c, C.scratch[16], sizeof(double) * 3 * (size_t)B.nsamples));    // tci
    FWT_TRY(buf_reserve(c, C.scratch[17], sizeof(double) * (size_t)B.nsamples));        // ndci
    B.s = (double *)C.scratch[14].p;
    B.ci = (double *)C.scratch[15].p;
    B.tci = (double *)C.scratch[16].p;
    B.ndci = (double *)C.scratch[17].p;
    B.seg = tile_mode ? nullptr : (SubSeg *)C.scratch[18].p;
    B.rec = tile_mode ? (SegRec *)C.scratch[18].p : nullptr;
    km = kt_begin(c, KT_CENTERLINE);
    sample_kernel<<<wblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, c->d_x, c->d_y, c->d_z, B.cze, B.Len,
                                                  B.node_base, B.coe, B.ntf, B.dtf, B.soff, B.s, B.ci);
    chord_kernel<<<wblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf, B.soff, B.ci, B.tci, B.ndci);
    subseg_kernel<<<wblocks, 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf, B.soff, B.qoff, B.s, B.ci, B.tci,
                                                  B.ndci, la, c->p.N, c->p.Rtube_ratio, B.seg, B.rec, B.coe, B.dtf,
                                                  c->p.dzeta_sup, c->p.eta_t);
    kt_end(c, km);
    c->launches += 3;
    FWT_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace fwt
