// k_deposit.cuh -- per-point Burgers-tube arithmetic shared by the deposition kernels.
#pragma once

#include "k_centerline.cuh"

namespace fwt {

// FP32 view of one sub-segment, local to its start point ci0 and to a grid-index origin.
struct SegF {
    float off[3];     // mesh point at the origin index minus ci0
    float dx;
    float tc0[3], tc1[3], dci[3];
    float g;          // W = t0 * g is the spline argument measured from the start, times Len
    float b[3][5];    // c(z0 + W) - c(z0) = sum_k b[k-1] W^k
    float R2, Rt;
    float smin, A, ph0, om, q;   // sigma = smin + A (sin(ph0 + om W) + 1); dsigma/dzeta = q cos(.)
    float Gamma, Linv, eta;
    // periodic bookkeeping of the reference's two single wraps (coo_curve_spline_5th wraps
    // c(zeta) once into [-pi,pi), cminus wraps x - c once): x - c(z) = (d0 - P) + 2 pi n with
    // n = kq + (P >= thi) - (P < tlo), then one cminus wrap
    int kq[3];        // (ci0 - poly(z0)) / 2pi
    float thi[3];     // pi - poly(z0): poly(z) >= pi  <=>  P >= thi
    float tlo[3];     // -pi - poly(z0): poly(z) < -pi <=>  P < tlo
};

// ---------------------------------------------------------------------------- FP32 set-up
__device__ __forceinline__ void seg_setup_f32(const SubSeg &S, const LineParam &P, const double *__restrict__ coe_all,
                              double dtf, double dzeta_sup, double eta0, int N, int i0, int j0, int k0, SegF &G)
{
    const double dx = dev_pi2() / N, xstart = -dev_pi();
    const double *coe = coe_all + 18 * (size_t)S.slot;
    const double L = P.Len;
    const int org[3] = {i0, j0, k0};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        // mesh coordinate of the 1-based unwrapped index org[d]: (i_plus - 1)*dx + xstart
        const double X0 = dadd(dmul((double)org[d] - 1.0, dx), xstart);
        G.off[d] = (float)(X0 - S.ci0[d]);
        G.tc0[d] = (float)S.tci0[d];
        G.tc1[d] = (float)S.tci1[d];
        G.dci[d] = (float)(S.ci1[d] - S.ci0[d]);
    }
    G.dx = (float)dx;
    G.g = (float)((S.s1 - S.s0) * L * (1.0 / S.ndci0));
    // Taylor shift of the quintic around z0 = zs0 * Len by repeated synthetic division:
    // c(z0 + W) = sum_k b_k W^k, b_0 = c(z0) (the unwrapped polynomial value at the start)
    const double z0 = S.zs0 * L;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double a[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) a[m] = coe[6 * d + m];
#pragma unroll
        for (int k = 0; k < 5; ++k)
#pragma unroll
            for (int j = 4; j >= k; --j) a[j] = fma(z0, a[j + 1], a[j]);
#pragma unroll
        for (int k = 1; k <= 5; ++k) G.b[d][k - 1] = (float)a[k];
        const double c0 = a[0];
        G.kq[d] = (int)rint((S.ci0[d] - c0) * (1.0 / dev_pi2()));
        G.thi[d] = (float)(dev_pi() - c0);
        G.tlo[d] = (float)(-dev_pi() - c0);
    }
    G.R2 = (float)(S.Rt * S.Rt);
    G.Rt = (float)S.Rt;
    // core size sigma(zeta) = smin + A (sin(omega zeta) + 1), zeta = s0 + W/Len
    const double omega = floor(P.length / dev_pi() + 0.5) * (double)P.n_T;
    const double A = (P.sigma_max - P.sigma_min) / 2.0;
    G.smin = (float)P.sigma_min;
    G.A = (float)A;
    G.om = (float)(omega / L);
    if (A == 0.0) {
        // constant core: sigma = sigma_min and d sigma / d zeta = 0 exactly
        G.ph0 = 0.0f;
        G.q = 0.0f;
    } else {
        G.ph0 = (float)fmod(omega * S.s0, dev_pi2());
        // central difference of dsigmadzeta (subroutine.f90:748-761) in closed form:
        // (sigma(z+h) - sigma(z-h)) / (2h) = A cos(omega z) sin(omega h) / h
        const double h = fmin(dzeta_sup, 1.0 * dtf);
        G.q = (float)(A * sin(omega * h) / h);
    }
    G.Gamma = (float)P.Gamma;
    G.Linv = (float)(1.0 / L);
    G.eta = (float)eta0;
}


// Contribution of sub-segment G at grid offset (ii, jj, kk) from G's origin index
// (tube.f90:806-892 in the local frame).  General=false is the exact specialisation for a
// constant core (sigma_ratio = 1) and no twist (eta = 0), where the reference's vorticity
// reduces to tp * Gamma * T.
template <bool General>
__device__ __forceinline__ bool point_f32(const SegF &G, int ii, int jj, int kk, float out[3])
{
    const float d0x = fmaf((float)ii, G.dx, G.off[0]);
    const float d0y = fmaf((float)jj, G.dx, G.off[1]);
    const float d0z = fmaf((float)kk, G.dx, G.off[2]);
    const float t0 = d0x * G.tc0[0] + d0y * G.tc0[1] + d0z * G.tc0[2];
    if (!(t0 >= 0.0f)) return false;
    const float ex = d0x - G.dci[0], ey = d0y - G.dci[1], ez = d0z - G.dci[2];
    const float t1 = ex * G.tc1[0] + ey * G.tc1[1] + ez * G.tc1[2];
    if (!(t1 < 0.0f)) return false;
    const float r2 = d0x * d0x + d0y * d0y + d0z * d0z - t0 * t0;
    if (!(r2 < G.R2)) return false;
    const float W = t0 * G.g;
    float P[3], c1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float *b = G.b[d];
        P[d] = W * fmaf(W, fmaf(W, fmaf(W, fmaf(W, b[4], b[3]), b[2]), b[1]), b[0]);
        c1[d] = fmaf(W, fmaf(W, fmaf(W, fmaf(W, 5.0f * b[4], 4.0f * b[3]), 3.0f * b[2]), 2.0f * b[1]), b[0]);
    }
    float xc[3] = {d0x - P[0], d0y - P[1], d0z - P[2]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        // x - wrap(c(z)) of the reference, then its cminus wrap (see SegF::kq)
        int n = G.kq[d] + (P[d] >= G.thi[d] ? 1 : 0) - (P[d] < G.tlo[d] ? 1 : 0);
        const float v = n ? fmaf(6.28318530717958647692f, (float)n, xc[d]) : xc[d];
        if (v > 3.14159265358979f) n -= 1;
        else if (v < -3.14159265358979f) n += 1;
        if (n) xc[d] = fmaf(6.28318530717958647692f, (float)n, xc[d]);
    }
    const float rho2 = xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2];
    const float n1 = sqrtf(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    const float in1 = 1.0f / n1;
    const float T[3] = {c1[0] * in1, c1[1] * in1, c1[2] * in1};
    if constexpr (!General) {
        const float s2 = G.smin * G.smin;
        const float inv2s2 = 0.5f / s2;
        const float tp = (expf(-rho2 * inv2s2) - expf(-G.R2 * inv2s2)) * (0.159154943f / s2) * G.Gamma;
        out[0] = tp * T[0];
        out[1] = tp * T[1];
        out[2] = tp * T[2];
        return true;
    } else {
        float c2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float *b = G.b[d];
            c2[d] = fmaf(W, fmaf(W, fmaf(W, 20.0f * b[4], 12.0f * b[3]), 6.0f * b[2]), 2.0f * b[1]);
        }
        const float ph = fmaf(G.om, W, G.ph0);
        float sn, cs;
        sincosf(ph, &sn, &cs);
        const float sigma = fmaf(G.A, sn + 1.0f, G.smin);
        const float s2 = sigma * sigma;
        const float inv2s2 = 0.5f / s2;
        const float tp = (expf(-rho2 * inv2s2) - expf(-G.R2 * inv2s2)) * (0.159154943f / s2) * G.Gamma;
        const float dsds = G.q * cs * in1 * G.Linv;
        const float rho = sqrtf(rho2);
        const float X[3] = {c1[1] * c2[2] - c1[2] * c2[1], c1[2] * c2[0] - c1[0] * c2[2], c1[0] * c2[1] - c1[1] * c2[0]};
        const float nX = sqrtf(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
        const float inr = 1.0f / (rho + 1.0e-15f);
        if (nX < 1.0e-8f) {
            const float er[3] = {xc[0] * inr, xc[1] * inr, xc[2] * inr};
            const float eth[3] = {er[1] * T[2] - er[2] * T[1], er[2] * T[0] - er[0] * T[2], er[0] * T[1] - er[1] * T[0]};
            const float a = G.eta * rho, bq = rho * dsds / sigma;
#pragma unroll
            for (int d = 0; d < 3; ++d) out[d] = tp * (T[d] + a * eth[d] + bq * er[d]);
        } else {
            const float inX = 1.0f / nX;
            const float B[3] = {X[0] * inX, X[1] * inX, X[2] * inX};
            const float Nv[3] = {B[1] * T[2] - B[2] * T[1], B[2] * T[0] - B[0] * T[2], B[0] * T[1] - B[1] * T[0]};
            const float kap = nX * in1 * in1 * in1;
            const float costh = (xc[0] * Nv[0] + xc[1] * Nv[1] + xc[2] * Nv[2]) * inr;
            const float sinth = (xc[0] * B[0] + xc[1] * B[1] + xc[2] * B[2]) * inr;
            const float iden = 1.0f / (1.0f - kap * rho * costh);
            const float t5 = -sinth * rho * iden, t6 = costh * rho * iden;
            const float t7 = costh * rho * dsds / sigma * iden, t8 = sinth * rho * dsds / sigma * iden;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                out[d] = tp * (T[d] + G.eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
        }
        return true;
    }
}

constexpr int kNoWrap = 1 << 20;   // SegRec::kq[0] marker: the record never needs the wrap logic

// Compact FP32 record of one sub-segment for the tile kernel (224 bytes, 16-byte aligned):
// the local frame of SegF taken at the box origin box_lo, the line constants, and the box.
struct __align__(16) SegRec {
    float off[3], g;        // off: mesh point at box_lo minus ci0
    float tc0[3], R2;
    float tc1[3], ph0;
    float dci[3], q;
    float b[15], smin;
    float thi[3], A;
    float tlo[3], om;
    float Gamma, Linv, eta, dx;
    int kq[3];
    float inv2s2;           // constant core: 1 / (2 sigma^2)
    int box_lo[3];
    float ftd;              // constant core: exp(-Rtube^2 / (2 sigma^2)), the truncation offset
    int box_hi[3];
    float amp;              // constant core: Gamma / (2 pi sigma^2)
};
static_assert(sizeof(SegRec) == 224, "SegRec layout");

__device__ __forceinline__ void segrec_from(const SegF &G, const SubSeg &S, SegRec &R)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        R.off[d] = G.off[d];
        R.tc0[d] = G.tc0[d];
        R.tc1[d] = G.tc1[d];
        R.dci[d] = G.dci[d];
        R.thi[d] = G.thi[d];
        R.tlo[d] = G.tlo[d];
        R.kq[d] = G.kq[d];
        R.box_lo[d] = S.box_lo[d];
        R.box_hi[d] = S.box_hi[d];
#pragma unroll
        for (int k = 0; k < 5; ++k) R.b[5 * d + k] = G.b[d][k];
    }
    R.g = G.g;
    R.R2 = G.R2;
    R.ph0 = G.ph0;
    R.q = G.q;
    R.smin = G.smin;
    R.A = G.A;
    R.om = G.om;
    R.Gamma = G.Gamma;
    R.Linv = G.Linv;
    R.eta = G.eta;
    R.dx = G.dx;
    // per-record constants of the constant-core profile (tube.f90:845-847 with sigma = smin)
    const float s2 = G.smin * G.smin;
    R.inv2s2 = 0.5f / s2;
    R.ftd = expf(-G.R2 * R.inv2s2);
    R.amp = G.Gamma * (0.159154943091895336f / s2);
    // No-wrap flag (kq[0] = kNoWrap): for every point that passes the tests, |W| <= Wm, so
    // |P| stays clear of both wrap thresholds and |x - c| < pi; the wrap bookkeeping of
    // point_rec then reduces to x - c = d0 - P.
    const float dl = sqrtf(G.dci[0] * G.dci[0] + G.dci[1] * G.dci[1] + G.dci[2] * G.dci[2]);
    const float Wm = (dl + G.Rt) * fabsf(G.g) * 1.01f;
    bool nowrap = true;
    float pmax = 0.0f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float *b = G.b[d];
        const float pb = Wm * (fabsf(b[0]) + Wm * (fabsf(b[1]) + Wm * (fabsf(b[2]) + Wm * (fabsf(b[3]) + Wm * fabsf(b[4])))));
        pmax = fmaxf(pmax, pb);
        if (G.kq[d] != 0 || !(G.thi[d] > pb * 1.01f + 1e-5f) || !(G.tlo[d] < -pb * 1.01f - 1e-5f)) nowrap = false;
    }
    if ((dl + 2.0f * G.Rt) * 1.7321f + pmax > 3.0f) nowrap = false;
    // t0 <= dl + Rt tan(bend) <= dl + Rt holds for bends below 45 degrees
    if (G.tc0[0] * G.tc1[0] + G.tc0[1] * G.tc1[1] + G.tc0[2] * G.tc1[2] < 0.75f) nowrap = false;
    if (nowrap) R.kq[0] = kNoWrap;
}

// SegF of record R with its origin moved by (di, dj, dk) grid points from box_lo
__device__ __forceinline__ void segf_from(const SegRec &R, int di, int dj, int dk, SegF &G)
{
    const int dd[3] = {di, dj, dk};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        G.off[d] = fmaf((float)dd[d], R.dx, R.off[d]);
        G.tc0[d] = R.tc0[d];
        G.tc1[d] = R.tc1[d];
        G.dci[d] = R.dci[d];
        G.thi[d] = R.thi[d];
        G.tlo[d] = R.tlo[d];
        G.kq[d] = R.kq[d];
#pragma unroll
        for (int k = 0; k < 5; ++k) G.b[d][k] = R.b[5 * d + k];
    }
    G.dx = R.dx;
    G.g = R.g;
    G.R2 = R.R2;
    G.Rt = sqrtf(R.R2);
    G.smin = R.smin;
    G.A = R.A;
    G.ph0 = R.ph0;
    G.om = R.om;
    G.q = R.q;
    G.Gamma = R.Gamma;
    G.Linv = R.Linv;
    G.eta = R.eta;
}

// The three acceptance tests of tube.f90:806-818 for the grid point at offset d = x - ci0 in
// the record's local frame: t0 >= 0, t1 < 0 and rho^2 < Rtube^2.  The arithmetic is spelled
// out with explicit fmaf so that every caller (the row filter and the evaluation of the tile
// kernel) decides a point identically.  t0 is returned for the spline argument.
template <typename RecT>
__device__ __forceinline__ bool rec_tests(const RecT &R, float d0x, float d0y, float d0z, float &t0)
{
    t0 = fmaf(d0z, R.tc0[2], fmaf(d0y, R.tc0[1], d0x * R.tc0[0]));
    if (!(t0 >= 0.0f)) return false;
    const float ex = d0x - R.dci[0], ey = d0y - R.dci[1], ez = d0z - R.dci[2];
    const float t1 = fmaf(ez, R.tc1[2], fmaf(ey, R.tc1[1], ex * R.tc1[0]));
    if (!(t1 < 0.0f)) return false;
    const float r2 = fmaf(-t0, t0, fmaf(d0z, d0z, fmaf(d0y, d0y, d0x * d0x)));
    return r2 < R.R2;
}

// The vorticity of tube.f90:819-892 for the spline argument W = zb + w, measured from the
// z0 of a record's Taylor coefficients R.b (c(z0 + W) - c(z0) = sum_k b[k-1] W^k), and the
// squared truncation radius R2 of the accepting chord.
//
// Delta = false: zb = 0 and d = x - c(z0) (up to the record's wrap bookkeeping), so
// x - c(z) = d - P(W) with P evaluated by Horner.
// Delta = true: d = x - c(z0 + zb), the offset from the accepting chord's start sample, and
// x - c(z) = d - (P(zb + w) - P(zb)), the difference taken in the divided-difference form
// w sum_k b_k D_k, D_k = ((zb + w)^k - zb^k) / w, which keeps its relative accuracy however
// large zb is.  The wrap decisions still use P(W), which needs no such accuracy: a decision
// moved by rounding is undone by the final single wrap.
template <bool General, bool Delta, typename RecT>
__device__ __forceinline__ void vort_w(const RecT &R, float d0x, float d0y, float d0z, float zb, float w, float R2,
                                       float out[3])
{
    const float W = Delta ? zb + w : w;
    float P[3], c1[3], Q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float *b = R.b + 5 * d;
        P[d] = W * fmaf(W, fmaf(W, fmaf(W, fmaf(W, b[4], b[3]), b[2]), b[1]), b[0]);
        c1[d] = fmaf(W, fmaf(W, fmaf(W, fmaf(W, 5.0f * b[4], 4.0f * b[3]), 3.0f * b[2]), 2.0f * b[1]), b[0]);
    }
    if constexpr (Delta) {
        const float u = zb, v = W;
        const float u2 = u * u, u3 = u2 * u, u4 = u3 * u;
        const float D2 = v + u, D3 = fmaf(v, D2, u2), D4 = fmaf(v, D3, u3), D5 = fmaf(v, D4, u4);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float *b = R.b + 5 * d;
            Q[d] = w * fmaf(b[4], D5, fmaf(b[3], D4, fmaf(b[2], D3, fmaf(b[1], D2, b[0]))));
        }
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) Q[d] = P[d];
    }
    const float d0[3] = {d0x, d0y, d0z};
    float xc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) xc[d] = d0[d] - Q[d];
    if (R.kq[0] != kNoWrap) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int n = R.kq[d] + (P[d] >= R.thi[d] ? 1 : 0) - (P[d] < R.tlo[d] ? 1 : 0);
            const float v = n ? fmaf(6.28318530717958647692f, (float)n, xc[d]) : xc[d];
            if (v > 3.14159265358979f) n -= 1;
            else if (v < -3.14159265358979f) n += 1;
            if (n) xc[d] = fmaf(6.28318530717958647692f, (float)n, xc[d]);
        }
    }
    const float rho2 = xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2];
    const float in1 = rsqrtf(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    const float T[3] = {c1[0] * in1, c1[1] * in1, c1[2] * in1};
    if constexpr (!General) {
        const float tp = (expf(-rho2 * R.inv2s2) - R.ftd) * R.amp;
        out[0] = tp * T[0];
        out[1] = tp * T[1];
        out[2] = tp * T[2];
    } else {
        float c2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float *b = R.b + 5 * d;
            c2[d] = fmaf(W, fmaf(W, fmaf(W, 20.0f * b[4], 12.0f * b[3]), 6.0f * b[2]), 2.0f * b[1]);
        }
        const float ph = fmaf(R.om, W, R.ph0);
        float sn, cs;
        sincosf(ph, &sn, &cs);
        const float sigma = fmaf(R.A, sn + 1.0f, R.smin);
        const float s2 = sigma * sigma;
        const float inv2s2 = 0.5f / s2;
        const float tp = (expf(-rho2 * inv2s2) - expf(-R2 * inv2s2)) * (0.159154943f / s2) * R.Gamma;
        const float dsds = R.q * cs * in1 * R.Linv;
        const float rho = sqrtf(rho2);
        const float X[3] = {c1[1] * c2[2] - c1[2] * c2[1], c1[2] * c2[0] - c1[0] * c2[2], c1[0] * c2[1] - c1[1] * c2[0]};
        const float nX = sqrtf(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
        const float inr = 1.0f / (rho + 1.0e-15f);
        if (nX < 1.0e-8f) {
            const float er[3] = {xc[0] * inr, xc[1] * inr, xc[2] * inr};
            const float eth[3] = {er[1] * T[2] - er[2] * T[1], er[2] * T[0] - er[0] * T[2], er[0] * T[1] - er[1] * T[0]};
            const float a = R.eta * rho, bq = rho * dsds / sigma;
#pragma unroll
            for (int d = 0; d < 3; ++d) out[d] = tp * (T[d] + a * eth[d] + bq * er[d]);
        } else {
            const float inX = 1.0f / nX;
            const float B[3] = {X[0] * inX, X[1] * inX, X[2] * inX};
            const float Nv[3] = {B[1] * T[2] - B[2] * T[1], B[2] * T[0] - B[0] * T[2], B[0] * T[1] - B[1] * T[0]};
            const float kap = nX * in1 * in1 * in1;
            const float costh = (xc[0] * Nv[0] + xc[1] * Nv[1] + xc[2] * Nv[2]) * inr;
            const float sinth = (xc[0] * B[0] + xc[1] * B[1] + xc[2] * B[2]) * inr;
            const float iden = 1.0f / (1.0f - kap * rho * costh);
            const float t5 = -sinth * rho * iden, t6 = costh * rho * iden;
            const float t7 = costh * rho * dsds / sigma * iden, t8 = sinth * rho * dsds / sigma * iden;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                out[d] = tp * (T[d] + R.eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
        }
    }
}

// The vorticity of tube.f90:819-892 for a point that passed rec_tests with argument t0
// (sub-segment record: W = t0 g).
template <bool General, typename RecT>
__device__ __forceinline__ void rec_vorticity(const RecT &R, float d0x, float d0y, float d0z, float t0, float out[3])
{
    vort_w<General, false>(R, d0x, d0y, d0z, 0.0f, t0 * R.g, R.R2, out);
}

// Predicate and vorticity together (tube.f90:806-892 in the local frame).
template <bool General, typename RecT>
__device__ __forceinline__ bool point_rec(const RecT &R, float d0x, float d0y, float d0z, float out[3])
{
    float t0;
    if (!rec_tests(R, d0x, d0y, d0z, t0)) return false;
    rec_vorticity<General>(R, d0x, d0y, d0z, t0, out);
    return true;
}

int launch_walk(Ctx *c, const CenterlineBatch &B, unsigned long long *d_acc);
int launch_tile(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out);
int launch_piece(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out);

// Lines whose truncation radius Rtube_ratio * sigma_max is at most this many grid spacings go
// through the piece kernel; thicker tubes through the sub-segment kernel, whose analytic
// row intervals skip most of a large box.
constexpr double kPieceMaxRtCells = 8.0;

}  // namespace fwt
