// k_deposit.cuh -- per-point Burgers-tube arithmetic shared by the deposition kernels.
#pragma once

#include "k_centerline.cuh"

namespace fwt {

// ---------------------------------------------------------------------------- FP64 reference
// The reference's inner body (tube.f90:806-892) split in two: the acceptance tests
// (tube.f90:806-818) and the vorticity of an accepted point (tube.f90:819-892), statement for
// statement in FP64.  m: mesh coordinates of the 1-based unwrapped grid index.
__device__ __forceinline__ void ref_mesh_f64(double dx, int ip, int jp, int kp, double m[3])
{
    const double xstart = -dev_pi();
    m[0] = dadd(dmul((double)ip - 1.0, dx), xstart);
    m[1] = dadd(dmul((double)jp - 1.0, dx), xstart);
    m[2] = dadd(dmul((double)kp - 1.0, dx), xstart);
}

// t0 = (x - ci0) . tci0 and t1' = (x - ci1) . tci0 (the projections ζ is interpolated from);
// returns whether the point passes the three tests.
__device__ __forceinline__ bool ref_tests_f64(const SubSeg &S, const double m[3], double &t0, double &t1p)
{
    const double a0 = dsub(m[0], S.ci0[0]), a1 = dsub(m[1], S.ci0[1]), a2 = dsub(m[2], S.ci0[2]);
    t0 = dadd(dadd(dmul(a0, S.tci0[0]), dmul(a1, S.tci0[1])), dmul(a2, S.tci0[2]));
    const double e0 = dsub(m[0], S.ci1[0]), e1 = dsub(m[1], S.ci1[1]), e2 = dsub(m[2], S.ci1[2]);
    const double t1 = dadd(dadd(dmul(e0, S.tci1[0]), dmul(e1, S.tci1[1])), dmul(e2, S.tci1[2]));
    t1p = dadd(dadd(dmul(e0, S.tci0[0]), dmul(e1, S.tci0[1])), dmul(e2, S.tci0[2]));
    if (!(t0 >= 0.0) || !(t1 < 0.0)) return false;
    const double rho = sqrt(dsub(dadd(dadd(dmul(a0, a0), dmul(a1, a1)), dmul(a2, a2)), dmul(t0, t0)));
    return rho < S.Rt;
}

__device__ __forceinline__ void ref_value_f64(const SubSeg &S, const LineParam &P, const double *coe, double dtf,
                                              double dzeta_sup, double eta, const double m[3], double t0,
                                              double t1, double out[3])
{
    const double zeta = (S.s1 * t0 - S.s0 * t1) / S.ndci0;
    const double zsec = zeta - S.ssec;
    const double L = P.Len;
    double cz[3], dc[3], ddc[3];
    spl_pos(coe, zsec * L, cz);
    const double dzeta = fmin(dzeta_sup, 1.0 * dtf);
    spl_d1(coe, zsec * L, dc);
    const double ndc = sqrt(dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2]);
    double T[3] = {dc[0] / ndc, dc[1] / ndc, dc[2] / ndc};
    spl_d2(coe, zsec * L, ddc);
    double X[3] = {dc[1] * ddc[2] - dc[2] * ddc[1], dc[2] * ddc[0] - dc[0] * ddc[2], dc[0] * ddc[1] - dc[1] * ddc[0]};
    const double nX = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
    double xc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        double v = m[d] - cz[d];
        if (v > dev_pi()) v = v - dev_pi2();
        if (v < -dev_pi()) v = v + dev_pi2();
        xc[d] = v;
    }
    const double nxc = sqrt(xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2]);
    const double rho = nxc;
    const double sigma = sigma_func(zeta, P.length, P.sigma_max, P.sigma_min, P.n_T);
    const double s2 = sigma * sigma;
    double tp = exp(-(rho * rho) / 2.0 / s2) / (dev_pi2() * s2);
    const double ftd = -exp(-(S.Rt * S.Rt) / 2.0 / s2) / (dev_pi2() * s2);
    tp = tp + ftd;
    const double sl = sigma_func(zeta - dzeta, P.length, P.sigma_max, P.sigma_min, P.n_T);
    const double sr = sigma_func(zeta + dzeta, P.length, P.sigma_max, P.sigma_min, P.n_T);
    double dsds = (sr - sl) / (2.0 * dzeta);
    dsds = dsds / ndc / L;
    const double G = P.Gamma;
    if (nX < 1.0e-8) {
        double er[3], eth[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) er[d] = xc[d] / (nxc + 1.0e-15);
        eth[0] = er[1] * T[2] - er[2] * T[1];
        eth[1] = er[2] * T[0] - er[0] * T[2];
        eth[2] = er[0] * T[1] - er[1] * T[0];
#pragma unroll
        for (int d = 0; d < 3; ++d) out[d] = tp * G * (T[d] + eta * rho * eth[d] + (rho * dsds / sigma) * er[d]);
    } else {
        double B[3], Nv[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) B[d] = X[d] / nX;
        Nv[0] = B[1] * T[2] - B[2] * T[1];
        Nv[1] = B[2] * T[0] - B[0] * T[2];
        Nv[2] = B[0] * T[1] - B[1] * T[0];
        const double kap = nX / (ndc * ndc * ndc);
        const double costh = (xc[0] * Nv[0] + xc[1] * Nv[1] + xc[2] * Nv[2]) / (nxc + 1.0e-15);
        const double sinth = (xc[0] * B[0] + xc[1] * B[1] + xc[2] * B[2]) / (nxc + 1.0e-15);
        const double den = 1.0 - kap * rho * costh;
        const double t5 = -(sinth * rho) / den;
        const double t6 = costh * rho / den;
        const double t7 = costh * rho * dsds / sigma / den;
        const double t8 = sinth * rho * dsds / sigma / den;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            out[d] = tp * G * (T[d] + eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
    }
}

// The reference's body at grid index (ip, jp, kp) (1-based, unwrapped): true and the
// contribution if accepted.
__device__ __forceinline__ bool point_ref_f64(const SubSeg &S, const LineParam &P, const double *coe, double dtf,
                                              double dzeta_sup, double eta, double dx, int ip, int jp, int kp,
                                              double out[3])
{
    double m[3], t0, t1;
    ref_mesh_f64(dx, ip, jp, kp, m);
    if (!ref_tests_f64(S, m, t0, t1)) return false;
    ref_value_f64(S, P, coe, dtf, dzeta_sup, eta, m, t0, t1, out);
    return true;
}

// FP64 data of a batch that the tile kernels read to redo a (point, sub-segment) pair in the
// reference's arithmetic: the section's spline coefficients and sample spacing, the line's
// constants, and the map from a record to its section.  A record is a sub-segment
// (pieces = false: rec -> slot = map[rec], chord j = rec - first[slot]) or a chord piece
// (pieces = true: rec -> slot = map[rec], chords j0.. of piece rec - first[slot]).
struct RedoCtx {
    const LineParam *lp;
    const int *slot_line, *map, *ntf;
    const int64_t *first;
    const int64_t *qoff;       // section slot -> its first sub-segment
    const SubSeg *seg;         // FP64 sub-segment records (the FP64 tile path), or null
    unsigned long long *tally; // [0] accepted pairs evaluated, [1] pairs redone in FP64
    const double *X, *Y, *Z, *cze, *coe, *dtf;
    int64_t node_base;
    int N, pieces;
    int zs, nz;                // planes of the context's field: zs .. zs + nz - 1
    double Rtube_ratio, dzeta_sup, eta, scale;
};

// Sub-segment j of section `slot` in FP64, built as the record builders build it
// (tube.f90:703-798): samples j, j+1, j+2 of the section's extended sample list, chords, the
// mark1 unwrap, Rtube and the box.
__device__ __forceinline__ void redo_subseg(const RedoCtx &R, int slot, int j, SubSeg &S, LineParam &P)
{
    P = R.lp[R.slot_line[slot]];
    const int t = slot - (int)P.slot_off;
    const int np = P.n_sec;
    const int n = R.ntf[slot];
    const double L = P.Len;
    const double *czl = R.cze + (P.node_off - R.node_base);
    const double zl = cze_pl_at(czl, np, t), zl1 = cze_pl_at(czl, np, t + 1);
    const double d = R.dtf[slot];
    const double *cf = R.coe + 18 * (size_t)slot;
    const int inext = (t + 1 < np) ? t + 1 : 0;
    double c[3][3];
#pragma unroll 1
    for (int s = 0; s < 3; ++s) {
        const int k = j + s;
        if (k < n) {
            spl_pos_fma(cf, (zl + d * k - zl) * L, c[s]);
        } else if (k == n) {
            c[s][0] = R.X[P.node_off + inext];
            c[s][1] = R.Y[P.node_off + inext];
            c[s][2] = R.Z[P.node_off + inext];
        } else {
            spl_pos_fma(R.coe + 18 * (size_t)(slot + 1), (zl1 + R.dtf[slot + 1] * 1 - zl1) * L, c[s]);
        }
    }
    double ch0[3], ch1[3];
    cminus3(c[1], c[0], ch0);
    cminus3(c[2], c[1], ch1);
    const double n0 = sqrt(ch0[0] * ch0[0] + ch0[1] * ch0[1] + ch0[2] * ch0[2]);
    const double n1 = sqrt(ch1[0] * ch1[0] + ch1[1] * ch1[1] + ch1[2] * ch1[2]);
    const double i0 = 1.0 / n0, i1 = 1.0 / n1;
    const double s0 = zl + d * j, s1 = zl + d * (j + 1);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double a = c[0][k], b = c[1][k];
        if (b - a > dev_pi()) a = a + dev_pi2();
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
        Rt = R.Rtube_ratio * P.sigma_min;
    } else {
        Rt = R.Rtube_ratio * sigma_func(s0, P.length, P.sigma_max, P.sigma_min, P.n_T);
        Rt = fmax(Rt, R.Rtube_ratio * sigma_func(s1, P.length, P.sigma_max, P.sigma_min, P.n_T));
    }
    S.Rt = Rt;
    S.slot = slot;
    S.line = 0;
    const double inv_dx = (double)R.N / dev_pi2(), xstart = -dev_pi();
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double mn = fmin(S.ci0[k], S.ci1[k]), mx = fmax(S.ci0[k], S.ci1[k]);
        S.box_lo[k] = (int)floor((mn - xstart - Rt) * inv_dx + 1.0);
        S.box_hi[k] = (int)ceil((mx - xstart + Rt) * inv_dx + 1.0);
    }
}

// Chord j of record `rec` (a sub-segment, or chord `ch` of a piece) and its section.
__device__ __forceinline__ void redo_locate(const RedoCtx &R, uint32_t rec, int ch, int &slot, int &j)
{
    slot = R.map[rec];
    const int i = (int)((int64_t)rec - R.first[slot]);
    if (!R.pieces) {
        j = i;
        return;
    }
    // pieces split a section's ntf chords as evenly as possible (piece_build_kernel)
    const int ns = R.ntf[slot];
    const int npc = (ns + 7) / 8;
    const int base = ns / npc, rem = ns % npc;
    j = i * base + min(i, rem) + ch;
}

// The reference's FP64 vorticity of the pair (grid point g = wrapped 0-based indices,
// record rec, chord ch), as a fixed-point contribution; the grid point's image inside the
// sub-segment's box (narrower than one period) is the one the reference visits.  decide =
// false: the FP32 tests accepted the pair.  decide = true: an FP32 plane test fell within its
// rounding bound of zero, and the reference's FP64 tests (tube.f90:806-818) decide; a rejected
// pair contributes nothing.  Returns 1 (accepted), 0 (rejected) or -1 (fixed-point overflow).
__device__ __forceinline__ int redo_pair_f64(const RedoCtx &R, uint32_t rec, int ch, bool decide, int gx, int gy,
                                                 int gz, long long q[3])
{
    q[0] = q[1] = q[2] = 0;
    int slot, j;
    redo_locate(R, rec, ch, slot, j);
    SubSeg S;
    LineParam P;
    redo_subseg(R, slot, j, S, P);
    const int g[3] = {gx, gy, gz};
    int ix[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int o = (g[k] + 1 - S.box_lo[k]) % R.N;
        if (o < 0) o += R.N;
        ix[k] = S.box_lo[k] + o;
    }
    double m[3], t0, t1, v[3];
    ref_mesh_f64(dev_pi2() / R.N, ix[0], ix[1], ix[2], m);
    const bool pass = ref_tests_f64(S, m, t0, t1);
    if (decide && !pass) return 0;
    ref_value_f64(S, P, R.coe + 18 * (size_t)slot, R.dtf[slot], R.dzeta_sup, R.eta, m, t0, t1, v);
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double sv = v[k] * R.scale;
        const bool in = fabs(sv) < 4.0e18;
        q[k] = in ? __double2ll_rn(sv) : 0;
        ok = ok && in;
    }
    return ok ? 1 : -1;
}

// Bound of the FP32 rounding of a plane test (x - p) . n evaluated from a record's local
// offsets d = off + i dx (i along the box, box extents ext grid points) with the offset dci
// between the record's two plane points: every rounding (off, dx, d, n, the three products and
// sums) is at most 2^-24 of a term bounded by E = sum_k max|d_k| + |dci_k|, about ten of them;
// 2e-6 E keeps a factor of three.  Beyond it the FP32 sign is the FP64 sign.
__device__ __forceinline__ float plane_eps(const float off[3], const int ext[3], float dx, const float dci[3])
{
    float E = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        E += fmaxf(fabsf(off[k]), fabsf(fmaf((float)ext[k], dx, off[k]))) + fabsf(dci[k]);
    return 2.0e-6f * E + 1.0e-30f;
}

// Curved-branch amplification |1/(1 - kappa rho cos theta)| (tube.f90:876-879) above which an
// FP32 evaluation cannot hold 1e-5: such pairs are evaluated in FP64 (redo_pair_f64).
constexpr float kRedoCond = 4.0f;

// FP32 view of one sub-segment, local to its start point ci0 and to a grid-index origin.
struct SegF {
    float off[3];     // mesh point at the origin index minus ci0
    float dx;
    float tc0[3], tc1[3], dci[3];
    float g;          // W = t0 * g is the spline argument measured from the start, times Len
    float b[3][5];    // c(z0 + W) - c(z0) = sum_k b[k-1] W^k
    float R2, Rt;
    float pe;         // rounding bound of the plane tests (plane_eps)
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
    const int ext[3] = {S.box_hi[0] - i0, S.box_hi[1] - j0, S.box_hi[2] - k0};
    G.pe = plane_eps(G.off, ext, G.dx, G.dci);
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
// reduces to tp * Gamma * T.  Returns 0 (rejected), 1 (accepted, out holds the contribution)
// or 2: a plane test within its rounding bound G.pe of zero, left to the FP64 tests.
template <bool General>
__device__ __forceinline__ int point_f32(const SegF &G, int ii, int jj, int kk, float out[3], float &cond)
{
    cond = 1.0f;
    const float d0x = fmaf((float)ii, G.dx, G.off[0]);
    const float d0y = fmaf((float)jj, G.dx, G.off[1]);
    const float d0z = fmaf((float)kk, G.dx, G.off[2]);
    const float t0 = d0x * G.tc0[0] + d0y * G.tc0[1] + d0z * G.tc0[2];
    if (!(t0 >= -G.pe)) return 0;
    const float ex = d0x - G.dci[0], ey = d0y - G.dci[1], ez = d0z - G.dci[2];
    const float t1 = ex * G.tc1[0] + ey * G.tc1[1] + ez * G.tc1[2];
    if (!(t1 < G.pe)) return 0;
    const float r2 = d0x * d0x + d0y * d0y + d0z * d0z - t0 * t0;
    if (!(r2 < G.R2)) return 0;
    if (!(t0 >= G.pe) || !(t1 < -G.pe)) return 2;
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
        return 1;
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
            cond = fabsf(iden);
            const float t5 = -sinth * rho * iden, t6 = costh * rho * iden;
            const float t7 = costh * rho * dsds / sigma * iden, t8 = sinth * rho * dsds / sigma * iden;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                out[d] = tp * (T[d] + G.eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
        }
        return 1;
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
    R.ftd = __expf(-G.R2 * R.inv2s2);   // the same exponential as the per-point term
    R.amp = G.Gamma * (0.159154943091895336f / s2);
    // No-wrap flag (kq[0] = kNoWrap): for every point that passes the tests, |W| <= Wm, so
    // |P| stays clear of both wrap thresholds and |x - c| < pi; the wrap bookkeeping of
    // point_rec then reduces to x - c = d0 - P.  An accepted point has 0 <= t0 <= dl + Rt
    // (bends below 45 degrees, checked below) and a distance below Rt from the chord line, so
    // |d0| <= sqrt((dl + Rt)^2 + Rt^2) and |x - c| <= |d0| + |P|.
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
    if (sqrtf((dl + G.Rt) * (dl + G.Rt) + G.R2) + pmax > 3.0f) nowrap = false;
    // t0 <= dl + Rt tan(bend) <= dl + Rt holds for bends below 45 degrees
    if (G.tc0[0] * G.tc1[0] + G.tc0[1] * G.tc1[1] + G.tc0[2] * G.tc1[2] < 0.75f) nowrap = false;
    if (nowrap) R.kq[0] = kNoWrap;
}

// The three acceptance tests of tube.f90:806-818 for the grid point at offset d = x - ci0 in
// the record's local frame (t0 >= 0, t1 < 0 and rho^2 < Rtube^2), with the planes' rounding
// bound pe (plane_eps): 0 rejected, 1 accepted, 2 a plane test within pe of zero.  The
// arithmetic is spelled out with explicit fmaf, and t0 is recomputed the same way for the
// spline argument of an accepted pair.  The reference's field jumps across the plane shared
// by two consecutive chords (zeta is interpolated along each chord separately), so a pair of
// the third kind is decided by the reference's FP64 tests; beyond pe the FP32 signs are the
// FP64 signs.
template <typename RecT>
__device__ __forceinline__ int rec_classify(const RecT &R, float d0x, float d0y, float d0z, float pe)
{
    const float t0 = fmaf(d0z, R.tc0[2], fmaf(d0y, R.tc0[1], d0x * R.tc0[0]));
    if (!(t0 >= -pe)) return 0;
    const float ex = d0x - R.dci[0], ey = d0y - R.dci[1], ez = d0z - R.dci[2];
    const float t1 = fmaf(ez, R.tc1[2], fmaf(ey, R.tc1[1], ex * R.tc1[0]));
    if (!(t1 < pe)) return 0;
    const float r2 = fmaf(-t0, t0, fmaf(d0z, d0z, fmaf(d0y, d0y, d0x * d0x)));
    if (!(r2 < R.R2)) return 0;
    return (t0 >= pe && t1 < -pe) ? 1 : 2;
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
                                       float out[3], float &cond)
{
    cond = 1.0f;
    const float W = Delta ? zb + w : w;
    float P[3], c1[3], Q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        // P(W) by Horner's scheme, and P'(W) from its partial sums h_k by the derivative
        // recurrence h0 + W (h1 + W (h2 + W (h3 + W b4))) = b0 + 2 b1 W + ... + 5 b4 W^4
        const float *b = R.b + 5 * d;
        const float h3 = fmaf(W, b[4], b[3]);
        const float h2 = fmaf(W, h3, b[2]);
        const float h1 = fmaf(W, h2, b[1]);
        const float h0 = fmaf(W, h1, b[0]);
        P[d] = W * h0;
        c1[d] = fmaf(W, fmaf(W, fmaf(W, fmaf(W, b[4], h3), h2), h1), h0);
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
        const float tp = (__expf(-rho2 * R.inv2s2) - R.ftd) * R.amp;
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
        const float tp = (__expf(-rho2 * inv2s2) - __expf(-R2 * inv2s2)) * (0.159154943f / s2) * R.Gamma;
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
            cond = fabsf(iden);
            const float t5 = -sinth * rho * iden, t6 = costh * rho * iden;
            const float t7 = costh * rho * dsds / sigma * iden, t8 = sinth * rho * dsds / sigma * iden;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                out[d] = tp * (T[d] + R.eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
        }
    }
}

// The vorticity of tube.f90:819-892 for a point that passed rec_classify with argument t0
// (sub-segment record: W = t0 g), and its curved-branch amplification.
template <bool General, typename RecT>
__device__ __forceinline__ void rec_vorticity(const RecT &R, float d0x, float d0y, float d0z, float t0, float out[3],
                                              float &cond)
{
    vort_w<General, false>(R, d0x, d0y, d0z, 0.0f, t0 * R.g, R.R2, out, cond);
}

int launch_walk(Ctx *c, const CenterlineBatch &B, unsigned long long *d_acc);
int launch_tile(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out);
int launch_piece(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out);
int launch_scatter(Ctx *c, const CenterlineBatch &B);

// Lines whose truncation radius Rtube_ratio * sigma_max is at most this many grid spacings go
// through the piece kernel; thicker tubes through the sub-segment kernel, whose analytic
// row intervals skip most of a large box.
constexpr double kPieceMaxRtCells = 8.0;
// Piece lines whose truncation radius is at most this many grid spacings can have their pieces
// rasterised once (piece_raster) instead of searched in every tile.  Off by default: on the
// 1024^3 workload the raster pass plus the per-tile filtering of its point lists took 1.3x
// (radius 1.9 grid spacings) and 2.4x (3.8) the time of the per-tile search; it stays available
// through fwt_set_tuning.
constexpr double kRasterMaxRtCells = 0.0;
// Piece lines whose truncation radius is at most this many grid spacings are deposited without
// tiles (scatter_piece_kernel, FP32 only): each piece is searched once and its contributions
// added with int64 global reductions, instead of once in every tile its box meets.  On the
// 1024^3 workload the scatter path took 0.34x (radius 1.9 grid spacings) and 0.75x (3.8) of the
// tile path's deposition time, and 1.5x at 7.6, where a chord accepts hundreds of points.
constexpr double kScatterMaxRtCells = 5.0;

}  // namespace fwt
