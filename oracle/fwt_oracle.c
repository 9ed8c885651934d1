/*
 * fwt_oracle.c -- FP64 CPU ORACLE (test infrastructure only).
 *
 * This file is the checker for the CUDA path, never the product: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference leg load it.
 *
 * It restates, statement by statement and in double precision, the vortex-tube
 * construction loop of the reference program `Weav_ver5_8_2`:
 *   - centerline preprocessing (periodic arc-length cze, Len_Disc, c', c'')   tube.f90:392-515
 *   - quintic Hermite spline coefficients                                   subroutine.f90:440-488
 *   - spline evaluation c, c', c''                                          subroutine.f90:490-560
 *   - adaptive sub-segmentation (turning-angle presampling, ntf)            tube.f90:616-751
 *   - core-size law sigma(zeta) and d sigma / d zeta                        subroutine.f90:164-173, 748-761
 *   - the deposition box walk and Burgers-tube vorticity                    tube.f90:762-904
 *
 * Parity status: UNPINNED against the reference binary.  The reference is Fortran +
 * MPI + FFTW and there is no Fortran compiler in this image, and the reference ships
 * no golden outputs.  The restatement is pinned instead by analytic known-answer
 * tests (straight periodic tube, spline node reproduction, Etot/up^2 = 3/2 ...).
 *
 * Deliberate, documented deviations from the literal Fortran:
 *   - `dsigmadzeta` (subroutine.f90:755-756) calls sigma_func with 5 of its 6
 *     arguments, so n_T is undefined there; this oracle passes the line's n_T.
 *   - real powers `x**k.0d0` are evaluated as repeated products.
 *   - the MPI z-slab split is replaced by an OpenMP split over z-slabs with the
 *     same ownership rule (each grid point owned by one thread), so every grid point
 *     receives its contributions in the serial reference order (line, section,
 *     sub-segment).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.141592653589793115997963468544185161590576171875 /* 4*datan(1d0) */
#define ORC_PI2 6.28318530717958623199592693708837032318115234375 /* 8*datan(1d0) */

/* ---------------------------------------------------------------- a2: line preprocessing */

/* tube.f90:417-501.  cze: normalised periodic arc-length parameter in [0,2pi);
 * ck/ckk: first/second derivative by periodic central differences (3*np, coordinate-major). */
void orc_line_prep(int np, const double *cx, const double *cy, const double *cz,
                   double *cze, double *ck, double *ckk, double *len_disc)
{
    const double *c[3] = {cx, cy, cz};
    double cd[3], dist;
    cze[0] = 0.0;
    for (int i = 1; i < np; ++i) {
        for (int d = 0; d < 3; ++d) {
            cd[d] = fabs(c[d][i] - c[d][i - 1]);
            if (cd[d] > ORC_PI) cd[d] = cd[d] - ORC_PI2;
        }
        dist = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
        cze[i] = cze[i - 1] + dist;
    }
    for (int d = 0; d < 3; ++d) {
        cd[d] = fabs(c[d][0] - c[d][np - 1]);
        if (cd[d] > ORC_PI) cd[d] = cd[d] - ORC_PI2;
    }
    dist = sqrt(cd[0] * cd[0] + cd[1] * cd[1] + cd[2] * cd[2]);
    const double total = cze[np - 1] + dist;
    const double L = total / ORC_PI2;
    *len_disc = L;
    for (int i = 0; i < np; ++i) cze[i] = cze[i] * ORC_PI2 / total;

    /* first derivative (tube.f90:440-466) */
    for (int i = 0; i < np; ++i) {
        int ip, im;
        double dz;
        if (i == 0) { ip = 1; im = np - 1; dz = cze[1] - cze[np - 1] + ORC_PI2; }
        else if (i == np - 1) { ip = 0; im = np - 2; dz = cze[0] - cze[np - 2] + ORC_PI2; }
        else { ip = i + 1; im = i - 1; dz = cze[i + 1] - cze[i - 1]; }
        for (int d = 0; d < 3; ++d) {
            double v = c[d][ip] - c[d][im];
            if (v > ORC_PI) v = v - ORC_PI2;
            if (v < -ORC_PI) v = v + ORC_PI2;
            ck[d * np + i] = v / (dz * L);
        }
    }
    /* second derivative (tube.f90:469-489): differences of ck, no wrap */
    for (int i = 0; i < np; ++i) {
        int ip, im;
        double dz;
        if (i == 0) { ip = 1; im = np - 1; dz = cze[1] - cze[np - 1] + ORC_PI2; }
        else if (i == np - 1) { ip = 0; im = np - 2; dz = cze[0] - cze[np - 2] + ORC_PI2; }
        else { ip = i + 1; im = i - 1; dz = cze[i + 1] - cze[i - 1]; }
        for (int d = 0; d < 3; ++d)
            ckk[d * np + i] = (ck[d * np + ip] - ck[d * np + im]) / (dz * L);
    }
}

/* ---------------------------------------------------------------- a3/a4: quintic spline */

/* subroutine.f90:440-461 (get_spline_5th_coe) */
static void spline5_coe(double *coe, double zr, double xl, double xr, double vl, double vr,
                        double al, double ar)
{
    double xpl = xl, xpr = xr;
    if (xl - xr > ORC_PI) xpr = xr + ORC_PI2;
    else if (xl - xr < -ORC_PI) xpl = xl + ORC_PI2;
    const double z2 = zr * zr, z3 = z2 * zr, z4 = z3 * zr, z5 = z4 * zr;
    coe[0] = xl;
    coe[1] = vl;
    coe[2] = al / 2.0;
    coe[3] = (20.0 * (xpr - xpl) - (12.0 * vl + 8.0 * vr) * zr - (3.0 * al - ar) * z2) / (2.0 * z3);
    coe[4] = (-30.0 * (xpr - xpl) + (16.0 * vl + 14.0 * vr) * zr + (3.0 * al - 2.0 * ar) * z2) / (2.0 * z4);
    coe[5] = (12.0 * (xpr - xpl) - 6.0 * (vl + vr) * zr - (al - ar) * z2) / (2.0 * z5);
}

/* coe layout: [section][coord][6] */
static void spline5_pos(const double *coe, double z, double *c3) /* subroutine.f90:490-518 */
{
    const double z2 = z * z, z3 = z2 * z, z4 = z3 * z, z5 = z4 * z;
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        c3[d] = a[5] * z5 + a[4] * z4 + a[3] * z3 + a[2] * z2 + a[1] * z + a[0];
    }
    for (int d = 0; d < 3; ++d) if (c3[d] >= ORC_PI) c3[d] = c3[d] - ORC_PI2;
    for (int d = 0; d < 3; ++d) if (c3[d] < -ORC_PI) c3[d] = c3[d] + ORC_PI2;
}

static void spline5_d1(const double *coe, double z, double *c3) /* subroutine.f90:520-539 */
{
    const double z2 = z * z, z3 = z2 * z, z4 = z3 * z;
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        c3[d] = 5.0 * a[5] * z4 + 4.0 * a[4] * z3 + 3.0 * a[3] * z2 + 2.0 * a[2] * z + a[1];
    }
}

static void spline5_d2(const double *coe, double z, double *c3) /* subroutine.f90:541-560 */
{
    const double z2 = z * z, z3 = z2 * z;
    for (int d = 0; d < 3; ++d) {
        const double *a = coe + 6 * d;
        c3[d] = 20.0 * a[5] * z3 + 12.0 * a[4] * z2 + 6.0 * a[3] * z + 2.0 * a[2];
    }
}

static inline void cross3(const double *a, const double *b, double *c) /* subroutine.f90:799-804 */
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static inline void cminus(const double *r, const double *l, double *d) /* subroutine.f90:695-712 */
{
    for (int k = 0; k < 3; ++k) {
        double v = r[k] - l[k];
        if (v > ORC_PI) v = v - ORC_PI2;
        if (v < -ORC_PI) v = v + ORC_PI2;
        d[k] = v;
    }
}

/* subroutine.f90:164-173 */
static inline double sigma_func(double zeta, double length, double smax, double smin, int n_T)
{
    const double omega = floor(length / ORC_PI + 0.5) * (double)n_T;
    return smin + (smax - smin) * (sin(omega * zeta) + 1.0) / 2.0;
}

/* ------------------------------------------------------------------ per-line set-up */

typedef struct {
    int n_sec, ntf_max;
    double L, length;
    double *cze_pl;   /* n_sec+2 */
    double *coe;      /* (n_sec+1)*18 */
    int *ntf;         /* n_sec+1 */
    double *dtf;      /* n_sec+1 */
    double *s2;       /* (n_sec+1)*(ntf_max+1) */
    double *ci;       /* (n_sec+1)*(ntf_max+1)*3 */
    double *ndci;     /* n_sec*(ntf_max+1) */
    double *tci;      /* n_sec*(ntf_max+1)*3 */
} orc_line;

static void line_free(orc_line *ln)
{
    free(ln->cze_pl); free(ln->coe); free(ln->ntf); free(ln->dtf);
    free(ln->s2); free(ln->ci); free(ln->ndci); free(ln->tci);
    memset(ln, 0, sizeof(*ln));
}

/* tube.f90:543-751 for one line.  Returns 0 on success. */
static int line_setup(int np, const double *cx, const double *cy, const double *cz,
                      int ntf_times, int ntf_pre, orc_line *ln)
{
    memset(ln, 0, sizeof(*ln));
    if (np < 2) return -1;
    double *cze = malloc(sizeof(double) * np);
    double *ck = malloc(sizeof(double) * 3 * np);
    double *ckk = malloc(sizeof(double) * 3 * np);
    double L;
    orc_line_prep(np, cx, cy, cz, cze, ck, ckk, &L);
    const int ns = np;
    ln->n_sec = ns;
    ln->L = L;
    ln->length = L * ORC_PI2;
    /* periodic extension (tube.f90:561-596) */
    const double *c[3] = {cx, cy, cz};
    double *x_pl = malloc(sizeof(double) * 3 * (ns + 2));
    double *v_pl = malloc(sizeof(double) * 3 * (ns + 2));
    double *a_pl = malloc(sizeof(double) * 3 * (ns + 2));
    ln->cze_pl = malloc(sizeof(double) * (ns + 2));
    for (int i = 0; i < ns + 2; ++i) {
        const int src = (i < ns) ? i : (i - ns);
        for (int d = 0; d < 3; ++d) {
            x_pl[d * (ns + 2) + i] = c[d][src];
            v_pl[d * (ns + 2) + i] = ck[d * np + src];
            a_pl[d * (ns + 2) + i] = ckk[d * np + src];
        }
        ln->cze_pl[i] = (i < ns) ? cze[i] : (i == ns ? ORC_PI2 : ORC_PI2 + cze[1]);
    }
    /* spline coefficients (tube.f90:598 -> subroutine.f90:463-488); argument is cze_pl*Len */
    ln->coe = malloc(sizeof(double) * 18 * (ns + 1));
    for (int i = 0; i < ns + 1; ++i) {
        const double zr = ln->cze_pl[i + 1] * L - ln->cze_pl[i] * L;
        for (int d = 0; d < 3; ++d) {
            const double *X = x_pl + d * (ns + 2), *V = v_pl + d * (ns + 2), *A = a_pl + d * (ns + 2);
            spline5_coe(ln->coe + 18 * i + 6 * d, zr, X[i], X[i + 1], V[i], V[i + 1], A[i], A[i + 1]);
        }
    }
    free(x_pl); free(v_pl); free(a_pl);
    free(cze); free(ck); free(ckk);

    /* turning-angle presampling, ntf (tube.f90:625-657) */
    ln->ntf = malloc(sizeof(int) * (ns + 1));
    ln->dtf = malloc(sizeof(double) * (ns + 1));
    int ntf_max = 0;
    for (int ti = 0; ti < ns + 1; ++ti) {
        const double *coe = ln->coe + 18 * ti;
        const double dtfp = (ln->cze_pl[ti + 1] - ln->cze_pl[ti]) / (1.0 * ntf_pre);
        double theta = 0.0;
        for (int tj = 0; tj <= ntf_pre; ++tj) {
            const double s = ln->cze_pl[ti] + dtfp * tj;
            const double z = (s - ln->cze_pl[ti]) * L;
            double dc[3], ddc[3], x[3];
            spline5_d1(coe, z, dc);
            const double ndc = norm3(dc);
            spline5_d2(coe, z, ddc);
            cross3(dc, ddc, x);
            const double nx = norm3(x);
            theta = theta + nx / (ndc * ndc) * dtfp * L;
        }
        ln->ntf[ti] = (int)ceil(ntf_times * theta / ORC_PI2) + 1;
        ln->dtf[ti] = (ln->cze_pl[ti + 1] - ln->cze_pl[ti]) / (1.0 * ln->ntf[ti]);
        if (ln->ntf[ti] > ntf_max) ntf_max = ln->ntf[ti];
    }
    ln->ntf_max = ntf_max;
    const int W = ntf_max + 1;
    ln->s2 = malloc(sizeof(double) * (ns + 1) * W);
    ln->ci = malloc(sizeof(double) * 3 * (ns + 1) * W);
    ln->ndci = malloc(sizeof(double) * ns * W);
    ln->tci = malloc(sizeof(double) * 3 * ns * W);
    /* sample points (tube.f90:706-713) */
    for (int ti = 0; ti < ns + 1; ++ti) {
        const double *coe = ln->coe + 18 * ti;
        for (int tj = 0; tj <= ln->ntf[ti]; ++tj) {
            const double s = ln->cze_pl[ti] + ln->dtf[ti] * tj;
            ln->s2[ti * W + tj] = s;
            spline5_pos(coe, (s - ln->cze_pl[ti]) * L, ln->ci + 3 * (ti * W + tj));
        }
    }
    /* endpoint copy (tube.f90:721-723) */
    for (int ti = 0; ti < ns; ++ti)
        memcpy(ln->ci + 3 * (ti * W + ln->ntf[ti]), ln->ci + 3 * ((ti + 1) * W), 3 * sizeof(double));
    /* chords (tube.f90:740-751) */
    for (int ti = 0; ti < ns; ++ti) {
        for (int tj = 0; tj <= ln->ntf[ti]; ++tj) {
            double *dci = ln->tci + 3 * (ti * W + tj);
            if (tj < ln->ntf[ti]) cminus(ln->ci + 3 * (ti * W + tj + 1), ln->ci + 3 * (ti * W + tj), dci);
            else cminus(ln->ci + 3 * ((ti + 1) * W + 1), ln->ci + 3 * ((ti + 1) * W), dci);
            const double n = norm3(dci);
            ln->ndci[ti * W + tj] = n;
            for (int d = 0; d < 3; ++d) dci[d] = dci[d] / n;
        }
    }
    return 0;
}

/* -------------------------------------------------------------- exported set-up probes */

/* Per-section ntf (n_sec+1 entries) and spline coefficients ((n_sec+1)*18, [sec][coord][6]). */
int orc_line_ntf(int np, const double *cx, const double *cy, const double *cz, int ntf_times,
                 int ntf_pre, int *ntf_out, double *dtf_out, double *coe_out, double *len_disc)
{
    orc_line ln;
    if (line_setup(np, cx, cy, cz, ntf_times, ntf_pre, &ln)) return -1;
    if (ntf_out) memcpy(ntf_out, ln.ntf, sizeof(int) * (np + 1));
    if (dtf_out) memcpy(dtf_out, ln.dtf, sizeof(double) * (np + 1));
    if (coe_out) memcpy(coe_out, ln.coe, sizeof(double) * 18 * (np + 1));
    if (len_disc) *len_disc = ln.L;
    line_free(&ln);
    return 0;
}

/* Flattened sub-segment table for one line (sections 0..np-1, sub-segments 0..ntf-1):
 * per sub-segment s0,s1, ci0[3], ci1[3] (before the mark1 unwrap), tci0[3], tci1[3], ndci0
 * -> 15 doubles.  Returns the number of sub-segments, or -1.  Pass out=NULL to count. */
long orc_line_subsegs(int np, const double *cx, const double *cy, const double *cz, int ntf_times,
                      int ntf_pre, double *out)
{
    orc_line ln;
    if (line_setup(np, cx, cy, cz, ntf_times, ntf_pre, &ln)) return -1;
    const int W = ln.ntf_max + 1;
    long n = 0;
    for (int ti = 0; ti < ln.n_sec; ++ti) {
        for (int tj = 0; tj < ln.ntf[ti]; ++tj, ++n) {
            if (!out) continue;
            double *o = out + 15 * n;
            o[0] = ln.s2[ti * W + tj];
            o[1] = ln.s2[ti * W + tj + 1];
            memcpy(o + 2, ln.ci + 3 * (ti * W + tj), 3 * sizeof(double));
            memcpy(o + 5, ln.ci + 3 * (ti * W + tj + 1), 3 * sizeof(double));
            memcpy(o + 8, ln.tci + 3 * (ti * W + tj), 3 * sizeof(double));
            memcpy(o + 11, ln.tci + 3 * (ti * W + tj + 1), 3 * sizeof(double));
            o[14] = ln.ndci[ti * W + tj];
        }
    }
    line_free(&ln);
    return n;
}

/* ------------------------------------------------------------------ a6: deposition */

typedef struct {
    int N;              /* nx = ny = nz */
    double sigma_ratio; /* sigma_max / sigma_min */
    double eta0;        /* eta_t */
    int ntf_times, ntf_pre;
    double Rtube_ratio, dzeta_sup;
} orc_grid;

/* Deposit one centerline into vor (3 arrays of N^3, x fastest = Fortran (i,j,k) order).
 * tube.f90:536-904.  Returns the number of sub-segments, or -1. stats[0]=sum(ntf),
 * stats[1]=ntf_max, stats[2]=accepted points. */
static long deposit_line(const orc_grid *g, int np, const double *cx, const double *cy, const double *cz,
                         double sigma_min, double Gamma, int n_T, double *vorx, double *vory, double *vorz,
                         int nthreads, double *stats, double *cond);

long orc_deposit_line(const orc_grid *g, int np, const double *cx, const double *cy, const double *cz,
                      double sigma_min, double Gamma, int n_T, double *vorx, double *vory,
                      double *vorz, int nthreads, double *stats)
{
    return deposit_line(g, np, cx, cy, cz, sigma_min, Gamma, n_T, vorx, vory, vorz, nthreads, stats, NULL);
}

/* Same, and cond[idx] = max(cond[idx], |1 / (1 - kappa rho cos theta)|) over the point's
 * contributions (1 on the straight branch): the amplification of the curved branch's
 * denominator (tube.f90:876-879).  Near the centre of curvature of a bend tighter than the
 * tube radius it grows without bound and the reference's own FP64 value is ill-conditioned. */
long orc_deposit_line_cond(const orc_grid *g, int np, const double *cx, const double *cy, const double *cz,
                           double sigma_min, double Gamma, int n_T, double *vorx, double *vory,
                           double *vorz, int nthreads, double *stats, double *cond)
{
    return deposit_line(g, np, cx, cy, cz, sigma_min, Gamma, n_T, vorx, vory, vorz, nthreads, stats, cond);
}

static long deposit_line(const orc_grid *g, int np, const double *cx, const double *cy, const double *cz,
                         double sigma_min, double Gamma, int n_T, double *vorx, double *vory, double *vorz,
                         int nthreads, double *stats, double *cond)
{
    orc_line ln;
    if (line_setup(np, cx, cy, cz, g->ntf_times, g->ntf_pre, &ln)) return -1;
    const int N = g->N;
    const double sigma_max = g->sigma_ratio * sigma_min;
    const double xstart = -ORC_PI, dx = ORC_PI2 / N;
    const int W = ln.ntf_max + 1;
    const double L = ln.L, length = ln.length;
    long nsub = 0, ntf_sum = 0;
    for (int ti = 0; ti < ln.n_sec; ++ti) nsub += ln.ntf[ti];
    for (int ti = 0; ti < ln.n_sec + 1; ++ti) ntf_sum += ln.ntf[ti];
    long accepted_total = 0;
    double *vor[3] = {vorx, vory, vorz};
    if (nthreads < 1) nthreads = 1;
    if (nthreads > N) nthreads = N;

#pragma omp parallel num_threads(nthreads) reduction(+ : accepted_total)
    {
        int tid = 0, nth = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nth = omp_get_num_threads();
#endif
        /* this thread owns z planes [kz0, kz1) (1-based k = kz0+1 .. kz1) */
        const int kz0 = (int)((long)N * tid / nth), kz1 = (int)((long)N * (tid + 1) / nth);
        for (int ti = 0; ti < ln.n_sec; ++ti) {
            const double *coe = ln.coe + 18 * ti;
            for (int tj = 0; tj < ln.ntf[ti]; ++tj) {
                const double s0 = ln.s2[ti * W + tj], s1 = ln.s2[ti * W + tj + 1];
                double ci0[3], ci1[3], tci0[3], tci1[3];
                memcpy(ci0, ln.ci + 3 * (ti * W + tj), sizeof ci0);
                memcpy(ci1, ln.ci + 3 * (ti * W + tj + 1), sizeof ci1);
                memcpy(tci0, ln.tci + 3 * (ti * W + tj), sizeof tci0);
                memcpy(tci1, ln.tci + 3 * (ti * W + tj + 1), sizeof tci1);
                const double ndci0 = ln.ndci[ti * W + tj];
                for (int d = 0; d < 3; ++d) { /* mark1, tube.f90:779-785 */
                    if (ci1[d] - ci0[d] > ORC_PI) ci0[d] = ci0[d] + ORC_PI2;
                    else if (ci1[d] - ci0[d] < -ORC_PI) ci1[d] = ci1[d] + ORC_PI2;
                }
                double Rt = g->Rtube_ratio * sigma_func(s0, length, sigma_max, sigma_min, n_T);
                const double r1 = g->Rtube_ratio * sigma_func(s1, length, sigma_max, sigma_min, n_T);
                if (r1 > Rt) Rt = r1;
                int lo[3], hi[3];
                for (int d = 0; d < 3; ++d) {
                    const double mn = ci0[d] < ci1[d] ? ci0[d] : ci1[d];
                    const double mx = ci0[d] > ci1[d] ? ci0[d] : ci1[d];
                    lo[d] = (int)floor((mn - xstart - Rt) / dx + 1);
                    hi[d] = (int)ceil((mx - xstart + Rt) / dx + 1);
                }
                for (int kp = lo[2]; kp <= hi[2]; ++kp) {
                    const int k = ((kp + N - 1) % N) + 1;
                    if (!(k > kz0 && k <= kz1)) continue;
                    if (k <= 0) continue;
                    const double mz = (kp - 1.0) * dx + xstart;
                    for (int jp = lo[1]; jp <= hi[1]; ++jp) {
                        const double my = (jp - 1.0) * dx + xstart;
                        for (int ip = lo[0]; ip <= hi[0]; ++ip) {
                            const double mxp = (ip - 1.0) * dx + xstart;
                            const double t0 = (mxp - ci0[0]) * tci0[0] + (my - ci0[1]) * tci0[1] + (mz - ci0[2]) * tci0[2];
                            if (!(t0 >= 0.0)) continue;
                            double t1 = (mxp - ci1[0]) * tci1[0] + (my - ci1[1]) * tci1[1] + (mz - ci1[2]) * tci1[2];
                            if (!(t1 < 0.0)) continue;
                            const double ax = mxp - ci0[0], ay = my - ci0[1], az = mz - ci0[2];
                            double rho = sqrt(ax * ax + ay * ay + az * az - t0 * t0);
                            if (!(rho < Rt)) continue;
                            t1 = (mxp - ci1[0]) * tci0[0] + (my - ci1[1]) * tci0[1] + (mz - ci1[2]) * tci0[2];
                            const double zeta = (s1 * t0 - s0 * t1) / ndci0;
                            const double zsec = zeta - ln.s2[ti * W];
                            double cz3[3], dc[3], ddc[3], dcddc[3], T[3], m[3], xc[3];
                            spline5_pos(coe, zsec * L, cz3);
                            const double dzeta = fmin(g->dzeta_sup, 1.0 * ln.dtf[ti]);
                            spline5_d1(coe, zsec * L, dc);
                            const double ndc = norm3(dc);
                            for (int d = 0; d < 3; ++d) T[d] = dc[d] / ndc;
                            spline5_d2(coe, zsec * L, ddc);
                            cross3(dc, ddc, dcddc);
                            const double ndcddc = norm3(dcddc);
                            m[0] = mxp; m[1] = my; m[2] = mz;
                            cminus(m, cz3, xc);
                            const double nxc = norm3(xc);
                            rho = nxc;
                            const double sigma = sigma_func(zeta, length, sigma_max, sigma_min, n_T);
                            const double s2 = sigma * sigma;
                            double tp = exp(-(rho * rho) / 2.0 / s2) / (ORC_PI2 * s2);
                            const double ftd = -exp(-(Rt * Rt) / 2.0 / s2) / (ORC_PI2 * s2);
                            tp = tp + ftd;
                            const double sl = sigma_func(zeta - dzeta, length, sigma_max, sigma_min, n_T);
                            const double sr = sigma_func(zeta + dzeta, length, sigma_max, sigma_min, n_T);
                            double dsds = (sr - sl) / (2.0 * dzeta);
                            dsds = dsds / ndc / L;
                            const double eta = g->eta0;
                            const int i = ((ip + N - 1) % N) + 1, j = ((jp + N - 1) % N) + 1;
                            const size_t idx = (size_t)(i - 1) + (size_t)N * ((size_t)(j - 1) + (size_t)N * (size_t)(k - 1));
                            if (ndcddc < 1.0e-8) { /* straight branch, tube.f90:854-866 */
                                double er[3], eth[3];
                                for (int d = 0; d < 3; ++d) er[d] = xc[d] / (nxc + 1.0e-15);
                                cross3(er, T, eth);
                                for (int d = 0; d < 3; ++d)
                                    vor[d][idx] = vor[d][idx] + tp * Gamma * (T[d] + eta * rho * eth[d] + (rho * dsds / sigma) * er[d]);
                                if (cond && cond[idx] < 1.0) cond[idx] = 1.0;
                            } else { /* curved branch, tube.f90:868-892 */
                                double B[3], Nv[3];
                                for (int d = 0; d < 3; ++d) B[d] = dcddc[d] / ndcddc;
                                cross3(B, T, Nv);
                                const double kap = ndcddc / (ndc * ndc * ndc);
                                const double costh = dot3(xc, Nv) / (nxc + 1.0e-15);
                                const double sinth = dot3(xc, B) / (nxc + 1.0e-15);
                                const double den = 1.0 - kap * rho * costh;
                                const double t5 = -(sinth * rho) / den;
                                const double t6 = costh * rho / den;
                                const double t7 = costh * rho * dsds / sigma / den;
                                const double t8 = sinth * rho * dsds / sigma / den;
                                for (int d = 0; d < 3; ++d)
                                    vor[d][idx] = vor[d][idx] + tp * Gamma * (T[d] + eta * (t5 * Nv[d] + t6 * B[d]) + (t7 * Nv[d] + t8 * B[d]));
                                if (cond && cond[idx] < fabs(1.0 / den)) cond[idx] = fabs(1.0 / den);
                            }
                            accepted_total += 1;
                        }
                    }
                }
            }
        }
    }
    if (stats) {
        stats[0] = (double)ntf_sum;
        stats[1] = (double)ln.ntf_max;
        stats[2] = (double)accepted_total;
    }
    line_free(&ln);
    return nsub;
}

/* ------------------------------------------------------------------ misc helpers */

/* Sequential FP64 sum of a.b over n (cal_helicity, subroutine.f90:1550-1569, without dv). */
double orc_dot_sum(long n, const double *ax, const double *ay, const double *az, const double *bx,
                   const double *by, const double *bz)
{
    double h = 0.0;
    for (long i = 0; i < n; ++i) h = h + ax[i] * bx[i] + ay[i] * by[i] + az[i] * bz[i];
    return h;
}

/* Structure functions, subroutine.f90:64-129 (serial FP64 loop as in the reference).
 * u*: N^3 arrays x fastest; r: nr separations; Sp out: [pmax][nr]. */
void orc_sp(int N, const double *ux, const double *uy, const double *uz, int pmax, const int *r,
            int nr, double *Sp, int nthreads)
{
    const double inv = 1.0;
    (void)inv;
    if (nthreads < 1) nthreads = 1;
    for (int q = 0; q < pmax * nr; ++q) Sp[q] = 0.0;
    /* parallel over (p, m) pairs; each pair accumulated serially in the reference order */
#pragma omp parallel for num_threads(nthreads) schedule(dynamic)
    for (int q = 0; q < pmax * nr; ++q) {
        const int p = q / nr + 1, m = q % nr, rr = r[m];
        double acc = 0.0;
        for (int k = 0; k < N; ++k)
            for (int j = 0; j < N; ++j)
                for (int i = 0; i < N; ++i) {
                    const size_t id = (size_t)i + (size_t)N * ((size_t)j + (size_t)N * k);
                    const size_t ix = (size_t)((i + rr) % N) + (size_t)N * ((size_t)j + (size_t)N * k);
                    const size_t iy = (size_t)i + (size_t)N * ((size_t)((j + rr) % N) + (size_t)N * k);
                    const size_t iz = (size_t)i + (size_t)N * ((size_t)j + (size_t)N * ((k + rr) % N));
                    const double dux = ux[ix] - ux[id], duy = uy[iy] - uy[id], duz = uz[iz] - uz[id];
                    double px = 1.0, py = 1.0, pz = 1.0;
                    for (int e = 0; e < p; ++e) { px *= dux; py *= duy; pz *= duz; }
                    double sp = px + py + pz;
                    sp = sp / N / N / N / 3.0;
                    acc = acc + sp;
                }
        Sp[(p - 1) * nr + m] = acc;
    }
}
