// fwt_scaling.cpp -- scaling exponents zeta_p and flatness from S_p(r), the reference's
// post-processing of Sp.dat (output/stat/Sp_zeta.m:3-23, output/stat/Flatness.m:14-19):
//   zeta_p   least-squares slope of log|S_p| against log(r dr) over the six rows
//            i_e - 5 .. i_e, i_e = nrows - 4 (1-based rows of Sp.dat)
//   F(r)     S_4(r) / S_2(r)^2 on every row
// Host arithmetic in FP64; no device work.
#include <cmath>
#include <string>

#include "fwt_internal.h"

namespace fwt {

// slope of the degree-1 least-squares fit y = a x + b
static double ls_slope(const double *x, const double *y, int n)
{
    double sx = 0, sy = 0;
    for (int i = 0; i < n; ++i) {
        sx += x[i];
        sy += y[i];
    }
    const double mx = sx / n, my = sy / n;
    double sxy = 0, sxx = 0;
    for (int i = 0; i < n; ++i) {
        sxy += (x[i] - mx) * (y[i] - my);
        sxx += (x[i] - mx) * (x[i] - mx);
    }
    return sxy / sxx;
}

int scaling_exponents(const double *rdr, const double *Sp, int nr, int pmax, double *zeta, double *flat)
{
    if (!rdr || !Sp || nr < 1 || pmax < 1) return fail(FWT_E_ARG, "sp_exponents: null argument or empty table");
    if (zeta) {
        if (nr < 10) return fail(FWT_E_RANGE, "sp_exponents: zeta_p needs at least 10 separations");
        const int ie = nr - 4, is = ie - 5;   // 1-based rows, Sp_zeta.m:6-7
        double x[6], y[6];
        for (int p = 1; p <= pmax; ++p) {
            for (int k = 0; k < 6; ++k) {
                const int m = is - 1 + k;
                x[k] = std::log(rdr[m]);
                y[k] = std::log(std::fabs(Sp[(size_t)(p - 1) * nr + m]));
            }
            zeta[p - 1] = ls_slope(x, y, 6);
        }
    }
    if (flat) {
        if (pmax < 4) return fail(FWT_E_RANGE, "sp_exponents: flatness needs S_2 and S_4");
        for (int m = 0; m < nr; ++m) {
            const double s2 = Sp[(size_t)1 * nr + m], s4 = Sp[(size_t)3 * nr + m];
            flat[m] = s4 / (s2 * s2);
        }
    }
    return 0;
}

}  // namespace fwt

extern "C" int fwt_sp_exponents(const double *rdr, const double *Sp, int nr, int pmax, double *zeta, double *flat)
{
    return fwt::scaling_exponents(rdr, Sp, nr, pmax, zeta, flat);
}
