// fwt_io.cpp -- the reference's file interface: input parsing (tube.f90:168-223, 341-379)
// and the output tree (tube.f90:171,226-258,519-526,623,672-676,943-953,972-1188,1197-1211;
// subroutine.f90:42-62,114-123,1389-1399,1604-1638).
//
// List-directed output follows the Intel Fortran layout the reference was built with
// (Makefile: mpiifx): INTEGER as I12, REAL(4) as G15.7 with 1P E-form, REAL(8) as G24.15
// with 1P E-form and a 3-digit exponent, character items preceded by one blank.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "fwt_internal.h"

namespace fwt {

// ---------------------------------------------------------------------------- formatting
static std::string f_int(long long v)
{
    char b[40];
    snprintf(b, sizeof b, "%12lld", v);
    return b;
}

// Fortran Gw.d editing with scale factor 1 for the E form.
static std::string f_g(double x, int w, int d, int e)
{
    char b[96];
    if (x == 0.0) {
        // Intel prints zero in E form for list-directed reals
        snprintf(b, sizeof b, "%.*fE+%0*d", d, 0.0, e, 0);
        std::string s = b;
        return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
    }
    if (!std::isfinite(x)) {
        std::string s = std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity");
        return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
    }
    // decimal exponent after rounding to d significant digits
    snprintf(b, sizeof b, "%.*e", d - 1, x);
    const char *ep = strchr(b, 'e');
    const int k = atoi(ep + 1) + 1;   // 10^(k-1) <= |x| < 10^k
    const double ax = std::fabs(x);
    if (ax >= 0.1 && k <= d && k >= 0) {
        const int fw = w - (e + 2);
        snprintf(b, sizeof b, "%*.*f", fw, d - k, x);
        return std::string(b) + std::string(e + 2, ' ');
    }
    // 1PEw.dEe: one digit before the point, d decimals
    snprintf(b, sizeof b, "%.*e", d, x);
    std::string s = b;
    const size_t p = s.find('e');
    std::string mant = s.substr(0, p);
    int ex = atoi(s.c_str() + p + 1);
    char eb[16];
    snprintf(eb, sizeof eb, "E%c%0*d", ex < 0 ? '-' : '+', e, std::abs(ex));
    s = mant + eb;
    return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
}

static std::string f_r4(float x) { return f_g((double)x, 15, 7, 2); }
static std::string f_r8(double x) { return f_g(x, 24, 15, 3); }
static std::string f_str(const std::string &s) { return " " + s; }

// ESw.d
static std::string f_es(double x, int w, int d)
{
    char b[64];
    snprintf(b, sizeof b, "%.*e", d, x);
    std::string s = b;
    const size_t p = s.find('e');
    int ex = atoi(s.c_str() + p + 1);
    char eb[16];
    snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    s = s.substr(0, p) + eb;
    return std::string(w > (int)s.size() ? w - (int)s.size() : 0, ' ') + s;
}

// ---------------------------------------------------------------------------- input
static int read_tokens(const char *path, std::vector<std::string> &lines)
{
    std::ifstream f(path);
    if (!f) return fail(FWT_E_IO, std::string("cannot open ") + path);
    std::string ln;
    while (std::getline(f, ln)) lines.push_back(ln);
    return 0;
}

int io_read_centerlines(const char *path, std::vector<int64_t> &npoint, std::vector<double> &xyz)
{
    std::ifstream f(path);
    if (!f) return fail(FWT_E_IO, std::string("cannot open ") + path);
    double v;
    if (!(f >> v)) return fail(FWT_E_IO, "centerline file: missing nline");
    const long nline = (long)v;
    if (nline < 1 || (double)nline != v) return fail(FWT_E_IO, "centerline file: bad nline");
    npoint.resize(nline);
    int64_t total = 0;
    for (long i = 0; i < nline; ++i) {
        if (!(f >> v) || v < 2 || v != std::floor(v)) return fail(FWT_E_IO, "centerline file: bad npoint (need >= 2)");
        npoint[i] = (int64_t)v;
        total += npoint[i];
    }
    xyz.resize((size_t)total * 3);
    std::string tok;
    for (int64_t i = 0; i < total * 3; ++i) {
        if (!(f >> tok)) return fail(FWT_E_IO, "centerline file: truncated node list");
        // strtod also reads Fortran's NaN / Infinity spellings, which are then refused as such
        for (char &ch : tok)
            if (ch == 'D' || ch == 'd') ch = 'E';
        char *end = nullptr;
        xyz[i] = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str() || *end != 0)
            return fail(FWT_E_IO, "centerline file: non-numeric coordinate '" + tok + "'");
        if (!std::isfinite(xyz[i])) return fail(FWT_E_IO, "centerline file: non-finite coordinate");
    }
    return 0;
}

static bool parse_num(const std::string &s, double &v)
{
    std::istringstream is(s);
    return (bool)(is >> v);
}

int io_read_params(const char *path, int nline, fwt_params &p, std::vector<double> &sigma, std::vector<double> &Gamma,
                   std::vector<int> &n_T, std::vector<int> &if_filter)
{
    std::vector<std::string> L;
    FWT_TRY(read_tokens(path, L));
    // label / value pairs (tube.f90:192-217); value rows are the even 1-based lines
    const int vrow[10] = {1, 3, 5, 7, 9, 11, 14, 16, 18, 20};
    double v[10];
    for (int i = 0; i < 10; ++i) {
        if ((int)L.size() <= vrow[i] || !parse_num(L[vrow[i]], v[i]))
            return fail(FWT_E_IO, std::string("parameters file: bad value on line ") + std::to_string(vrow[i] + 1));
    }
    p.N = (int)v[0];
    p.N_downsample = (int)v[1];
    p.line_s = (int)v[2];
    p.line_e = (int)v[3];
    p.sigma_ratio = v[4];
    p.eta_t = v[5];
    p.ntf_times = (int)v[6];
    p.ntf_pre = (int)v[7];
    p.Rtube_ratio = v[8];
    p.dzeta_sup = v[9];
    sigma.assign(nline, 0.0);
    Gamma.assign(nline, 0.0);
    n_T.assign(nline, 0);
    if_filter.assign(nline, 0);
    std::vector<char> seen(nline, 0);
    for (int r = 0; r < nline; ++r) {
        const size_t row = 23 + r;
        if (row >= L.size()) return fail(FWT_E_IO, "parameters file: fewer line rows than nline");
        std::istringstream is(L[row]);
        double i, s, g, t, fl;
        if (!(is >> i >> s >> g >> t >> fl)) return fail(FWT_E_IO, "parameters file: bad line row " + std::to_string(r + 1));
        const int ii = (int)i - 1;
        if (ii < 0 || ii >= nline) return fail(FWT_E_IO, "parameters file: line index out of range");
        sigma[ii] = s;
        Gamma[ii] = g;
        n_T[ii] = (int)t;
        if_filter[ii] = (int)fl;
        seen[ii] = 1;
    }
    for (int i = 0; i < nline; ++i)
        if (!seen[i]) return fail(FWT_E_IO, "parameters file: missing row for line " + std::to_string(i + 1));
    return 0;
}

// ---------------------------------------------------------------------------- output
static int mkdir_p(const std::string &d)
{
    std::string cur;
    std::stringstream ss(d);
    std::string part;
    if (!d.empty() && d[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return fail(FWT_E_IO, "cannot create " + cur);
    }
    return 0;
}

static int open_w(const std::string &path, FILE **f)
{
    *f = fopen(path.c_str(), "w");
    if (!*f) return fail(FWT_E_IO, "cannot write " + path);
    return 0;
}

int io_write_outputs(Ctx *c, const char *outdir)
{
    const std::string od = outdir;
    FWT_TRY(mkdir_p(od));
    FWT_TRY(mkdir_p(od + "/stat"));
    FILE *f;
    // parameters_output.dat (tube.f90:226-258)
    FWT_TRY(open_w(od + "/parameters_output.dat", &f));
    fprintf(f, "%s\n%s\n", f_str("N").c_str(), f_int(c->p.N).c_str());
    fprintf(f, "%s\n%s\n", f_str("N_downsample").c_str(), f_int(c->p.N_downsample).c_str());
    fprintf(f, "%s\n%s\n", f_str("line_s").c_str(), f_int(c->p.line_s).c_str());
    fprintf(f, "%s\n%s\n", f_str("line_e").c_str(), f_int(c->p.line_e).c_str());
    fprintf(f, "%s\n%s\n", f_str("sigma_ratio").c_str(), f_r8(c->p.sigma_ratio).c_str());
    fprintf(f, "%s\n%s\n", f_str("eta_t").c_str(), f_r8(c->p.eta_t).c_str());
    fprintf(f, "%s\n", f_str("---------------").c_str());
    fprintf(f, "%s\n%s\n", f_str("ntf_times").c_str(), f_int(c->p.ntf_times).c_str());
    fprintf(f, "%s\n%s\n", f_str("ntf_pre").c_str(), f_int(c->p.ntf_pre).c_str());
    fprintf(f, "%s\n%s\n", f_str("Rtube_ratio").c_str(), f_r8(c->p.Rtube_ratio).c_str());
    fprintf(f, "%s\n%s\n", f_str("dzeta_sup").c_str(), f_r8(c->p.dzeta_sup).c_str());
    fprintf(f, "%s\n", f_str("---------------").c_str());
    fprintf(f, "%s\n", f_str("variables=\"i_line\",\"sigma\",\"Gamma\",\"n_T\",\"if_filter\"").c_str());
    for (int l = 0; l < c->nline; ++l)
        fprintf(f, "%s%s%s%s%s\n", f_int(l + 1).c_str(), f_r4((float)c->sigma[l]).c_str(), f_r4((float)c->Gamma[l]).c_str(),
                f_int(c->n_T[l]).c_str(), f_int(c->if_filter[l]).c_str());
    fclose(f);
    // centerline_output.dat (tube.f90:171-173,345-372), nodes read back from the device
    const int64_t nn = c->node_off[c->nline];
    std::vector<double> X(nn), Y(nn), Z(nn);
    FWT_CUDA(cudaMemcpyAsync(X.data(), c->d_x, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(Y.data(), c->d_y, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(Z.data(), c->d_z, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    FWT_TRY(open_w(od + "/centerline_output.dat", &f));
    fprintf(f, "%s\n", f_int(c->nline).c_str());
    for (int l = 0; l < c->nline; ++l) fprintf(f, "%s\n", f_int(c->npoint[l]).c_str());
    for (int64_t i = 0; i < nn; ++i) fprintf(f, "%s%s%s\n", f_r8(X[i]).c_str(), f_r8(Y[i]).c_str(), f_r8(Z[i]).c_str());
    fclose(f);
    // total length of every line (tube.f90:501-502): Len_Disc * 2pi, i.e. the periodic
    // polygon length; lines outside line_s..line_e were not set up on the device
    c->lengthtot = 0.0;
    for (int l = 0; l < c->nline; ++l) {
        double L = (l < (int)c->line_len.size()) ? c->line_len[l] : 0.0;
        if (L == 0.0) {
            const int64_t o = c->node_off[l], n = c->npoint[l];
            double cze = 0.0;
            for (int64_t i = 0; i < n; ++i) {
                const int64_t j = (i + 1) % n;
                const double dd[3] = {std::fabs(X[o + j] - X[o + i]), std::fabs(Y[o + j] - Y[o + i]),
                                      std::fabs(Z[o + j] - Z[o + i])};
                double s2 = 0;
                for (int d = 0; d < 3; ++d) {
                    double v = dd[d];
                    if (v > kPi) v -= kPi2;
                    s2 += v * v;
                }
                cze += std::sqrt(s2);
            }
            L = cze;
        }
        c->lengthtot += L;
    }
    // test_data.dat (tube.f90:623,673-676): two records per deposited line
    FWT_TRY(open_w(od + "/test_data.dat", &f));
    for (int l = c->p.line_s - 1; l < c->p.line_e && l < (int)c->line_ntf_sum.size(); ++l) {
        fprintf(f, "%s%s\n", f_str("ntf_average=").c_str(), f_int(c->line_ntf_sum[l] / (c->npoint[l] + 1)).c_str());
        fprintf(f, "%s%s\n", f_str("ntf_max=").c_str(), f_int(c->line_ntf_max[l]).c_str());
    }
    fclose(f);
    // info.dat (tube.f90:519-526,943-953,983-1034,1193-1210); times are device times (s)
    FWT_TRY(open_w(od + "/info.dat", &f));
    fprintf(f, "%s%s\n", f_str("Initialization time is").c_str(), f_r8(c->t_ms[0] * 1e-3).c_str());
    fprintf(f, "%s\n", f_str("==============================").c_str());
    fprintf(f, "%s\n", f_str("   [i] [Section count] [Spline time] [Construction time]").c_str());
    for (int l = c->p.line_s - 1; l < c->p.line_e && 2 * l + 1 < (int)c->timing_line.size(); ++l) {
        char b[16];
        snprintf(b, sizeof b, "%6d", l + 1);
        char b2[24];
        snprintf(b2, sizeof b2, "%16lld", (long long)c->npoint[l]);
        fprintf(f, "%s%s%s%s\n", b, b2, f_es(c->timing_line[2 * l], 18, 3).c_str(),
                f_es(c->timing_line[2 * l + 1], 18, 3).c_str());
    }
    fprintf(f, "%s\n", f_str("==============================").c_str());
    fprintf(f, "%s%s\n", f_str("Total construction time =").c_str(), f_r8(c->t_ms[1] * 1e-3).c_str());
    fprintf(f, "%s\n", f_str("velocity calculation begin").c_str());
    fprintf(f, "%s\n", f_str("velocity calculation done").c_str());
    fprintf(f, "%s%s\n", f_str("Etot_temp =").c_str(), f_r8(c->Etot).c_str());
    fprintf(f, "%s%s\n", f_str("up_temp =").c_str(), f_r8(c->up).c_str());
    fprintf(f, "%s%s\n", f_str("Post processing time =").c_str(), f_r8((c->t_ms[2] + c->t_ms[3]) * 1e-3).c_str());
    fprintf(f, "%s\n", f_str("==============================").c_str());
    fprintf(f, "%s%s\n", f_str("N = ").c_str(), f_int(c->p.N).c_str());
    fprintf(f, "%s%s\n", f_str("Total length of curve = ").c_str(), f_r8(c->lengthtot).c_str());
    fprintf(f, "%s%s\n", f_str("Gamma_1 = ").c_str(), f_r8(c->Gamma.empty() ? 0.0 : c->Gamma[0] / c->up).c_str());
    fprintf(f, "%s%s\n", f_str("twist eta = ").c_str(), f_r8(c->p.eta_t).c_str());
    fprintf(f, "%s%s\n", f_str("Etot = ").c_str(), f_r8(c->Etot / c->up / c->up).c_str());
    fprintf(f, "%s%s\n", f_str("Enstrophy = ").c_str(), f_r8(c->enstrophy).c_str());
    fclose(f);
    // spectra (subroutine.f90:1636): i, REAL(4) spectrum_k
    FWT_TRY(open_w(od + "/stat/spectrum_vor_temp.dat", &f));
    for (size_t i = 0; i < c->spec_w.size(); ++i)
        fprintf(f, "%s%s\n", f_int((long long)i + 1).c_str(), f_r4((float)c->spec_w[i]).c_str());
    fclose(f);
    FWT_TRY(open_w(od + "/stat/spectrum.dat", &f));
    const double iu2 = 1.0 / (c->up * c->up);
    for (size_t i = 0; i < c->spec_u.size(); ++i)
        fprintf(f, "%s%s\n", f_int((long long)i + 1).c_str(), f_r4((float)(c->spec_u[i] * iu2)).c_str());
    fclose(f);
    // PDFs (subroutine.f90:58-60)
    if (c->p.if_pdf) {
        FWT_TRY(open_w(od + "/stat/pdf_um.dat", &f));
        for (size_t i = 0; i < c->pdf_u.size(); ++i)
            fprintf(f, "%s%s\n", f_r4(c->pdf_u_val[i]).c_str(), f_r4(c->pdf_u[i]).c_str());
        fclose(f);
        FWT_TRY(open_w(od + "/stat/pdf_wm.dat", &f));
        for (size_t i = 0; i < c->pdf_w.size(); ++i)
            fprintf(f, "%s%s\n", f_r4(c->pdf_w_val[i]).c_str(), f_r4(c->pdf_w[i]).c_str());
        fclose(f);
    }
    // Sp.dat (subroutine.f90:114-123): r*dr then S_1..S_p, ES16.5 each
    if (c->p.if_Sp && !c->sp_r.empty()) {
        FWT_TRY(open_w(od + "/stat/Sp.dat", &f));
        const double dr = kPi2 / c->p.N;
        const int nr = (int)c->sp_r.size();
        const int pm = (int)(c->sp.size() / nr);
        for (int m = 0; m < nr; ++m) {
            std::string row = f_es(c->sp_r[m] * dr, 16, 5);
            for (int p = 0; p < pm; ++p) row += f_es(c->sp[p * nr + m], 16, 5);
            fprintf(f, "%s\n", row.c_str());
        }
        fclose(f);
    }
    // Sp_zeta.dat (output/stat/Sp_zeta.m:47-67): p, zeta_p and the K41 value p/3 for even
    // p = 2..10, tab-separated
    if (c->p.if_Sp && c->sp_r.size() >= 10 && c->sp.size() / c->sp_r.size() >= 10) {
        const int nr = (int)c->sp_r.size();
        std::vector<double> rdr(nr), zeta(10);
        for (int m = 0; m < nr; ++m) rdr[m] = c->sp_r[m] * (kPi2 / c->p.N);
        FWT_TRY(scaling_exponents(rdr.data(), c->sp.data(), nr, 10, zeta.data(), nullptr));
        FWT_TRY(open_w(od + "/stat/Sp_zeta.dat", &f));
        for (int p = 2; p <= 10; p += 2) fprintf(f, "%d\t%.15g\t%.15g\n", p, zeta[p - 1], p / 3.0);
        fclose(f);
    }
    // field_wh.dat: raw float32 stream, Fortran order (n_d, n_d, n_d, 2) (subroutine.f90:1396-1398)
    if (c->p.vorticity_output && !c->field_wh.empty()) {
        FWT_TRY(open_w(od + "/field_wh.dat", &f));
        const size_t n = c->field_wh.size();
        if (fwrite(c->field_wh.data(), sizeof(float), n, f) != n) {
            fclose(f);
            return fail(FWT_E_IO, "short write of field_wh.dat");
        }
        fclose(f);
    }
    // field_uw.dat (n_d^3 x 6: ux, uy, uz, wx, wy, wz) and field_wd.dat (n_d^3 x 2: |w|,
    // S_ij S_ij), the same stream format, when the reference's u_out / d_out are set
    // (tube.f90:1075-1120, inside its vorticity_output block)
    const size_t nd3 = (size_t)c->p.N_downsample * c->p.N_downsample * c->p.N_downsample;
    for (int which = 0; which < 2; ++which) {
        if (!c->p.vorticity_output || !(which == 0 ? c->u_out : c->d_out)) continue;
        const size_t n = (which == 0 ? 6 : 2) * nd3;
        std::vector<float> box(n);
        FWT_TRY(which == 0 ? stats_field_uw(c, box.data()) : stats_field_wd(c, box.data()));
        const std::string name = which == 0 ? "/field_uw.dat" : "/field_wd.dat";
        FWT_TRY(open_w(od + name, &f));
        if (fwrite(box.data(), sizeof(float), n, f) != n) {
            fclose(f);
            return fail(FWT_E_IO, "short write of " + name.substr(1));
        }
        fclose(f);
    }
    return 0;
}

}  // namespace fwt
