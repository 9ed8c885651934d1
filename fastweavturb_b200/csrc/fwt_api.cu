// fwt_api.cu -- the C-ABI of libfwt (include/fwt.h): context life cycle, inputs, the phase
// entry points and the whole-program driver.
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>

#include "k_centerline.cuh"

namespace fwt {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int buf_reserve(Ctx *c, DevBuf &b, size_t bytes)
{
    if (bytes <= b.bytes && b.p) return 0;
    // a buffer that grows takes 25 % headroom: cudaFree waits for the whole device, which
    // would stall the other contexts' streams whenever a realisation is slightly larger
    if (b.p && bytes < b.bytes + b.bytes / 4) {
        const size_t grown = b.bytes + b.bytes / 4;
        if (!c->p.mem_cap || c->mem_held - b.bytes + grown <= c->p.mem_cap) bytes = grown;
    }
    if (b.p) {
        cudaFree(b.p);
        c->mem_held -= b.bytes;
        b.p = nullptr;
        b.bytes = 0;
    }
    if (bytes == 0) bytes = 16;
    if (c->p.mem_cap && c->mem_held + bytes > c->p.mem_cap)
        return fail(FWT_E_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes exceeds the memory cap");
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        b.p = nullptr;
        cudaGetLastError();
        return fail(FWT_E_NOMEM, "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    b.bytes = bytes;
    c->mem_held += bytes;
    return 0;
}

void buf_free(Ctx *c, DevBuf &b)
{
    if (b.p) {
        cudaFree(b.p);
        c->mem_held -= b.bytes;
    }
    b.p = nullptr;
    b.bytes = 0;
}

int kt_begin(Ctx *c, int cat)
{
    if (c->ev_used + 2 > c->ev_pool.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
    }
    const int id = (int)c->ev_used;
    c->ev_used += 2;
    cudaEventRecord(c->ev_pool[id], c->stream);
    c->ev_marks.push_back({cat, id});
    return id;
}

void kt_end(Ctx *c, int mark)
{
    cudaEventRecord(c->ev_pool[mark + 1], c->stream);
    // FWT_SYNC_CHECK=1: wait after every timed kernel group and name the group of a fault
    static const bool check = std::getenv("FWT_SYNC_CHECK") != nullptr;
    if (check) {
        const cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) {
            int cat = -1;
            for (auto &m : c->ev_marks)
                if (m.second == mark) cat = m.first;
            std::fprintf(stderr, "libfwt: %s after kernel group %d (mark %d, %lld launches)\n", cudaGetErrorString(e),
                         cat, mark, (long long)c->launches);
        }
    }
}

void kt_reset(Ctx *c)
{
    c->ev_used = 0;
    c->ev_marks.clear();
    for (int i = 0; i < 8; ++i) {
        c->ktime[i] = 0;
        c->kcount[i] = 0;
    }
}

int kt_collect(Ctx *c)
{
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    for (auto &m : c->ev_marks) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c->ev_pool[m.second], c->ev_pool[m.second + 1]) == cudaSuccess) {
            c->ktime[m.first] += ms;
            c->kcount[m.first] += 1;
        }
    }
    c->ev_marks.clear();
    c->ev_used = 0;
    return 0;
}

// de-interleave m rows of row-major xyz (m x 3) into SoA x[], y[], z[] of stride n
__global__ void deinterleave_kernel(const double *__restrict__ aos, int64_t m, int64_t n, double *__restrict__ soa)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        soa[i] = aos[3 * i];
        soa[n + i] = aos[3 * i + 1];
        soa[2 * n + i] = aos[3 * i + 2];
    }
}

static int validate(const fwt_params &p)
{
    if (p.N < 4 || p.N > 2048 || (p.N & 1)) return fail(FWT_E_ARG, "N must be even and in 4..2048");
    if (p.N_downsample < 1 || p.N % p.N_downsample) return fail(FWT_E_ARG, "N_downsample must divide N");
    if (p.precision != 32 && p.precision != 64) return fail(FWT_E_ARG, "precision must be 32 or 64");
    if (p.ntf_times < 0 || p.ntf_pre < 1) return fail(FWT_E_ARG, "ntf_times >= 0 and ntf_pre >= 1 required");
    if (!(p.Rtube_ratio > 0) || !(p.dzeta_sup > 0) || !(p.sigma_ratio > 0))
        return fail(FWT_E_ARG, "Rtube_ratio, dzeta_sup and sigma_ratio must be positive");
    if (p.pdf_bins < 1 || p.pdf_bins > 8192) return fail(FWT_E_ARG, "pdf_bins must be 1..8192");
    if (p.Sp_order < 1 || p.Sp_order > 10) return fail(FWT_E_ARG, "Sp_order must be 1..10");
    return 0;
}

static void reset_state(Ctx *c)
{
    c->have_w = c->have_u = c->normalised = false;
    c->w_written = c->wmm_valid = c->umm_valid = false;
}

struct PhaseTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit PhaseTimer(cudaStream_t st) : s(st)
    {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    double stop()
    {
        float ms = 0;
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
    ~PhaseTimer()
    {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

int finish_upload(Ctx *c)
{
    if (!c->up_stream) return 0;
    const cudaError_t e = cudaStreamSynchronize(c->up_stream);
    for (auto &pe : c->up_events) cudaEventDestroy(pe.second);
    c->up_events.clear();
    if (e != cudaSuccess) return fail(FWT_E_CUDA, std::string("node upload: ") + cudaGetErrorString(e));
    return 0;
}

int wait_nodes(Ctx *c, int64_t upto)
{
    for (const auto &pe : c->up_events) {
        if (pe.first >= upto) {
            FWT_CUDA(cudaStreamWaitEvent(c->stream, pe.second, 0));
            return 0;
        }
    }
    return 0;
}

}  // namespace fwt

using namespace fwt;

extern "C" {

int fwt_last_error(char *buf, int len)
{
    if (!buf || len <= 0) return FWT_E_ARG;
    std::strncpy(buf, g_err.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
    return 0;
}

int fwt_default_params(fwt_params *p)
{
    if (!p) return fail(FWT_E_ARG, "null params");
    std::memset(p, 0, sizeof(*p));
    p->N = 256;
    p->N_downsample = 256;
    p->line_s = 1;
    p->line_e = 1;
    p->sigma_ratio = 4.0;
    p->eta_t = 0.0;
    p->ntf_times = 50;
    p->ntf_pre = 1000;
    p->Rtube_ratio = 3.0;
    p->dzeta_sup = 1e-4;
    p->precision = 32;
    p->deposit_mode = 0;
    p->device = 0;
    p->stream = nullptr;
    p->if_pdf = 1;
    p->if_Sp = 1;
    p->Sp_order = 10;
    p->pdf_bins = 1000;
    p->vorticity_output = 1;
    p->mem_cap = 0;
    return 0;
}

int fwt_create(const fwt_params *p, fwt_ctx **out)
{
    if (!p || !out) return fail(FWT_E_ARG, "null argument");
    FWT_TRY(validate(*p));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(FWT_E_CUDA, "no CUDA device: the woven-field library has no CPU path");
    }
    if (p->device < 0 || p->device >= ndev) return fail(FWT_E_ARG, "device ordinal out of range");
    Ctx *c = new Ctx();
    c->p = *p;
    c->dev = p->device;
    cudaError_t e = cudaSetDevice(c->dev);
    if (e != cudaSuccess) {
        delete c;
        return fail(FWT_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    if (p->stream) {
        c->stream = (cudaStream_t)p->stream;
    } else {
        e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete c;
            return fail(FWT_E_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        }
        c->own_stream = true;
    }
    *out = (fwt_ctx *)c;
    return 0;
}

int fwt_destroy(fwt_ctx *h)
{
    Ctx *c = (Ctx *)h;
    if (!c) return 0;
    cudaSetDevice(c->dev);
    cudaStreamSynchronize(c->stream);
    finish_upload(c);
    if (c->up_stream) cudaStreamDestroy(c->up_stream);
    if (c->plans) {
        cufftDestroy(c->plan_r2c);
        cufftDestroy(c->plan_c2r);
    }
    for (auto &p : c->fbb_plans) cufftDestroy(p.h);
    c->fbb_plans.clear();
    buf_free(c, c->b_nodes);
    buf_free(c, c->b_w);
    buf_free(c, c->b_u);
    buf_free(c, c->b_spec);
    buf_free(c, c->b_fftws);
    buf_free(c, c->b_aux_spec);
    buf_free(c, c->b_aux_real);
    buf_free(c, c->b_aux_acc);
    buf_free(c, c->b_aux_out);
    for (auto &b : c->scratch) buf_free(c, b);
    buf_free(c, c->b_defer);
    buf_free(c, c->b_side);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return 0;
}

static int set_lines_common(Ctx *c, int nline, const int64_t *npoint, const double *sigma, const double *Gamma,
                            const int *n_T, const int *if_filter)
{
    if (nline < 1 || !npoint || !sigma || !Gamma || !n_T) return fail(FWT_E_ARG, "bad centerline arguments");
    c->nline = nline;
    c->npoint.assign(npoint, npoint + nline);
    c->node_off.assign(nline + 1, 0);
    for (int l = 0; l < nline; ++l) {
        if (npoint[l] < 2) return fail(FWT_E_ARG, "every line needs at least 2 nodes");
        if (npoint[l] > (1 << 30)) return fail(FWT_E_RANGE, "line too long");
        if (!(sigma[l] > 0)) return fail(FWT_E_ARG, "sigma must be positive");
        c->node_off[l + 1] = c->node_off[l] + npoint[l];
    }
    c->sigma.assign(sigma, sigma + nline);
    c->Gamma.assign(Gamma, Gamma + nline);
    c->n_T.assign(n_T, n_T + nline);
    if (if_filter) c->if_filter.assign(if_filter, if_filter + nline);
    else c->if_filter.assign(nline, 0);
    c->have_lines = true;
    reset_state(c);
    return 0;
}

// The caller's row-major array in chunks of up to 32 Mi nodes (fast when it is pinned) through
// a staging buffer (scratch[27]), each chunk made SoA on the device.  Synchronous: on the
// context's stream, waited for.  Asynchronous: on the upload stream, one event per chunk, which
// wait_nodes makes the context's stream wait for batch by batch.
static int set_centerlines_host(Ctx *c, int nline, const int64_t *npoint, const double *xyz, const double *sigma,
                                const double *Gamma, const int *n_T, const int *if_filter, bool async)
{
    if (!c || !xyz) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    FWT_TRY(finish_upload(c));   // an earlier upload still reads the staging buffer
    FWT_TRY(set_lines_common(c, nline, npoint, sigma, Gamma, n_T, if_filter));
    const int64_t n = c->node_off[nline];
    FWT_TRY(buf_reserve(c, c->b_nodes, sizeof(double) * 3 * (size_t)n));
    double *d = (double *)c->b_nodes.p;
    const int64_t chunk = std::min<int64_t>(n, (int64_t)1 << 25);
    FWT_TRY(buf_reserve(c, c->scratch[27], sizeof(double) * 3 * (size_t)std::max<int64_t>(chunk, 1)));
    double *stage = (double *)c->scratch[27].p;
    cudaStream_t st = c->stream;
    if (async) {
        if (!c->up_stream) FWT_CUDA(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
        // the buffers may still be read by the context's earlier work
        cudaEvent_t ready;
        FWT_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        FWT_CUDA(cudaEventRecord(ready, c->stream));
        FWT_CUDA(cudaStreamWaitEvent(c->up_stream, ready, 0));
        cudaEventDestroy(ready);
        st = c->up_stream;
    }
    for (int64_t o = 0; o < n; o += chunk) {
        const int64_t m = std::min(chunk, n - o);
        FWT_CUDA(cudaMemcpyAsync(stage, xyz + 3 * o, sizeof(double) * 3 * (size_t)m, cudaMemcpyHostToDevice, st));
        deinterleave_kernel<<<(unsigned)std::min<int64_t>((m + 255) / 256, 148 * 16), 256, 0, st>>>(stage, m, n,
                                                                                                    d + o);
        c->launches += 1;
        FWT_CUDA(cudaGetLastError());
        if (async) {
            cudaEvent_t ev;
            FWT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            FWT_CUDA(cudaEventRecord(ev, st));
            c->up_events.emplace_back(o + m, ev);
        }
    }
    if (!async) FWT_CUDA(cudaStreamSynchronize(c->stream));
    c->d_x = d;
    c->d_y = d + n;
    c->d_z = d + 2 * n;
    return 0;
}

int fwt_set_centerlines(fwt_ctx *h, int nline, const int64_t *npoint, const double *xyz, const double *sigma,
                        const double *Gamma, const int *n_T, const int *if_filter)
{
    return set_centerlines_host((Ctx *)h, nline, npoint, xyz, sigma, Gamma, n_T, if_filter, false);
}

int fwt_set_centerlines_async(fwt_ctx *h, int nline, const int64_t *npoint, const double *xyz, const double *sigma,
                              const double *Gamma, const int *n_T, const int *if_filter)
{
    return set_centerlines_host((Ctx *)h, nline, npoint, xyz, sigma, Gamma, n_T, if_filter, true);
}

int fwt_set_centerlines_device(fwt_ctx *h, int nline, const int64_t *npoint, const double *d_x, const double *d_y,
                               const double *d_z, const double *sigma, const double *Gamma, const int *n_T,
                               const int *if_filter)
{
    Ctx *c = (Ctx *)h;
    if (!c || !d_x || !d_y || !d_z) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    FWT_TRY(finish_upload(c));
    FWT_TRY(set_lines_common(c, nline, npoint, sigma, Gamma, n_T, if_filter));
    c->d_x = d_x;
    c->d_y = d_y;
    c->d_z = d_z;
    return 0;
}

int fwt_check_inputs(const char *cpath, const char *ppath, fwt_params *p, int *nline, int64_t *nodes)
{
    if (!cpath || !ppath || !p) return fail(FWT_E_ARG, "null argument");
    std::vector<int64_t> np;
    std::vector<double> xyz, sig, gam;
    std::vector<int> nT, filt;
    FWT_TRY(io_read_centerlines(cpath, np, xyz));
    FWT_TRY(io_read_params(ppath, (int)np.size(), *p, sig, gam, nT, filt));
    FWT_TRY(validate(*p));
    if (p->line_s < 1 || p->line_e > (int)np.size() || p->line_s > p->line_e)
        return fail(FWT_E_ARG, "line_s..line_e outside 1..nline");
    for (size_t i = 0; i < np.size(); ++i)
        if (!(sig[i] > 0) || !std::isfinite(gam[i]) || nT[i] < 0)
            return fail(FWT_E_ARG, "line " + std::to_string(i + 1) + ": sigma must be positive, Gamma finite, n_T >= 0");
    if (nline) *nline = (int)np.size();
    if (nodes) {
        int64_t t = 0;
        for (auto v : np) t += v;
        *nodes = t;
    }
    return 0;
}

int fwt_load_inputs(fwt_ctx *h, const char *cpath, const char *ppath)
{
    Ctx *c = (Ctx *)h;
    if (!c || !cpath || !ppath) return fail(FWT_E_ARG, "null argument");
    std::vector<int64_t> np;
    std::vector<double> xyz, sig, gam;
    std::vector<int> nT, filt;
    FWT_TRY(io_read_centerlines(cpath, np, xyz));
    fwt_params p = c->p;
    FWT_TRY(io_read_params(ppath, (int)np.size(), p, sig, gam, nT, filt));
    FWT_TRY(validate(p));
    if (p.N != c->p.N || p.precision != c->p.precision) {
        // the grid size fixes the FFT plans and field buffers: rebuild them
        if (c->plans) {
            cufftDestroy(c->plan_r2c);
            cufftDestroy(c->plan_c2r);
            c->plans = false;
        }
    }
    c->p = p;
    return fwt_set_centerlines(h, (int)np.size(), np.data(), xyz.data(), sig.data(), gam.data(), nT.data(), filt.data());
}

int fwt_deposit(fwt_ctx *h, int line_s, int line_e)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    cudaSetDevice(c->dev);
    kt_reset(c);
    c->t_setup_acc = 0;
    PhaseTimer t(c->stream);
    const int rc = deposit_lines(c, line_s, line_e);
    c->t_ms[1] = t.stop();
    c->t_ms[0] = c->t_setup_acc;
    if (rc == 0) FWT_TRY(kt_collect(c));
    return rc;
}

int fwt_filter(fwt_ctx *h, double k_c)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    cudaSetDevice(c->dev);
    return spectral_filter(c, k_c);
}

int fwt_biot_savart(fwt_ctx *h)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    cudaSetDevice(c->dev);
    PhaseTimer t(c->stream);
    const int rc = spectral_biot_savart(c);
    c->t_ms[2] = t.stop();
    return rc;
}

int fwt_normalize(fwt_ctx *h, double *up, double *Etot, double *enstrophy)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    FWT_TRY(stats_normalise(c));
    if (up) *up = c->up;
    if (Etot) *Etot = c->Etot;
    if (enstrophy) *enstrophy = c->enstrophy;
    return 0;
}

int fwt_spectrum(fwt_ctx *h, int which, double *Ek, int nshell)
{
    Ctx *c = (Ctx *)h;
    if (!c || !Ek) return fail(FWT_E_ARG, "null argument");
    if (!c->have_u) return fail(FWT_E_STATE, "spectrum before Biot-Savart");
    if (which == 1 && !c->normalised) return fail(FWT_E_STATE, "velocity spectrum before normalisation");
    const std::vector<double> &s = which ? c->spec_u : c->spec_w;
    const double sc = which ? 1.0 / (c->up * c->up) : 1.0;
    for (int i = 0; i < nshell; ++i) Ek[i] = i < (int)s.size() ? s[i] * sc : 0.0;
    return 0;
}

int fwt_pdf(fwt_ctx *h, int which, int component, int nbins, float *val, float *pdf, uint64_t *counts)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    cudaSetDevice(c->dev);
    return stats_pdf(c, which, component, nbins, val, pdf, counts);
}

int fwt_sp(fwt_ctx *h, int pmax, const int *r, int nr, double *Sp)
{
    Ctx *c = (Ctx *)h;
    if (!c || !r || !Sp) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return stats_sp(c, pmax, r, nr, Sp);
}

int fwt_field_wh(fwt_ctx *h, float *host_out)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    cudaSetDevice(c->dev);
    return stats_field_wh(c, host_out);
}

int fwt_set_slab(fwt_ctx *h, int z0, int nz)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    const int N = c->p.N;
    if (nz == 0 && z0 == 0) {
        c->slab_z0 = c->slab_nz = 0;
    } else {
        if (z0 < 0 || nz <= 0 || z0 + nz > N || z0 % 8 || nz % 8)
            return fail(FWT_E_ARG, "slab: planes z0 .. z0 + nz - 1 within the grid, z0 and nz multiples of 8");
        if (c->p.deposit_mode != 0) return fail(FWT_E_ARG, "slab: the tile-owned deposition only (deposit_mode 0)");
        c->slab_z0 = z0;
        c->slab_nz = nz;
    }
    // the field buffers change size: the next deposition starts from zero
    buf_free(c, c->b_w);
    buf_free(c, c->b_u);
    buf_free(c, c->b_side);
    c->side_dirty = false;
    reset_state(c);
    return 0;
}

int fwt_biot_savart_block(fwt_ctx *h, void *spec, int y0, int ny, double *sums)
{
    Ctx *c = (Ctx *)h;
    if (!c || !spec || !sums) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return spectral_block(c, spec, y0, ny, sums);
}

int fwt_sp_block(fwt_ctx *h, const void *u, int n0, int n1, int n2, int axis, double scale, const int *r, int nr,
                 double *sums)
{
    Ctx *c = (Ctx *)h;
    if (!c || !u || !r || !sums) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return stats_sp_block(c, u, n0, n1, n2, axis, scale, r, nr, sums);
}

int fwt_vsf_deviation(fwt_ctx *h, const void *d_phi, double *deviation)
{
    Ctx *c = (Ctx *)h;
    if (!c || !deviation) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return diag_vsf_deviation(c, d_phi, deviation);
}

int fwt_helicity(fwt_ctx *h, double *helicity)
{
    Ctx *c = (Ctx *)h;
    if (!c || !helicity) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return diag_helicity(c, helicity);
}

int fwt_isosurface(fwt_ctx *h, float iso, float *tris, int64_t max_tris, int64_t *ntris, float *iso_used)
{
    Ctx *c = (Ctx *)h;
    if (!c || !ntris) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return iso_extract(c, iso, tris, max_tris, ntris, iso_used);
}

int fwt_field_device(fwt_ctx *h, int which, void **ptr)
{
    Ctx *c = (Ctx *)h;
    if (!c || !ptr) return fail(FWT_E_ARG, "null argument");
    if (which != 0 && which != 1) return fail(FWT_E_ARG, "field_device: which must be 0 (omega) or 1 (u)");
    if (which == 0 && !c->have_w) return fail(FWT_E_STATE, "omega not built");
    if (which == 1 && !c->have_u) return fail(FWT_E_STATE, "u not built");
    *ptr = which ? c->b_u.p : c->b_w.p;
    return 0;
}

int fwt_copy_field(fwt_ctx *h, int which, int component, double *host)
{
    Ctx *c = (Ctx *)h;
    if (!c || !host) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return stats_copy_field(c, which, component, host);
}

// r_m = floor(sqrt(2.0)**m + 0.5), m = 0..2*lg2L in REAL(4) (subroutine.f90:78,97-98)
static std::vector<int> sp_separations(int N)
{
    const float l2 = std::log((float)N) / std::log(2.0f);
    const int lg2L = (int)std::floor(l2 + 0.01f);
    const float s2 = std::sqrt(2.0f);
    std::vector<int> r;
    for (int m = 0; m <= 2 * lg2L; ++m) {
        float p = 1.0f, base = s2;
        int e = m;
        while (e) {
            if (e & 1) p = p * base;
            base = base * base;
            e >>= 1;
        }
        r.push_back((int)std::floor(p + 0.5f));
    }
    return r;
}

int fwt_run(fwt_ctx *h)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    if (!c->have_lines) return fail(FWT_E_STATE, "no centerlines set");
    cudaSetDevice(c->dev);
    const int64_t l0 = c->launches;
    reset_state(c);
    kt_reset(c);
    c->t_setup_acc = 0;
    PhaseTimer total(c->stream);
    {
        PhaseTimer t(c->stream);
        FWT_TRY(deposit_lines(c, c->p.line_s, c->p.line_e > 0 ? c->p.line_e : c->nline));
        c->t_ms[1] = t.stop();
    }
    {
        PhaseTimer t(c->stream);
        FWT_TRY(spectral_biot_savart(c));
        FWT_TRY(stats_normalise(c));
        c->t_ms[2] = t.stop();
    }
    {
        PhaseTimer t(c->stream);
        const int nb = c->p.pdf_bins;
        if (c->p.if_pdf) {
            c->pdf_u_val.resize(nb);
            c->pdf_u.resize(nb);
            c->pdf_w_val.resize(nb);
            c->pdf_w.resize(nb);
            FWT_TRY(stats_pdf(c, 0, -1, nb, c->pdf_u_val.data(), c->pdf_u.data(), nullptr));
            FWT_TRY(stats_pdf(c, 1, -1, nb, c->pdf_w_val.data(), c->pdf_w.data(), nullptr));
        }
        if (c->p.if_Sp) {
            c->sp_r = sp_separations(c->p.N);
            c->sp.assign((size_t)c->p.Sp_order * c->sp_r.size(), 0.0);
            FWT_TRY(stats_sp(c, c->p.Sp_order, c->sp_r.data(), (int)c->sp_r.size(), c->sp.data()));
        }
        if (c->p.vorticity_output) {
            // built on the device here; copied to the host by fwt_field_wh / fwt_write_outputs
            FWT_TRY(stats_field_wh(c, nullptr));
            c->field_wh.clear();
        }
        c->t_ms[3] = t.stop();
    }
    c->t_ms[4] = total.stop();
    c->t_ms[0] = c->t_setup_acc;
    c->counters[4] = c->launches - l0;
    FWT_TRY(kt_collect(c));
    // per-line times: the batch times apportioned by section count
    c->timing_line.assign(2 * (size_t)c->nline, 0.0);
    int64_t secs = 0;
    const int le = c->p.line_e > 0 ? c->p.line_e : c->nline;
    for (int l = c->p.line_s - 1; l < le; ++l) secs += c->npoint[l];
    for (int l = c->p.line_s - 1; l < le; ++l) {
        const double f = secs ? (double)c->npoint[l] / secs : 0.0;
        c->timing_line[2 * l] = c->t_ms[0] * 1e-3 * f;
        c->timing_line[2 * l + 1] = c->t_ms[1] * 1e-3 * f;
    }
    return 0;
}

int fwt_write_outputs(fwt_ctx *h, const char *outdir)
{
    Ctx *c = (Ctx *)h;
    if (!c || !outdir) return fail(FWT_E_ARG, "null argument");
    if (!c->normalised) return fail(FWT_E_STATE, "write_outputs before the statistics were built");
    if (c->p.vorticity_output && c->field_wh.empty()) {
        const size_t nd = (size_t)c->p.N_downsample;
        c->field_wh.resize(2 * nd * nd * nd);
        FWT_TRY(stats_field_wh(c, c->field_wh.data()));
    }
    return io_write_outputs(c, outdir);
}

int fwt_run_dir(const char *rundir, const fwt_params *p0)
{
    if (!rundir) return fail(FWT_E_ARG, "null run directory");
    fwt_params p;
    if (p0) p = *p0;
    else fwt_default_params(&p);
    fwt_ctx *h = nullptr;
    FWT_TRY(fwt_create(&p, &h));
    const std::string d = rundir;
    int rc = fwt_load_inputs(h, (d + "/centerline_input.dat").c_str(), (d + "/parameters_input.dat").c_str());
    if (rc == 0) rc = fwt_run(h);
    if (rc == 0) rc = fwt_write_outputs(h, (d + "/output").c_str());
    std::string keep = g_err;
    fwt_destroy(h);
    if (rc) g_err = keep;
    return rc;
}

int fwt_timings(fwt_ctx *h, double *t, int n)
{
    Ctx *c = (Ctx *)h;
    if (!c || !t) return fail(FWT_E_ARG, "null argument");
    int k = 0;
    for (; k < n && k < 5; ++k) t[k] = c->t_ms[k];
    return k;
}

int fwt_kernel_times(fwt_ctx *h, double *ms, int64_t *launches, int n)
{
    Ctx *c = (Ctx *)h;
    if (!c || !ms) return fail(FWT_E_ARG, "null argument");
    int k = 0;
    for (; k < n && k < 8; ++k) {
        ms[k] = c->ktime[k];
        if (launches) launches[k] = c->kcount[k];
    }
    return k;
}

int fwt_set_tuning(fwt_ctx *h, int key, double value)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    if (key == FWT_TUNE_RASTER_RT_CELLS) {
        c->raster_rt_cells = value;
        return 0;
    }
    if (key == FWT_TUNE_PIECE_RT_CELLS) {
        c->piece_rt_cells = value;
        return 0;
    }
    if (key == FWT_TUNE_SCATTER_RT_CELLS) {
        c->scatter_rt_cells = value;
        return 0;
    }
    if (key == FWT_TUNE_DEFER_MAX_PAIRS) {
        c->defer_max_pairs = value;
        return 0;
    }
    return fail(FWT_E_ARG, "unknown tuning key");
}

int fwt_set_outputs(fwt_ctx *h, int u_out, int d_out)
{
    Ctx *c = (Ctx *)h;
    if (!c) return fail(FWT_E_ARG, "null context");
    c->u_out = u_out ? 1 : 0;
    c->d_out = d_out ? 1 : 0;
    return 0;
}

int fwt_field_uw(fwt_ctx *h, float *host_out)
{
    Ctx *c = (Ctx *)h;
    if (!c || !host_out) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return stats_field_uw(c, host_out);
}

int fwt_field_wd(fwt_ctx *h, float *host_out)
{
    Ctx *c = (Ctx *)h;
    if (!c || !host_out) return fail(FWT_E_ARG, "null argument");
    cudaSetDevice(c->dev);
    return stats_field_wd(c, host_out);
}

int fwt_counters(fwt_ctx *h, int64_t *v, int n)
{
    Ctx *c = (Ctx *)h;
    if (!c || !v) return fail(FWT_E_ARG, "null argument");
    int k = 0;
    for (; k < n && k < 7; ++k) v[k] = c->counters[k];
    return k;
}

int fwt_fbb_generate(fwt_ctx *h, uint64_t seed, int nlev, const int *tubes, const int *nodes, const double *H,
                     const double *dB, double *d_x, double *d_y, double *d_z)
{
    Ctx *c = (Ctx *)h;
    if (!c || nlev < 1 || !tubes || !nodes || !H || !dB || !d_x || !d_y || !d_z)
        return fail(FWT_E_ARG, "bad generator arguments");
    cudaSetDevice(c->dev);
    return fbb_generate(c, seed, nlev, tubes, nodes, H, dB, d_x, d_y, d_z);
}

}  // extern "C"
