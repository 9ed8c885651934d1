// fwt_internal.h -- shared declarations of libfwt (not part of the public C-ABI).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/fwt.h"

namespace fwt {

constexpr double kPi = 3.141592653589793115997963468544185161590576171875;   // 4*datan(1d0)
constexpr double kPi2 = 6.28318530717958623199592693708837032318115234375;   // 8*datan(1d0)

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define FWT_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return ::fwt::fail(FWT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
#define FWT_CUFFT(call)                                                                    \
    do {                                                                                   \
        cufftResult r_ = (call);                                                           \
        if (r_ != CUFFT_SUCCESS)                                                           \
            return ::fwt::fail(FWT_E_CUDA, std::string(#call) + ": cufft error " + std::to_string((int)r_)); \
    } while (0)
#define FWT_TRY(call)                                                                      \
    do {                                                                                   \
        int rc_ = (call);                                                                  \
        if (rc_ != 0) return rc_;                                                          \
    } while (0)

// A device buffer that grows on demand and is freed with the context.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// Per-line set-up parameters on the device.
struct LineParam {
    double sigma_min, sigma_max, Gamma, length, Len;
    int n_T;
    int n_sec;          // nodes of the line
    int64_t node_off;   // first node of the line in the node arrays
    int64_t slot_off;   // first section slot of the line (n_sec + 1 slots per line)
};

// Sub-segment record (FP64), one per (section, t_j), t_j < ntf (tube.f90:767-798).
struct SubSeg {
    double ci0[3];   // unwrapped start (mark1, tube.f90:779-785)
    double ci1[3];   // unwrapped end
    double tci0[3], tci1[3];
    double s0, s1, ndci0;
    double ssec;     // s_list2(t_i, 1): zeta of the section start
    double zs0;      // s0 - ssec: section-local zeta of the start
    double Rt;       // truncation radius Rtube_ratio * max(sigma(s0), sigma(s1))
    int slot;        // global section slot
    int line;        // line index (0-based)
    int box_lo[3];   // 1-based unwrapped box (tube.f90:793-798)
    int box_hi[3];
};

struct Timers {
    cudaEvent_t ev[8];
    bool made = false;
};

struct Ctx {
    fwt_params p{};
    int dev = 0;
    int slab_z0 = 0, slab_nz = 0;   // z-slab context (fwt_set_slab): planes slab_z0 .. + slab_nz - 1; 0: whole grid
    double piece_rt_cells = -1.0;   // tuning: piece kernel radius limit in grid spacings (< 0: default)
    double raster_rt_cells = -1.0;  // tuning: radius limit of rasterised pieces in grid spacings (< 0: default)
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // asynchronous node upload (fwt_set_centerlines_async): its stream, and per chunk the node
    // count uploaded so far with the event that completes it
    cudaStream_t up_stream = nullptr;
    std::vector<std::pair<int64_t, cudaEvent_t>> up_events;

    // inputs (host)
    int nline = 0;
    std::vector<int64_t> npoint, node_off;
    std::vector<double> sigma, Gamma;
    std::vector<int> n_T, if_filter;
    bool have_lines = false;

    // node coordinates on the device (SoA)
    const double *d_x = nullptr, *d_y = nullptr, *d_z = nullptr;
    DevBuf b_nodes;   // owned copy when set from host

    // fields
    DevBuf b_w;       // omega, 3 N^3 (float or double)
    DevBuf b_u;       // u, 3 N^3
    DevBuf b_spec;    // spectral buffer, 3 N^2 (N/2+1) complex
    DevBuf b_fftws;   // cuFFT work area
    // optional field outputs (field_uw.dat, field_wd.dat): the reference's u_out and d_out
    int u_out = 0, d_out = 0;
    DevBuf b_aux_spec, b_aux_real, b_aux_acc, b_aux_out;   // their buffers, made on first use
    cufftHandle plan_r2c = 0, plan_c2r = 0;
    // the generator's plans, kept between calls (plan creation costs milliseconds and a device
    // synchronisation): key n2 for the single circulant row (batch 0) or (n2, batch)
    struct FftPlan {
        int n2, batch;
        cufftHandle h;
    };
    std::vector<FftPlan> fbb_plans;
    bool plans = false;
    size_t fft_ws_bytes = 0;

    // scratch (centerline set-up, deposition, statistics)
    DevBuf scratch[29];
    // pairs the FP32 tile kernels defer to FP64 (k_tile_common.cuh): their list, and the int64
    // fixed-point sums of their contributions (kSideStride int64 per grid point), folded into
    // omega by side_fold
    DevBuf b_defer, b_side;
    bool side_dirty = false;
    double defer_per_pair = 0.2;   // deferred pairs per (tile, record) pair of the last tile launch
    double defer_per_piece = 0.05; // deferred pairs per piece of the last scatter launch
    double scatter_rt_cells = -1.0;  // tuning: radius limit of the scatter path in grid spacings (< 0: default)
    double defer_max_pairs = 0.0;    // tuning: entries an overflowed deferred list grows to (<= 0: 2^26)

    // state
    bool have_w = false, have_u = false, normalised = false;
    bool w_written = false;   // omega holds deposited data (later batches accumulate)
    bool wmm_valid = false;   // wmin/wmax hold the raw omega component range
    double up = 1.0, Etot = 0.0, Etot_raw = 0.0, enstrophy = 0.0, enstrophy_raw = 0.0, lengthtot = 0.0;
    bool umm_valid = false;   // umin/umax hold the raw u component range
    std::vector<double> spec_w, spec_u;   // shells 1..N/2
    std::vector<int64_t> line_ntf_sum, line_ntf_max;  // per deposited line
    std::vector<int> line_nsec;
    std::vector<double> line_len;
    std::vector<double> wmin, wmax, umin, umax;  // per component, raw (unnormalised) fields, exact

    // statistics kept for file output
    std::vector<float> pdf_u_val, pdf_u, pdf_w_val, pdf_w;
    std::vector<int> sp_r;
    std::vector<double> sp;
    std::vector<float> field_wh;

    // timers / counters
    Timers tm;
    double t_ms[5] = {0, 0, 0, 0, 0};
    double t_deposit_wall_init = 0;
    int64_t counters[7] = {0, 0, 0, 0, 0, 0, 0};   // see fwt_counters
    int64_t launches = 0;
    size_t mem_held = 0;

    std::vector<double> timing_line;   // per line: set-up ms, construction ms

    // per-kernel device times of the last fwt_run (CUDA events on the context's stream)
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> ev_marks;   // (category, index of the start event)
    size_t ev_used = 0;
    double ktime[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t kcount[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double t_setup_acc = 0;
};

// kernel time categories
enum { KT_SECTION = 0, KT_CENTERLINE = 1, KT_BINNING = 2, KT_DEPOSIT = 3, KT_SPECTRAL = 4, KT_FFT = 5, KT_STATS = 6,
       KT_GEN = 7 };
int kt_begin(Ctx *c, int cat);            // records a start event; returns a mark id
void kt_end(Ctx *c, int mark);            // records the matching stop event
void kt_reset(Ctx *c);
int kt_collect(Ctx *c);                   // synchronises and sums elapsed times per category

// device memory helpers
int buf_reserve(Ctx *c, DevBuf &b, size_t bytes);
void buf_free(Ctx *c, DevBuf &b);

// centerline set-up + deposition (k_centerline.cu, k_deposit.cu)
int deposit_lines(Ctx *c, int line_s, int line_e);
int side_fold(Ctx *c);   // add the deferred pairs' sums into omega (k_deposit_tile.cu)

// spectral (k_spectral.cu)
int spectral_init(Ctx *c);
int spectral_filter(Ctx *c, double k_c);
int spectral_biot_savart(Ctx *c);
int spectral_block(Ctx *c, void *spec, int y0, int ny, double *host_sums);

// statistics (k_stats.cu)
int stats_minmax(Ctx *c, int which);
int stats_normalise(Ctx *c);
int stats_pdf(Ctx *c, int which, int comp, int nbins, float *val, float *pdf, uint64_t *counts);
int stats_sp(Ctx *c, int pmax, const int *r, int nr, double *Sp);
int stats_sp_block(Ctx *c, const void *u, int n0, int n1, int n2, int axis, double s, const int *r, int nr,
                   double *sums);
int stats_field_wh(Ctx *c, float *host_out);
// Make the context's stream wait until nodes [0, upto) of an asynchronous upload are on the
// device (fwt_api.cu); nothing to do after a synchronous one.
int wait_nodes(Ctx *c, int64_t upto);
// Finish an asynchronous upload (before the nodes' buffers or the caller's array are reused).
int finish_upload(Ctx *c);
int stats_field_uw(Ctx *c, float *host_out);
int stats_field_wd(Ctx *c, float *host_out);
int stats_copy_field(Ctx *c, int which, int comp, double *host);

// diagnostics (k_diag.cu)
int diag_vsf_deviation(Ctx *c, const void *d_phi, double *deviation);
int diag_helicity(Ctx *c, double *helicity);
int iso_extract(Ctx *c, float iso, float *host_tris, int64_t max_tris, int64_t *ntris, float *iso_used);

// host I/O (fwt_io.cpp)
int io_read_centerlines(const char *path, std::vector<int64_t> &npoint, std::vector<double> &xyz);
int io_read_params(const char *path, int nline, fwt_params &p, std::vector<double> &sigma,
                   std::vector<double> &Gamma, std::vector<int> &n_T, std::vector<int> &if_filter);
int io_write_outputs(Ctx *c, const char *outdir);

// generator (k_fbb.cu)
int fbb_generate(Ctx *c, uint64_t seed, int nlev, const int *tubes, const int *nodes, const double *H,
                 const double *dB, double *d_x, double *d_y, double *d_z);

int scaling_exponents(const double *rdr, const double *Sp, int nr, int pmax, double *zeta, double *flat);
inline size_t field_elems(const Ctx *c)
{
    return (size_t)c->p.N * c->p.N * (size_t)(c->slab_nz ? c->slab_nz : c->p.N);
}
inline size_t real_bytes(const Ctx *c) { return c->p.precision == 64 ? 8 : 4; }

}  // namespace fwt
