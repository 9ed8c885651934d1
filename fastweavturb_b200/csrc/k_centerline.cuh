// k_centerline.cuh -- device-side centerline set-up of one batch of lines.
#pragma once

#include "k_common.cuh"

namespace fwt {

struct SegRec;
struct PieceRec;

// cze_pl of slot t of a line (tube.f90:565,578,590)
__device__ __forceinline__ double cze_pl_at(const double *cze_line, int np, int t)
{
    if (t < np) return cze_line[t];
    if (t == np) return dev_pi2();
    return dev_pi2() + cze_line[1];
}

// cminus (subroutine.f90:695-710): r - l wrapped once per component
__device__ __forceinline__ void cminus3(const double *r, const double *l, double *d)
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double v = r[k] - l[k];
        if (v > dev_pi()) v = v - dev_pi2();
        if (v < -dev_pi()) v = v + dev_pi2();
        d[k] = v;
    }
}

// Spline position in Horner form with one wrap into [-pi, pi) (coo_curve_spline_5th,
// subroutine.f90:490-518): the sample positions of the sub-segment set-up.
__device__ __forceinline__ void spl_pos_fma(const double *__restrict__ a6, double z, double *c3)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double *a = a6 + 6 * d;
        double v = fma(fma(fma(fma(fma(a[5], z, a[4]), z, a[3]), z, a[2]), z, a[1]), z, a[0]);
        if (v >= dev_pi()) v = v - dev_pi2();
        if (v < -dev_pi()) v = v + dev_pi2();
        c3[d] = v;
    }
}

// Device arrays of one batch of lines (all views into Ctx::scratch).
struct CenterlineBatch {
    int la = 0, nl = 0;          // first line (0-based) and number of lines
    int64_t node_base = 0;       // global index of the batch's first node
    int64_t nodes = 0, nslots = 0, nsamples = 0, nsub = 0;
    LineParam *lp = nullptr;     // nl
    int *slot_line = nullptr;    // nslots -> batch-local line
    double *cze = nullptr, *ck = nullptr, *ckk = nullptr, *Len = nullptr;
    double *coe = nullptr;       // nslots x 18  ([coord][6])
    int *ntf = nullptr;          // nslots
    double *dtf = nullptr;       // nslots
    int64_t *soff = nullptr;     // nslots + 1: first sample of each slot
    int64_t *qoff = nullptr;     // nslots + 1: first sub-segment of each slot
    double *s = nullptr, *ci = nullptr, *tci = nullptr, *ndci = nullptr;  // per sample
    SubSeg *seg = nullptr;       // nsub FP64 records (reference box walk)
    SegRec *rec = nullptr;       // nsub FP32 records (tile-owned kernel)
    int64_t npieces = 0;         // chord pieces (piece kernel)
    PieceRec *piece = nullptr;   // npieces FP32 piece records
    bool raster = false;                 // pieces rasterised once (thin tubes), see piece_raster
    bool scatter = false;                // pieces deposited without tiles (scatter_piece_kernel)
    const int64_t *ras_off = nullptr;    // piece -> first rasterised point (npieces + 1)
    const uint32_t *ras_pts = nullptr;   // chord | x << 3 | y << 12 | z << 21 per accepted point
    const int *rec_map = nullptr;        // record (sub-segment or piece) -> section slot
    const int64_t *rec_first = nullptr;  // section slot -> its first record
    std::vector<int64_t> line_ntf_sum;  // 2 x nl: sum(ntf), max(ntf) per line
    std::vector<double> Lens;           // Len_Disc per line
};

// Records built for the batch: sub-segment records for the tile kernel, FP64 sample arrays for
// the reference box walk, or chord pieces for the piece kernel.
enum class BatchRecords { SubSeg, Walk, Pieces };
int centerline_setup(Ctx *c, int la, int lb, CenterlineBatch &B, BatchRecords mode);
int piece_setup(Ctx *c, CenterlineBatch &B);
int subseg64_setup(Ctx *c, CenterlineBatch &B);
int scan_exclusive_i64(Ctx *c, int64_t *d_data, int64_t n, int64_t *d_total, DevBuf &tmp);

}  // namespace fwt
