// k_centerline.cuh -- device-side centerline set-up of one batch of lines.
#pragma once

#include "k_common.cuh"

namespace fwt {

struct SegRec;

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
    std::vector<int64_t> line_ntf_sum;  // 2 x nl: sum(ntf), max(ntf) per line
    std::vector<double> Lens;           // Len_Disc per line
};

int centerline_setup(Ctx *c, int la, int lb, CenterlineBatch &B);
int scan_exclusive_i64(Ctx *c, int64_t *d_data, int64_t n, int64_t *d_total, DevBuf &tmp);

}  // namespace fwt
