// k_deposit_piece.cu -- tile-owned deposition of thin tubes by chord pieces.
//
// The reference deposits sub-segment by sub-segment (tube.f90:762-904): chord j of a section
// accepts a mesh point x when t_j(x) = (x - ci_j) . tci_j >= 0, t_{j+1}(x) < 0 (the next
// chord's plane) and the distance to chord line j is below Rtube, inside chord j's box.
// Consecutive chords share their planes (tube.f90:721-723,740-751), so a run of chords of one
// section can share one record: the section's spline, the run's planes and per-sample frames.
// For tubes up to a few grid spacings thick, where a sub-segment accepts only a handful of
// points, this cuts the set-up, the binning and the record traffic by the run length.
//
// A piece is up to kPieceMax consecutive chords of one section.  Its record holds the
// section's quintic Taylor-shifted to the piece start, the planes (normal, offset), per sample
// the offset of the box origin in that sample's own frame, and per chord the spline slope,
// Rtube^2 and the chord's own box.  Pieces are binned into tiles like sub-segments; the kernel
// stages a warp's pieces with bulk asynchronous copies and gives each lane one chord, whose
// rows within the tile (along the axis best aligned with the chord) are limited, column by
// column, to the projection of the part of the chord's cylinder it can accept; the rows are
// spread over the lanes, each row's index interval that can pass the chord's two planes and
// its cylinder is solved in closed form, and only the points of that interval take the
// reference's tests, 32 candidates at a time.  The accepted (point, chord) pairs are queued
// and evaluated 32 at a time with the vorticity code of the sub-segment kernel, into the same
// int64 fixed-point cells.
#include <cstdio>
#include <cstdlib>

#include "k_deposit.cuh"
#include "k_tile_common.cuh"

namespace fwt {

constexpr int kPieceMax = 8;   // chords per piece
constexpr int kScatterMaxOff = 254;   // piece-frame offsets of the scatter kernel's 8-bit candidate codes

struct __align__(16) PieceRec {
    float off[3], dx;       // mesh point at box_lo minus the origin o (the piece's first sample)
    float b[15], smin;      // c(z0 + W) - c(z0) = sum_k b[k-1] W^k about the piece start z0
    float thi[3], A;        // wrap thresholds pi - c(z0) (see SegF); core amplitude
    float tlo[3], om;
    int kq[3];
    float ph0;
    float inv2s2, ftd, amp, Gamma;   // constant-core profile (tube.f90:845-847)
    float Linv, eta, q, guard;       // guard: rounding bound of the piece-frame plane tests
    int box_lo[3];
    int nch;                // chords of the piece, 1..kPieceMax
    int box_hi[3];
    int pad1;
    float4 pl[kPieceMax + 1];   // plane k: (tci_k, tci_k . p_k) with p_k = ci_k - o; plane nch is
                                // the next chord's
    float4 po[kPieceMax + 1];   // sample k: (mesh point at box_lo minus ci_k, zoff_k = z_k - z0)
    float4 chq[kPieceMax];      // chord j: (g_j, Rtube_j^2, box lo, box hi) boxes as 3 x 10-bit offsets
};
static_assert(sizeof(PieceRec) == 608, "PieceRec layout");

__device__ __forceinline__ uint32_t pack3(int a, int b, int c)
{
    return (uint32_t)a | ((uint32_t)b << 10) | ((uint32_t)c << 20);
}
__device__ __forceinline__ int unpack3(uint32_t v, int d) { return (int)((v >> (10 * d)) & 1023u); }

// ------------------------------------------------------------------------------ set-up
// pieces of every real section: ceil(ntf / kPieceMax), chords split as evenly as possible
__global__ void piece_counts_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line,
                                    int64_t nslots, const int *__restrict__ ntf, int64_t *__restrict__ poff)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const LineParam &P = lp[slot_line[s]];
    const bool real = (int)(s - P.slot_off) < P.n_sec;
    poff[s] = real ? (ntf[s] + kPieceMax - 1) / kPieceMax : 0;
}

// slot of every piece (one thread per section slot: a slot has ceil(ntf / 8) pieces, mostly 1-3)
__global__ void piece_map_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                                 const int *__restrict__ ntf, const int64_t *__restrict__ poff, int *__restrict__ map)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const LineParam &P = lp[slot_line[s]];
    if ((int)(s - P.slot_off) >= P.n_sec) return;
    const int n = (ntf[s] + kPieceMax - 1) / kPieceMax;
    const int64_t o = poff[s];
    for (int j = 0; j < n; ++j) map[o + j] = (int)s;
}

// One thread per piece: FP64 samples, chords and boxes as the sub-segment set-up
// (tube.f90:703-798), then the FP32 record in the piece's frame.  err bit 8: a piece box
// wider than 1023 points (the 10-bit chord box offsets).
constexpr int kBuildThreads = 64;   // piece_build_kernel's block: 32 KB of shared memory, six per SM
__global__ void __launch_bounds__(kBuildThreads, 6) piece_build_kernel(
    const LineParam *__restrict__ lp, const int *__restrict__ slot_line, const int *__restrict__ map, int64_t npieces,
    const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
    const double *__restrict__ cze, int64_t node_base, const double *__restrict__ coe, const int *__restrict__ ntf,
    const double *__restrict__ dtf, const int64_t *__restrict__ poff, int N, double Rtube_ratio, double dzeta_sup,
    double eta, PieceRec *__restrict__ rec, int *__restrict__ err)
{
    // the section's 18 coefficients are read by every sample evaluation of the walk: one
    // global read each into this thread's row of shared memory (rows of 19 doubles spread the
    // banks), instead of about 20 x 18 global loads that throttled the load/store unit
    __shared__ double s_cf[kBuildThreads][19];
    const int64_t pc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pc >= npieces) return;
    const int slot = map[pc];
    const LineParam P = lp[slot_line[slot]];
    const int t = slot - (int)P.slot_off;
    const int np = P.n_sec;
    const int ns = ntf[slot];
    const int npc = (ns + kPieceMax - 1) / kPieceMax;
    const int ip = (int)(pc - poff[slot]);
    const int base = ns / npc, rem = ns % npc;
    const int n = base + (ip < rem ? 1 : 0);
    const int j0 = ip * base + min(ip, rem);
    const double L = P.Len;
    const double *czl = cze + (P.node_off - node_base);
    const double zl = cze_pl_at(czl, np, t), zl1 = cze_pl_at(czl, np, t + 1);
    const double d = dtf[slot];
    double *cf = s_cf[threadIdx.x];
#pragma unroll
    for (int m = 0; m < 18; ++m) cf[m] = coe[18 * (size_t)slot + m];
    const int inext = (t + 1 < np) ? t + 1 : 0;
    // extended sample k of the section (as the sub-segment set-up: the endpoint copy and the
    // next section's first sample)
    auto sample = [&](int k, double *c3) {
        if (k < ns) {
            spl_pos_fma(cf, (zl + d * k - zl) * L, c3);
        } else if (k == ns) {
            c3[0] = X[P.node_off + inext];
            c3[1] = Y[P.node_off + inext];
            c3[2] = Z[P.node_off + inext];
        } else {
            spl_pos_fma(coe + 18 * (size_t)(slot + 1), (zl1 + dtf[slot + 1] * 1 - zl1) * L, c3);
        }
    };
    const bool const_core = P.sigma_max == P.sigma_min;
    const double inv_dx = (double)N / dev_pi2(), xstart = -dev_pi();
    const double zj0 = zl + d * j0;
    double o[3];
    sample(j0, o);
    // Walk the piece's chords j0 .. j0+n-1 and the plane after them.  visit(jj, ch, nd, pj, lo,
    // hi, s0, s1, Rt) receives chord jj (cminus of consecutive samples), the start pj of it in
    // the piece frame (o + pj is the unwrapped sample) and its box in the piece frame; for
    // jj == n only ch and pj are meaningful (the next chord's plane).
    auto walk = [&](auto &&visit) {
        double ca[3] = {o[0], o[1], o[2]}, cb[3], pj[3] = {0.0, 0.0, 0.0};
        sample(j0 + 1, cb);
        for (int jj = 0; jj <= n; ++jj) {
            const int j = j0 + jj;
            double ch[3];
            cminus3(cb, ca, ch);
            const double nd = sqrt(ch[0] * ch[0] + ch[1] * ch[1] + ch[2] * ch[2]);
            int lo3[3] = {0, 0, 0}, hi3[3] = {0, 0, 0};
            double s0 = zl + d * j, s1 = zl + d * (j + 1), Rt = 0.0;
            if (jj < n) {
                Rt = const_core ? Rtube_ratio * P.sigma_min
                                : fmax(Rtube_ratio * sigma_func(s0, P.length, P.sigma_max, P.sigma_min, P.n_T),
                                       Rtube_ratio * sigma_func(s1, P.length, P.sigma_max, P.sigma_min, P.n_T));
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    // the reference's box of this chord (mark1 on the wrapped samples,
                    // tube.f90:779-798), moved to the piece frame by the whole periods
                    // between the reference's start and o + pj
                    double a = ca[k], b = cb[k];
                    if (b - a > dev_pi()) a = a + dev_pi2();
                    else if (b - a < -dev_pi()) b = b + dev_pi2();
                    const int lo = (int)floor((fmin(a, b) - xstart - Rt) * inv_dx + 1.0);
                    const int hi = (int)ceil((fmax(a, b) - xstart + Rt) * inv_dx + 1.0);
                    const int K = (int)rint((a - (o[k] + pj[k])) * (1.0 / dev_pi2()));
                    lo3[k] = lo - K * N;
                    hi3[k] = hi - K * N;
                }
            }
            visit(jj, ch, nd, pj, lo3, hi3, s0, s1, Rt);
            if (jj == n) break;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                pj[k] += ch[k];
                ca[k] = cb[k];
            }
            sample(j + 2, cb);   // j + 2 <= j0 + n + 1 <= ntf + 1
        }
    };
    // One walk: per chord its plane (pl), its constants (chq) and its sample's z offset, and
    // the piece box (union of the chord boxes), the largest Rtube, the extent and the bend.  The
    // records' offsets depend on the piece box, so the samples' piece-frame offsets pj and the
    // chord boxes (relative to chord 0's) wait in shared memory until the walk is done.
    __shared__ double s_pj[kBuildThreads][kPieceMax + 1][3];
    __shared__ float s_zoff[kBuildThreads][kPieceMax + 1];
    __shared__ short s_box[kBuildThreads][kPieceMax][6];
    const int tid = threadIdx.x;
    PieceRec &R = rec[pc];
    int blo[3] = {1 << 30, 1 << 30, 1 << 30}, bhi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    int b0[3] = {0, 0, 0};   // chord 0's box origin: the reference of s_box
    double Rmax = 0.0, dlen = 0.0;
    float bendmin = 1.0f, Wm = 0.0f, cmax = 0.0f;
    double tprev[3] = {0.0, 0.0, 0.0};
    walk([&](int jj, const double *ch, double nd, const double *pj, const int *lo3, const int *hi3, double s0,
             double s1, double Rt) {
        const double inv = 1.0 / nd;
        const double tc[3] = {ch[0] * inv, ch[1] * inv, ch[2] * inv};
        if (jj > 0) bendmin = fminf(bendmin, (float)(tc[0] * tprev[0] + tc[1] * tprev[1] + tc[2] * tprev[2]));
        tprev[0] = tc[0];
        tprev[1] = tc[1];
        tprev[2] = tc[2];
        dlen = fmax(dlen, sqrt(pj[0] * pj[0] + pj[1] * pj[1] + pj[2] * pj[2]));
        const float ck = (float)(tc[0] * pj[0] + tc[1] * pj[1] + tc[2] * pj[2]);
        R.pl[jj] = make_float4((float)tc[0], (float)tc[1], (float)tc[2], ck);
        cmax = fmaxf(cmax, fabsf(ck));
        const float zoff = (float)((s0 - zj0) * L);
        s_zoff[tid][jj] = zoff;
#pragma unroll
        for (int k = 0; k < 3; ++k) s_pj[tid][jj][k] = pj[k];
        if (jj == n) return;
        Rmax = fmax(Rmax, Rt);
        if (jj == 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) b0[k] = lo3[k];
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            blo[k] = min(blo[k], lo3[k]);
            bhi[k] = max(bhi[k], hi3[k]);
            // within +-32767 of chord 0's origin: the piece box is checked below 1024 wide
            s_box[tid][jj][k] = (short)max(-32767, min(32767, lo3[k] - b0[k]));
            s_box[tid][jj][3 + k] = (short)max(-32767, min(32767, hi3[k] - b0[k]));
        }
        const float g = (float)((s1 - s0) * L * inv);
        R.chq[jj] = make_float4(g, (float)(Rt * Rt), 0.0f, 0.0f);
        Wm = fmaxf(Wm, (zoff + (float)(nd + Rt) * fabsf(g)) * 1.01f);
    });
    double X0[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (bhi[k] - blo[k] > 1023) atomicOr(err, 8);
        if (bhi[k] - blo[k] > kScatterMaxOff) atomicOr(err, 64);   // too wide for the scatter kernel
        R.box_lo[k] = blo[k];
        R.box_hi[k] = bhi[k];
        // mesh coordinate of the 1-based unwrapped index box_lo: (i - 1) dx + xstart
        X0[k] = dadd(dmul((double)blo[k] - 1.0, dev_pi2() / N), xstart);
        R.off[k] = (float)(X0[k] - o[k]);
    }
    R.dx = (float)(dev_pi2() / N);
    R.nch = n;
    // per sample: mesh point at box_lo minus sample jj (FP64, then FP32), the sample's own local
    // frame, as accurate as a sub-segment record's; per chord: its box relative to box_lo
    for (int jj = 0; jj <= n; ++jj) {
        float offj[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) offj[k] = (float)(X0[k] - (o[k] + s_pj[tid][jj][k]));
        R.po[jj] = make_float4(offj[0], offj[1], offj[2], s_zoff[tid][jj]);
        if (jj == n) break;
        const int sh[3] = {b0[0] - blo[0], b0[1] - blo[1], b0[2] - blo[2]};
        R.chq[jj].z = __uint_as_float(pack3(s_box[tid][jj][0] + sh[0], s_box[tid][jj][1] + sh[1], s_box[tid][jj][2] + sh[2]));
        R.chq[jj].w = __uint_as_float(pack3(s_box[tid][jj][3] + sh[0], s_box[tid][jj][4] + sh[1], s_box[tid][jj][5] + sh[2]));
    }
    // FP32 rounding of the piece-frame plane test d . tci_k - c_k: the offsets d (off, dx and
    // the fma, at most 4 u max|d_k| per axis), the normal (u |d|_1), c_k (u |c_k|) and the three
    // fused sums (u (|d|_1 + |c_k|) each) add up to 8 u (|d|_1 + |c_k|) with u = 2^-24, below
    // 5e-7 (|d|_1 + |c_k|); |d|_1 is bounded by the box corners' offsets.  The guard keeps a
    // factor of four.
    float dmax = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        dmax += fmaxf(fabsf(R.off[k]), fabsf(R.off[k] + (float)(bhi[k] - blo[k]) * R.dx));
    R.guard = 2.0e-6f * (dmax + cmax) + 1.0e-30f;
    // the section's quintic Taylor-shifted to the piece start z0 (synthetic division)
    const double z0 = (zj0 - zl) * L;
    bool nowrap = true;
    float pmax = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double a[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) a[m] = cf[6 * k + m];
#pragma unroll
        for (int r = 0; r < 5; ++r)
#pragma unroll
            for (int j = 4; j >= r; --j) a[j] = fma(z0, a[j + 1], a[j]);
#pragma unroll
        for (int r = 1; r <= 5; ++r) R.b[5 * k + r - 1] = (float)a[r];
        const double c0 = a[0];
        R.kq[k] = (int)rint((o[k] - c0) * (1.0 / dev_pi2()));
        R.thi[k] = (float)(dev_pi() - c0);
        R.tlo[k] = (float)(-dev_pi() - c0);
        const float *bb = R.b + 5 * k;
        const float pb =
            Wm * (fabsf(bb[0]) + Wm * (fabsf(bb[1]) + Wm * (fabsf(bb[2]) + Wm * (fabsf(bb[3]) + Wm * fabsf(bb[4])))));
        pmax = fmaxf(pmax, pb);
        if (R.kq[k] != 0 || !(R.thi[k] > pb * 1.01f + 1e-5f) || !(R.tlo[k] < -pb * 1.01f - 1e-5f)) nowrap = false;
    }
    // as segrec_from: every accepted point keeps |P| clear of the wrap thresholds and |x - c| < pi
    if (((float)dlen + 2.0f * (float)Rmax) * 1.7321f + pmax > 3.0f) nowrap = false;
    if (bendmin < 0.75f) nowrap = false;
    if (nowrap) R.kq[0] = kNoWrap;
    // core size sigma(zeta) = smin + A (sin(omega zeta) + 1), zeta = s_j0 + W / Len
    const double omega = floor(P.length / dev_pi() + 0.5) * (double)P.n_T;
    const double A = (P.sigma_max - P.sigma_min) / 2.0;
    R.smin = (float)P.sigma_min;
    R.A = (float)A;
    R.om = (float)(omega / L);
    if (A == 0.0) {
        R.ph0 = 0.0f;
        R.q = 0.0f;
    } else {
        R.ph0 = (float)fmod(omega * zj0, dev_pi2());
        const double h = fmin(dzeta_sup, 1.0 * d);
        R.q = (float)(A * sin(omega * h) / h);
    }
    R.Gamma = (float)P.Gamma;
    R.Linv = (float)(1.0 / L);
    R.eta = (float)eta;
    const double rt = Rtube_ratio * P.sigma_min;
    const float s2 = R.smin * R.smin;
    R.inv2s2 = 0.5f / s2;
    R.ftd = __expf(-(float)(rt * rt) * R.inv2s2);   // the same exponential as the per-point term
    R.amp = R.Gamma * (0.159154943091895336f / s2);
    R.pad1 = 0;
}

// ------------------------------------------------------------------------------ binning
// Tiles of a piece: its box, culled to the tiles that meet at least one chord's box.
template <typename F>
__device__ __forceinline__ void for_each_tile(const PieceRec &S, int N, F &&f)
{
    const int nch = S.nch;
    for_each_box_tile(S.box_lo, S.box_hi, N,
                      [&](int ox, int oy, int oz, int nx, int ny, int nz) {
                          for (int j = 0; j < nch; ++j) {
                              const uint32_t lo = __float_as_uint(S.chq[j].z), hi = __float_as_uint(S.chq[j].w);
                              if (unpack3(lo, 0) <= ox + nx - 1 && unpack3(hi, 0) >= ox && unpack3(lo, 1) <= oy + ny - 1 &&
                                  unpack3(hi, 1) >= oy && unpack3(lo, 2) <= oz + nz - 1 && unpack3(hi, 2) >= oz)
                                  return true;
                          }
                          return false;
                      },
                      f);
}

// ------------------------------------------------------------------------------ deposit
constexpr int kPChunk = 4;        // pieces staged per warp chunk: 32 chords, one per lane
constexpr int kPQueue = 64;       // accepted (point, chord) queue of a warp
static_assert(kPChunk * kPieceMax == 32, "one chord per lane");

// A piece's box clipped to the tile (one periodic image).
struct PBox {
    int lo[3];      // clipped origin, tile-local
    int n[3];       // clipped extent
    int dl[3];      // clipped origin relative to the piece's box_lo, minus lo
    int vol;
    int pad[3];
};

// Rows of one chord's box (clipped to the tile in the tile kernel, whole in the scatter kernel),
// along the axis best aligned with the chord; the box is in offsets from the piece's box origin
// (the kernels' rx, ry, rz).
constexpr int kMaxCol = 16;   // columns, and rows per column, of a per-column row table
struct ChordRows {          // lane-major (one entry per chord lane): conflict-free stores
    uint16_t o[3][32];      // box origin
    uint8_t n[3][32];       // box extent
    uint8_t axis[32], nb[32];   // walk axis; rows per column (extent along (axis+1)%3)
    uint8_t ncol[32];       // columns with their own row ranges (0: every row of the box)
    uint8_t pad[32];
    float rnb[32];          // (1 + 1e-6) / nb  (every row of the box)
    float isa[32];          // 1 / (dx n_j[axis])
    float isb[32];          // 1 / (dx n_{j+1}[axis]), 0 when |n_{j+1}[axis]| <= 0.05 (no bound from it)
    float q2[32], i2q[32];  // dx^2 (1 - n_j[axis]^2) (0: no cylinder bound) and 1 / (2 q2)
    uint16_t col[kMaxCol][32];  // column jc: first row of the column | first b offset << 12
};

// Row table of chord j of record R over the box [co, co + cnn) (piece-frame offsets, cnn > 0
// along every axis when nonempty): the walk axis (the one best aligned with the chord), the
// plane and cylinder coefficients of the row intervals, and where the chord's projected
// cylinder allows (at most kMaxCol columns of at most kMaxCol rows) per-column row ranges.
// The rows of a column (fixed offset along c = (axis+2)%3) are those inside the projection
// along the axis of the part of chord j's cylinder that the chord can accept: points
// S_j + t n + v with |v| < Rtube, v . n = 0 and 0 <= t < l + Rtube tan(theta) (theta: the
// angle between planes j and j + 1; plane j + 1 passes through S_j + l n).  That projection is
// the projected disk (semi-axes Rtube across n_bc and Rtube |n_a| along it) swept along n_bc,
// inside the disk's ellipse about the sweep's midpoint scaled by 1 + sweep / (2 minor axis).
// Writes lane `lane` of C; returns the number of rows.
__device__ __forceinline__ int chord_row_table(const PieceRec &R, int j, const int co[3], const int cnn[3],
                                               bool nonempty, ChordRows &C, int lane)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        C.o[d][lane] = (uint16_t)co[d];
        C.n[d][lane] = (uint8_t)cnn[d];
    }
    int nrows = 0;
    const float4 pj = R.pl[j], pk = R.pl[j + 1];
    const float ax = fabsf(pj.x), ay = fabsf(pj.y), az = fabsf(pj.z);
    const int a = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    C.axis[lane] = (uint8_t)a;
    const int nbv = a == 0 ? cnn[1] : (a == 1 ? cnn[2] : cnn[0]);
    const int ncv = a == 0 ? cnn[2] : (a == 1 ? cnn[0] : cnn[1]);
    C.nb[lane] = (uint8_t)nbv;
    C.rnb[lane] = nonempty ? 1.000001f / (float)nbv : 0.0f;
    const float ta = a == 0 ? pj.x : (a == 1 ? pj.y : pj.z);
    const float tb = a == 0 ? pk.x : (a == 1 ? pk.y : pk.z);
    // the bounds below carry margins of 0.05 point and 1 %: approximate reciprocals
    // (a few ulp) are ample, and the reference's tests decide every candidate
    C.isa[lane] = __fdividef(1.0f, R.dx * ta);
    C.isb[lane] = fabsf(tb) > 0.05f ? __fdividef(1.0f, R.dx * tb) : 0.0f;
    const float q2 = R.dx * R.dx * (1.0f - ta * ta);
    C.q2[lane] = q2 > 0.01f * R.dx * R.dx ? q2 : 0.0f;
    C.i2q[lane] = q2 > 0.01f * R.dx * R.dx ? __fdividef(0.5f, q2) : 0.0f;
    C.ncol[lane] = 0;
    nrows = nonempty ? nbv * ncv : 0;
    const float cth = pj.x * pk.x + pj.y * pk.y + pj.z * pk.z;
    if (nonempty && ncv <= kMaxCol && nbv <= kMaxCol && cth > 0.5f) {
        // the chord's sweep and the ellipse of its cross-section, in (b, c)
        const float4 oj = R.po[j], ok1 = R.po[j + 1];
        const float lx_ = oj.x - ok1.x, ly_ = oj.y - ok1.y, lz_ = oj.z - ok1.z;
        const float rt = sqrtf(R.chq[j].y);
        const float sweep = sqrtf(lx_ * lx_ + ly_ * ly_ + lz_ * lz_) +
                            __fdividef(rt * sqrtf(fmaxf(1.0f - cth * cth, 0.0f)), cth);
        const int b = a == 2 ? 0 : a + 1, cc = a == 0 ? 2 : a - 1;
        const float nb_ = b == 0 ? pj.x : (b == 1 ? pj.y : pj.z);
        const float nc_ = cc == 0 ? pj.x : (cc == 1 ? pj.y : pj.z);
        const float nbc = sqrtf(nb_ * nb_ + nc_ * nc_);
        const float inbc = nbc > 1e-4f ? __fdividef(1.0f, nbc) : 0.0f;
        const float wb = nbc > 1e-4f ? nb_ * inbc : 1.0f, wc = nbc > 1e-4f ? nc_ * inbc : 0.0f;
        const float Bm = rt * fabsf(ta);
        const float f = 1.0f + __fdividef(sweep * nbc, 2.0f * Bm);
        const float Ae = fmaf(f * rt, 1.01f, 0.05f * R.dx), Be = fmaf(f * Bm, 1.01f, 0.05f * R.dx);
        const float ia2 = __fdividef(1.0f, Ae * Ae), ib2 = __fdividef(1.0f, Be * Be);
        // centre: S_j + (sweep / 2) n, with S_j = -po[j] (mesh-point offsets times dx)
        const float sb = -(b == 0 ? oj.x : (b == 1 ? oj.y : oj.z)), sc = -(cc == 0 ? oj.x : (cc == 1 ? oj.y : oj.z));
        const float Cb = fmaf(0.5f * sweep, nb_, sb), Cc = fmaf(0.5f * sweep, nc_, sc);
        const int ob = b == 0 ? co[0] : (b == 1 ? co[1] : co[2]);
        const int oc = cc == 0 ? co[0] : (cc == 1 ? co[1] : co[2]);
        const float al = fmaf(wc * wc, ia2, wb * wb * ib2);
        const float cross_ = 2.0f * wb * wc * (ib2 - ia2);
        const float g2 = fmaf(wb * wb, ia2, wc * wc * ib2);
        const float i2a = __fdividef(0.5f, al);
        int rows = 0;
        const float idx = __fdividef(1.0f, R.dx);
#pragma unroll 1
        for (int jc = 0; jc < ncv; ++jc) {
            const float z = fmaf((float)(oc + jc), R.dx, -Cc);
            const float be = cross_ * z, ga = fmaf(g2 * z, z, -1.0f);
            const float disc = fmaf(be, be, -4.0f * al * ga);
            int jb0 = 0, nrow = 0;
            if (disc >= 0.0f) {
                const float sq = sqrtf(disc);
                const float y1 = (-be - sq) * i2a, y2 = (-be + sq) * i2a;
                const float u1 = fmaf(Cb + y1, idx, -(float)ob), u2 = fmaf(Cb + y2, idx, -(float)ob);
                jb0 = max(0, (int)ceilf(fmaxf(u1, -2.0f) - 0.05f));
                const int jb1 = min(nbv - 1, (int)floorf(fminf(u2, (float)nbv + 1.0f) + 0.05f));
                nrow = max(0, jb1 - jb0 + 1);
            }
            C.col[jc][lane] = (uint16_t)(rows | (jb0 << 12));
            rows += nrow;
        }
        C.ncol[lane] = (uint8_t)ncv;
        nrows = rows;
    }
    return nrows;
}

// Row rr of chord lane c (chord j of record R, row table C): the row's base point (bx, by, bz)
// (offsets from the piece's box origin), its axis a and the index interval [i, ihi] along the
// axis where the row can pass chord j's two planes and its cylinder (with a 0.05-point margin
// and Rtube^2 widened by 2e-3, far above the FP32 rounding of the bounds).
__device__ __forceinline__ void chord_row_span(const PieceRec &R, const ChordRows &C, int c, int j, int rr, int &bx,
                                               int &by, int &bz, int &a, int &i, int &ihi)
{
    a = C.axis[c];
    int jc, jb;
    if (C.ncol[c] > 0) {
        // column of row rr: last column whose first row is <= rr (ncol <= 16)
        jc = 0;
#pragma unroll
        for (int step = 8; step > 0; step >>= 1) {
            const int t = jc + step;
            if (t < C.ncol[c] && (int)(C.col[t][c] & 0xfffu) <= rr) jc = t;
        }
        jb = (int)(C.col[jc][c] >> 12) + (rr - (int)(C.col[jc][c] & 0xfffu));
    } else {
        jc = (int)((float)rr * C.rnb[c]);
        if (jc * C.nb[c] > rr) --jc;
        jb = rr - jc * C.nb[c];
    }
    bx = C.o[0][c] + (a == 0 ? 0 : (a == 1 ? jc : jb));
    by = C.o[1][c] + (a == 0 ? jb : (a == 1 ? 0 : jc));
    bz = C.o[2][c] + (a == 0 ? jc : (a == 1 ? jb : 0));
    const float4 pj = R.pl[j], pk = R.pl[j + 1], oj = R.po[j], ok1 = R.po[j + 1];
    // row base relative to sample j and to sample j + 1
    const float ex = fmaf((float)bx, R.dx, oj.x), ey = fmaf((float)by, R.dx, oj.y),
                ez = fmaf((float)bz, R.dx, oj.z);
    const float T0 = fmaf(ez, pj.z, fmaf(ey, pj.y, ex * pj.x));
    const float ta = a == 0 ? pj.x : (a == 1 ? pj.y : pj.z);
    const int na = a == 0 ? C.n[0][c] : (a == 1 ? C.n[1][c] : C.n[2][c]);
    float lo = -2.0f, hi = (float)na + 1.0f;
    const float r0f = -T0 * C.isa[c];          // t_j >= 0
    if (ta > 0.0f) lo = fmaxf(lo, r0f);
    else hi = fminf(hi, r0f);
    if (C.isb[c] != 0.0f) {                     // t_{j+1} < 0
        const float fx = fmaf((float)bx, R.dx, ok1.x), fy = fmaf((float)by, R.dx, ok1.y),
                    fz = fmaf((float)bz, R.dx, ok1.z);
        const float T1 = fmaf(fz, pk.z, fmaf(fy, pk.y, fx * pk.x));
        const float r1f = -T1 * C.isb[c];
        if (C.isb[c] > 0.0f) hi = fminf(hi, r1f);
        else lo = fmaxf(lo, r1f);
    }
    if (C.q2[c] > 0.0f) {                       // rho^2 < Rtube^2 about chord line j
        const float ea = a == 0 ? ex : (a == 1 ? ey : ez);
        const float e2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
        const float Q1 = 2.0f * R.dx * (ea - T0 * ta);
        const float Q0 = e2 - T0 * T0;
        const float R2w = fmaf(R.chq[j].y, 1.002f, 1e-6f * e2);
        const float disc = Q1 * Q1 - 4.0f * C.q2[c] * (Q0 - R2w);
        if (disc < 0.0f) {
            hi = -3.0f;
        } else {
            const float sq = sqrtf(disc);
            lo = fmaxf(lo, (-Q1 - sq) * C.i2q[c]);
            hi = fminf(hi, (-Q1 + sq) * C.i2q[c]);
        }
    }
    i = max(0, (int)ceilf(lo - 0.05f));
    ihi = min(na - 1, (int)floorf(hi + 0.05f));
}

struct PieceStage {
    PieceRec rec[kPChunk];
    PBox box[kPChunk];
    ChordRows cr;
    uint32_t cq[kPQueue];  // candidates: chord lane (piece << 3 | chord) | x << 5 | y << 9 | z << 12 (tile-local)
    uint32_t q[kPQueue];   // piece | chord << 3 | x << 6 | y << 10 | z << 13 (tile-local) | kPQDecide
    uint32_t id[kPChunk];  // global record ids of the staged pieces
    uint64_t bar;
    uint64_t pad;
};
constexpr size_t kPieceSmem = kAccBytes + sizeof(PieceStage) * kDepWarps;
constexpr uint32_t kPQDecide = 1u << 16;   // queued pair left to the reference's FP64 tests
// three blocks per SM (the register budget allows three as well): the kernel hides the
// latency of its record copies with the other blocks' warps
static_assert(3 * (kPieceSmem + 1024) <= 228 * 1024, "deposit_piece_kernel: three blocks per SM");

__device__ __forceinline__ void pclip(const PieceRec &R, uint32_t img, int N, int tx0, int ty0, int tz0, PBox &B)
{
    const int tl[3] = {tx0, ty0, tz0}, te[3] = {TX, TY, TZ};
    const int m[3] = {(int)(img % 3) - 1, (int)((img / 3) % 3) - 1, (int)(img / 9) - 1};
    bool nonempty = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int ulo = tl[d] + m[d] * N, uhi = min(tl[d] + te[d] - 1, N - 1) + m[d] * N;
        const int lo = max(ulo, R.box_lo[d] - 1), hi = min(uhi, R.box_hi[d] - 1);
        B.lo[d] = lo - ulo;
        B.n[d] = max(0, hi - lo + 1);
        B.dl[d] = (lo - (R.box_lo[d] - 1)) - B.lo[d];
        nonempty = nonempty && B.n[d] > 0;
    }
    B.vol = nonempty ? B.n[0] * B.n[1] * B.n[2] : 0;
}

// The reference's acceptance of mesh point (rx, ry, rz) (offsets from the piece's box origin)
// by chord j (tube.f90:806-818): t_j >= 0 and t_{j+1} < 0, tested in the piece frame, then the
// distance to chord line j below Rtube, in the chord's frame.  Returns 0 (rejected), 1
// (accepted) or 2: a plane test within its rounding bound (guard) of zero, which the
// reference's FP64 tests decide (the field jumps across the plane two consecutive chords
// share).  The caller keeps the point in chord j's box.
__device__ __forceinline__ int piece_classify(const PieceRec &R, int j, int rx, int ry, int rz)
{
    const float dxv = fmaf((float)rx, R.dx, R.off[0]);
    const float dyv = fmaf((float)ry, R.dx, R.off[1]);
    const float dzv = fmaf((float)rz, R.dx, R.off[2]);
    const float4 p0 = R.pl[j], p1 = R.pl[j + 1];
    const float tj = fmaf(dzv, p0.z, fmaf(dyv, p0.y, fmaf(dxv, p0.x, -p0.w)));
    const float tk = fmaf(dzv, p1.z, fmaf(dyv, p1.y, fmaf(dxv, p1.x, -p1.w)));
    if (!(tj >= -R.guard) || !(tk < R.guard)) return 0;
    const float4 cp = R.po[j];
    const float ex = fmaf((float)rx, R.dx, cp.x);
    const float ey = fmaf((float)ry, R.dx, cp.y);
    const float ez = fmaf((float)rz, R.dx, cp.z);
    const float t0 = fmaf(ez, p0.z, fmaf(ey, p0.y, ex * p0.x));
    const float r2 = fmaf(-t0, t0, fmaf(ez, ez, fmaf(ey, ey, ex * ex)));
    if (!(r2 < R.chq[j].y)) return 0;
    return (tj >= R.guard && tk < -R.guard) ? 1 : 2;
}

// The candidate test of the FP64 path: piece_classify with every test widened by far more than
// its FP32 rounding (the guard), so that every point the reference's FP64 tests accept is
// queued; the FP64 tests then decide.
__device__ __forceinline__ bool piece_accepts_wide(const PieceRec &R, int j, int rx, int ry, int rz)
{
    const float dxv = fmaf((float)rx, R.dx, R.off[0]);
    const float dyv = fmaf((float)ry, R.dx, R.off[1]);
    const float dzv = fmaf((float)rz, R.dx, R.off[2]);
    const float e = 10.0f * R.guard + 1e-3f * R.dx;
    const float4 p0 = R.pl[j], p1 = R.pl[j + 1];
    const float tj = fmaf(dzv, p0.z, fmaf(dyv, p0.y, fmaf(dxv, p0.x, -p0.w)));
    const float tk = fmaf(dzv, p1.z, fmaf(dyv, p1.y, fmaf(dxv, p1.x, -p1.w)));
    if (!(tj >= -e) || !(tk < e)) return false;
    const float4 cp = R.po[j];
    const float ex = fmaf((float)rx, R.dx, cp.x);
    const float ey = fmaf((float)ry, R.dx, cp.y);
    const float ez = fmaf((float)rz, R.dx, cp.z);
    const float t0 = fmaf(ez, p0.z, fmaf(ey, p0.y, ex * p0.x));
    const float e2 = fmaf(ez, ez, fmaf(ey, ey, ex * ex));
    const float R2 = R.chq[j].y;
    return fmaf(-t0, t0, e2) < R2 + 1e-5f * (e2 + R2) + e * e;
}

// ------------------------------------------------------------------------------ raster
// The thinnest tubes (truncation radius of a few grid spacings) accept only two or three points
// per chord, and a chord's box meets two to four tiles: searching each (tile, piece) pair's rows
// repeats the per-chord set-up in every tile for a handful of points.  Their pieces are
// therefore rasterised once, in a pass over pieces: one thread per piece walks, for each chord,
// the columns of the chord's box along the axis best aligned with the chord, bounds each column
// by the chord's two planes (0.05-point margin) and applies the deposition kernel's acceptance
// test (piece_classify; the widened test in the FP64 path) to the points in between.  A first
// pass counts the points of every piece, a scan gives each piece its offset, and a second pass
// writes them: chord | x << 3 | y << 12 | z << 21 | kRasDecide (left to the FP64 tests),
// offsets from the piece's box origin.  The
// deposition kernel then only evaluates the listed points that fall in its tile.  err bit 16:
// a chord box wider than 511 points (the 9-bit offsets).
constexpr int kRasterMaxOff = 511;
constexpr uint32_t kRasDecide = 1u << 30;

template <bool Wide, bool Write>
__global__ void __launch_bounds__(128) piece_raster_kernel(const PieceRec *__restrict__ rec, int64_t npieces,
                                                           int64_t *__restrict__ off, uint32_t *__restrict__ pts,
                                                           int *__restrict__ err)
{
    const int64_t pc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (pc >= npieces) return;
    const PieceRec &R = rec[pc];
    const int64_t o = Write ? off[pc] : 0;
    // the write pass stays inside the slots the counting pass reserved for this piece
    const int64_t cap = Write ? off[pc + 1] - o : 0;
    int64_t n = 0;
    const int nch = R.nch;
    const float dx = R.dx;
    for (int j = 0; j < nch; ++j) {
        const float4 pj = R.pl[j], pk = R.pl[j + 1];
        const uint32_t blo = __float_as_uint(R.chq[j].z), bhi = __float_as_uint(R.chq[j].w);
        int lo[3], hi[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            lo[d] = unpack3(blo, d);
            hi[d] = unpack3(bhi, d);
        }
        if (hi[0] > kRasterMaxOff || hi[1] > kRasterMaxOff || hi[2] > kRasterMaxOff) {
            atomicOr(err, 16);
            continue;
        }
        const float ax = fabsf(pj.x), ay = fabsf(pj.y), az = fabsf(pj.z);
        const int a = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
        const int b = a == 2 ? 0 : a + 1, c = a == 0 ? 2 : a - 1;
        const float ja = a == 0 ? pj.x : (a == 1 ? pj.y : pj.z);
        const float ka = a == 0 ? pk.x : (a == 1 ? pk.y : pk.z);
        const float sja = 1.0f / (dx * ja);
        const float ska = fabsf(ka) > 0.05f ? 1.0f / (dx * ka) : 0.0f;
        const int alo = a == 0 ? lo[0] : (a == 1 ? lo[1] : lo[2]);
        const int ahi = a == 0 ? hi[0] : (a == 1 ? hi[1] : hi[2]);
        const int clo = c == 0 ? lo[0] : (c == 1 ? lo[1] : lo[2]), chi = c == 0 ? hi[0] : (c == 1 ? hi[1] : hi[2]);
        const int blo_ = b == 0 ? lo[0] : (b == 1 ? lo[1] : lo[2]), bhi_ = b == 0 ? hi[0] : (b == 1 ? hi[1] : hi[2]);
        for (int ic = clo; ic <= chi; ++ic) {
            for (int ib = blo_; ib <= bhi_; ++ib) {
                // the column's point at a-offset 0, in the piece frame
                const int r0x = a == 0 ? 0 : (b == 0 ? ib : ic);
                const int r0y = a == 1 ? 0 : (b == 1 ? ib : ic);
                const int r0z = a == 2 ? 0 : (b == 2 ? ib : ic);
                const float dxv = fmaf((float)r0x, dx, R.off[0]);
                const float dyv = fmaf((float)r0y, dx, R.off[1]);
                const float dzv = fmaf((float)r0z, dx, R.off[2]);
                const float T0 = fmaf(dzv, pj.z, fmaf(dyv, pj.y, fmaf(dxv, pj.x, -pj.w)));
                // t_j(ra) = T0 + ra dx n_j[a] >= 0
                float flo = (float)alo - 0.05f, fhi = (float)ahi + 0.05f;
                const float r0 = -T0 * sja;
                if (ja > 0.0f) flo = fmaxf(flo, r0 - 0.05f);
                else fhi = fminf(fhi, r0 + 0.05f);
                if (ska != 0.0f) {   // t_{j+1}(ra) = T1 + ra dx n_{j+1}[a] < 0
                    const float T1 = fmaf(dzv, pk.z, fmaf(dyv, pk.y, fmaf(dxv, pk.x, -pk.w)));
                    const float r1 = -T1 * ska;
                    if (ka > 0.0f) fhi = fminf(fhi, r1 + 0.05f);
                    else flo = fmaxf(flo, r1 - 0.05f);
                }
                const int ilo = max(alo, (int)ceilf(flo)), ihi = min(ahi, (int)floorf(fhi));
                for (int ra = ilo; ra <= ihi; ++ra) {
                    const int rx = a == 0 ? ra : r0x, ry = a == 1 ? ra : r0y, rz = a == 2 ? ra : r0z;
                    const int cls = Wide ? (piece_accepts_wide(R, j, rx, ry, rz) ? 1 : 0) : piece_classify(R, j, rx, ry, rz);
                    if (cls == 0) continue;
                    if (Write) {
                        if (n >= cap) {
                            atomicOr(err, 32);
                            continue;
                        }
                        pts[o + n] = (uint32_t)j | ((uint32_t)rx << 3) | ((uint32_t)ry << 12) | ((uint32_t)rz << 21) |
                                     (cls == 2 ? kRasDecide : 0u);
                    }
                    ++n;
                }
            }
        }
    }
    if (!Write) off[pc] = n;
}

// Evaluate the first `cnt` queued (point, chord) pairs, one per lane, into the tile cells;
// pairs whose curved-branch amplification exceeds kRedoCond, and pairs left to the FP64 tests
// (kPQDecide), are deferred to FP64 (DeferList) instead.  In the emit-only pass nothing is
// added and only the deferred pairs are listed again.
template <bool General, bool F64>
__device__ __forceinline__ void drain_pieces(PieceStage &S, long long (*acc)[kAccN], int lane, int cnt, int &qn,
                                             unsigned &nacc, float fscale, float fmaxq, int *__restrict__ err,
                                             const RedoCtx &redo, const DeferList &D, int x0, int y0, int z0)
{
    bool flag = false, ok64 = false, counted = false;
    uint32_t rrec = 0;
    int lx = 0, ly = 0, lz = 0;
    if (F64 && lane < cnt) {
        // FP64 path: the candidate passed the widened FP32 tests; the reference's FP64 tests
        // decide, at the point's index in the chord's own box (the piece frame differs from it by
        // whole periods)
        const uint32_t e = S.q[lane];
        const int k = (int)(e & 7u), j = (int)((e >> 3) & 7u);
        lx = (int)((e >> 6) & 15u), ly = (int)((e >> 10) & 7u), lz = (int)((e >> 13) & 7u);
        const PBox &B = S.box[k];
        const PieceRec &R = S.rec[k];
        int slot, jj;
        redo_locate(redo, S.id[k] & ((1u << 26) - 1u), j, slot, jj);
        const int64_t q = redo.qoff[slot] + jj;
        const int *blo = redo.seg[q].box_lo;
        ok64 = eval_pair_f64(redo, q, box_index(R.box_lo[0] + lx + B.dl[0], blo[0], redo.N),
                      box_index(R.box_lo[1] + ly + B.dl[1], blo[1], redo.N),
                      box_index(R.box_lo[2] + lz + B.dl[2], blo[2], redo.N),
                      reinterpret_cast<double(*)[kAccN]>(acc), lx + kSY * ly + kSZ * lz);
    } else if (lane < cnt) {
        const uint32_t e = S.q[lane];
        const int k = (int)(e & 7u), j = (int)((e >> 3) & 7u);
        lx = (int)((e >> 6) & 15u), ly = (int)((e >> 10) & 7u), lz = (int)((e >> 13) & 7u);
        if (e & kPQDecide) {
            flag = true;
            rrec = (S.id[k] & ((1u << 26) - 1u)) | ((uint32_t)j << 26) | kDeferDecide;
        } else if (General || !D.emit_only) {
            counted = true;
            const PBox &B = S.box[k];
            const PieceRec &R = S.rec[k];
            const float4 cp = R.po[j], cq = R.chq[j], pn = R.pl[j];
            const float ex = fmaf((float)(lx + B.dl[0]), R.dx, cp.x);
            const float ey = fmaf((float)(ly + B.dl[1]), R.dx, cp.y);
            const float ez = fmaf((float)(lz + B.dl[2]), R.dx, cp.z);
            const float t0 = fmaf(ez, pn.z, fmaf(ey, pn.y, ex * pn.x));
            float vv[3], cond;
            vort_w<General, true>(R, ex, ey, ez, cp.w, t0 * cq.x, cq.y, vv, cond);
            const int p = lx + kSY * ly + kSZ * lz;
            flag = General && !(cond <= kRedoCond);
            if (flag) {
                rrec = (S.id[k] & ((1u << 26) - 1u)) | ((uint32_t)j << 26);
            } else if (!D.emit_only) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float sv = vv[d] * fscale;
                    if (!(fabsf(sv) < fmaxq)) {
                        atomicOr(err, 4);
                        sv = sv != sv ? 0.0f : copysignf(fmaxq, sv);
                    }
                    atomicAdd((unsigned long long *)&acc[d][p], (unsigned long long)__float2ll_rn(sv));
                }
            }
        }
    }
    if constexpr (F64) {
        nacc += __popc(__ballot_sync(0xffffffffu, ok64));
    } else {
        nacc += __popc(__ballot_sync(0xffffffffu, counted));
        defer_push(D, lane, flag, rrec, x0 + lx, y0 + ly, z0 + lz);
    }
    __syncwarp();
    const int rem = qn - cnt;
    const uint32_t keep = lane < rem ? S.q[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rem) S.q[lane] = keep;
    __syncwarp();
    qn = rem;
}

// Test the first `cnt` candidate points, one per lane (piece_classify), queue the accepted
// (point, chord) pairs and those left to the FP64 tests, drop the candidates and evaluate the
// queue when it holds 32 pairs.
template <bool General, bool F64>
__device__ __forceinline__ void test_candidates(PieceStage &S, long long (*acc)[kAccN], int lane, int cnt, int &cn,
                                                int &qn, unsigned &nacc, float fscale, float fmaxq,
                                                int *__restrict__ err, const RedoCtx &redo, const DeferList &D, int x0,
                                                int y0, int z0)
{
    bool ok = false;
    uint32_t code = 0u;
    if (lane < cnt) {
        const uint32_t e = S.cq[lane];
        const int c = (int)(e & 31u), k = c >> 3, j = c & 7;
        const int lx = (int)((e >> 5) & 15u), ly = (int)((e >> 9) & 7u), lz = (int)(e >> 12);
        const PBox &B = S.box[k];
        const int cls = F64 ? (piece_accepts_wide(S.rec[k], j, lx + B.dl[0], ly + B.dl[1], lz + B.dl[2]) ? 1 : 0)
                            : piece_classify(S.rec[k], j, lx + B.dl[0], ly + B.dl[1], lz + B.dl[2]);
        ok = cls != 0;
        code = (uint32_t)k | ((uint32_t)j << 3) | ((uint32_t)lx << 6) | ((uint32_t)ly << 10) | ((uint32_t)lz << 13) |
               (cls == 2 ? kPQDecide : 0u);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) S.q[qn + __popc(bal & ((1u << lane) - 1u))] = code;
    qn += __popc(bal);
    const int rem = cn - cnt;
    const uint32_t keep = lane < rem ? S.cq[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rem) S.cq[lane] = keep;
    __syncwarp();
    cn = rem;
    if (qn >= 32) drain_pieces<General, F64>(S, acc, lane, 32, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
}

// One CTA per tile.  Each warp claims chunks of kPChunk pieces (32 chords), stages their
// records with one bulk asynchronous copy each, then walks the rows of the chords' boxes within
// the tile, one row per lane: the row's candidate interval, then per candidate point the
// reference's tests (tube.f90:793-818: t_j >= 0, t_{j+1} < 0, distance to chord line j below
// Rtube) with the plane tests in the piece frame; within the rounding bound of a plane the
// reference's FP64 tests decide.  Accepted pairs are queued and evaluated 32 at a time.
template <bool General, bool Accumulate, bool F64, bool Raster>
__global__ void __launch_bounds__(kDepThreads, F64 ? 2 : 3) deposit_piece_kernel(
    const PieceRec *__restrict__ rec, int N, int ntx, int nty, int tz0, const int64_t *__restrict__ tile_off,
    const uint32_t *__restrict__ list, double scale, void *__restrict__ wx, void *__restrict__ wy,
    void *__restrict__ wz, int *__restrict__ err, const RedoCtx redo, const DeferList D,
    const int64_t *__restrict__ ras_off, const uint32_t *__restrict__ ras_pts)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    long long(*acc)[kAccN] = reinterpret_cast<long long(*)[kAccN]>(dsm);
    const int tile = (int)D.w0 + blockIdx.x;
    const int64_t c0 = tile_off[tile], c1 = tile_off[tile + 1];
    // a tile that no record of this batch meets keeps its values: earlier batches wrote them,
    // or the field was cleared before the first
    if (c0 == c1) return;
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tz0 + tile / (ntx * nty);
    const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
    // the context's planes: the whole grid, or its z-slab
    const int zs = redo.zs, zlim = redo.zs + redo.nz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PieceStage &S = reinterpret_cast<PieceStage *>(dsm + kAccBytes)[warp];
    if (lane == 0) mbar_init(&S.bar);
    // chunks are handed out through a shared counter: a warp that finishes early takes the
    // next one, so the warps of a tile end close together at the epilogue's barrier
    __shared__ int next_chunk;
    if (threadIdx.x == 0) next_chunk = kDepWarps;
    if constexpr (F64)
        tile_acc_init_f64<Accumulate>(reinterpret_cast<double(*)[kAccN]>(acc), N, x0, y0, z0, zs, zlim, (const double *)wx,
                                      (const double *)wy, (const double *)wz);
    else if (!D.emit_only)
        tile_acc_init<Accumulate>(acc, N, x0, y0, z0, zs, zlim, scale, (const float *)wx, (const float *)wy,
                                  (const float *)wz);
    __syncthreads();

    const int nchunks = (int)((c1 - c0 + kPChunk - 1) / kPChunk);
    const float fscale = (float)scale;
    const float fmaxq = 4.0e18f;
    uint32_t phase = 0;
    bool failed = false;
    int qn = 0;
    unsigned nacc = 0;   // pairs evaluated by this warp (warp-uniform)
    for (int ch = warp; ch < nchunks && !failed;) {
        const int64_t base = c0 + (int64_t)ch * kPChunk;
        const int nc = (c1 - base < kPChunk) ? (int)(c1 - base) : kPChunk;
        const uint32_t v = lane < nc ? __ldg(list + base + lane) : 0u;
        if (lane < nc) S.id[lane] = v;
        if (lane == 0) mbar_expect(&S.bar, (uint32_t)(nc * sizeof(PieceRec)));
        __syncwarp();
        if (lane < nc) bulk_g2s(&S.rec[lane], rec + (v & ((1u << 26) - 1u)), (uint32_t)sizeof(PieceRec), &S.bar);
        if (!mbar_wait(&S.bar, phase)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        if (lane < nc) {
            PBox B;
            pclip(S.rec[lane], v >> 26, N, x0, y0, z0, B);
            S.box[lane] = B;
        }
        __syncwarp();
        if constexpr (Raster) {
            // the staged pieces' rasterised points (piece_raster_kernel) that lie in this tile,
            // flattened over the pieces, one per lane
            int64_t p0 = 0, pn = 0;
            if (lane < nc) {
                const uint32_t id = v & ((1u << 26) - 1u);
                p0 = ras_off[id];
                pn = S.box[lane].vol > 0 ? ras_off[id + 1] - p0 : 0;
            }
            int64_t start[kPChunk], pbase[kPChunk], total = 0;
#pragma unroll
            for (int k = 0; k < kPChunk; ++k) {
                start[k] = total;
                pbase[k] = __shfl_sync(0xffffffffu, p0, k);
                total += __shfl_sync(0xffffffffu, pn, k);
            }
            for (int64_t t0 = 0; t0 < total; t0 += 32) {
                const int64_t t = t0 + lane;
                bool ok = false;
                uint32_t code = 0u;
                if (t < total) {
                    int k = 0;
#pragma unroll
                    for (int kk = 1; kk < kPChunk; ++kk)
                        if (kk < nc && t >= start[kk]) k = kk;
                    const uint32_t e = __ldg(ras_pts + pbase[k] + (t - start[k]));
                    const int j = (int)(e & 7u);
                    const PBox &B = S.box[k];
                    const int lx = (int)((e >> 3) & 511u) - B.dl[0], ly = (int)((e >> 12) & 511u) - B.dl[1],
                              lz = (int)((e >> 21) & 511u) - B.dl[2];
                    ok = lx >= B.lo[0] && lx < B.lo[0] + B.n[0] && ly >= B.lo[1] && ly < B.lo[1] + B.n[1] &&
                         lz >= B.lo[2] && lz < B.lo[2] + B.n[2];
                    code = (uint32_t)k | ((uint32_t)j << 3) | ((uint32_t)lx << 6) | ((uint32_t)ly << 10) |
                           ((uint32_t)lz << 13) | ((e & kRasDecide) ? kPQDecide : 0u);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) S.q[qn + __popc(bal & ((1u << lane) - 1u))] = code;
                qn += __popc(bal);
                __syncwarp();
                if (qn >= 32)
                    drain_pieces<General, F64>(S, acc, lane, 32, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
            }
        } else {
            // lane = (piece k, chord j): chord j's box clipped to the tile and its rows
            int nrows = 0;
            {
                const int k = lane >> 3, j = lane & 7;
                if (k < nc && j < S.rec[k].nch && S.box[k].vol > 0) {
                    const PieceRec &R = S.rec[k];
                    const PBox &B = S.box[k];
                    const uint32_t blo = __float_as_uint(R.chq[j].z), bhi = __float_as_uint(R.chq[j].w);
                    ChordRows &C = S.cr;
                    bool nonempty = true;
                    int co[3], cnn[3];
    #pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const int tlo = B.lo[d] + B.dl[d], thi = tlo + B.n[d] - 1;   // the tile part of the piece box
                        const int lo = max(tlo, unpack3(blo, d)), hi = min(thi, unpack3(bhi, d));
                        co[d] = lo;
                        cnn[d] = max(0, hi - lo + 1);
                        nonempty = nonempty && cnn[d] > 0;
                    }
                    nrows = chord_row_table(R, j, co, cnn, nonempty, C, lane);
                }
            }
            int incl = nrows;
    #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int roff = incl - nrows;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            __syncwarp();
            // Rows, one per lane: the index interval where the row can pass chord j's two planes
            // and its cylinder (with a 0.05-point margin and Rtube^2 widened by 2e-3, far above the
            // FP32 rounding of the bounds); its points join the candidate queue, which is tested
            // 32 at a time.
            int cn = 0;   // queued candidates (warp-uniform)
            for (int r0 = 0; r0 < total; r0 += 32) {
                const int r = r0 + lane;
                int c = 0;   // chord lane of row r: last lane whose first row is <= r
    #pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int t = c + step;
                    const int ot = __shfl_sync(0xffffffffu, roff, t);
                    if (ot <= r) c = t;
                }
                const int rc = __shfl_sync(0xffffffffu, roff, c);
                int i = 1, ihi = 0, a = 0, lx = 0, ly = 0, lz = 0;
                if (r < total) {
                    const int k = c >> 3, j = c & 7;
                    const ChordRows &C = S.cr;
                    const PieceRec &R = S.rec[k];
                    const PBox &B = S.box[k];
                    int bx, by, bz;
                    chord_row_span(R, C, c, j, r - rc, bx, by, bz, a, i, ihi);
                    lx = bx - B.dl[0];
                    ly = by - B.dl[1];
                    lz = bz - B.dl[2];
                }
                while (__any_sync(0xffffffffu, i <= ihi)) {
                    const bool has = i <= ihi;
                    uint32_t code = 0u;
                    if (has) {
                        code = (uint32_t)c | ((uint32_t)(lx + (a == 0 ? i : 0)) << 5) |
                               ((uint32_t)(ly + (a == 1 ? i : 0)) << 9) | ((uint32_t)(lz + (a == 2 ? i : 0)) << 12);
                        ++i;
                    }
                    const unsigned bal = __ballot_sync(0xffffffffu, has);
                    if (has) S.cq[cn + __popc(bal & ((1u << lane) - 1u))] = code;
                    cn += __popc(bal);
                    __syncwarp();
                    if (cn >= 32) test_candidates<General, F64>(S, acc, lane, 32, cn, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
                }
            }
            if (cn > 0) test_candidates<General, F64>(S, acc, lane, cn, cn, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
        }
        if (qn > 0) drain_pieces<General, F64>(S, acc, lane, qn, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
        __syncwarp();   // the warp's stage is reused by its next chunk
        int nxt = 0;
        if (lane == 0) nxt = atomicAdd(&next_chunk, 1);
        ch = __shfl_sync(0xffffffffu, nxt, 0);
    }
    if (failed && lane == 0) atomicOr(err, 2);
    if (lane == 0 && redo.tally && !D.emit_only) atomicAdd(redo.tally, (unsigned long long)nacc);
    __syncthreads();
    if constexpr (F64)
        tile_epilogue_f64(reinterpret_cast<double(*)[kAccN]>(acc), N, x0, y0, z0, zs, zlim, (double *)wx, (double *)wy,
                          (double *)wz);
    else if (!D.emit_only)
        tile_epilogue(acc, N, x0, y0, z0, zs, zlim, scale, (float *)wx, (float *)wy, (float *)wz);
}

// ------------------------------------------------------------------------------ scatter
// Thin tubes without tiles.  The tile kernels pay, for every (tile, piece) pair, a record copy
// and every chord's set-up within that tile; a thin chord accepts a few points and its box
// meets two to six tiles, so that overhead outweighs the evaluations.  The scatter kernel takes
// each piece once: a warp stages kPChunk pieces (32 chords, one per lane), each lane builds its
// chord's row table over the chord's whole box (chord_row_table), the rows are spread over the
// lanes (chord_row_span), their candidates tested 32 at a time (piece_classify) and the accepted
// pairs evaluated 32 at a time; each contribution is added as int64 fixed point into the side
// accumulator with global reductions.  Integer sums do not depend on the order, so the field is
// deterministic; side_fold adds the sums into omega after the batch loop.  Pairs for the FP64
// tests or arithmetic are deferred as in the tile kernels.
constexpr int kScatterWarps = 8;
constexpr uint32_t kSQDecide = 1u << 31;     // queued pair left to the reference's FP64 tests
struct ScatterStage {
    PieceRec rec[kPChunk];
    ChordRows cr;
    uint32_t cq[kPQueue];   // candidates: chord lane | x << 5 | y << 13 | z << 21 (offsets from the piece's box origin)
    uint32_t q[kPQueue];    // accepted pairs: the same | kSQDecide
};
constexpr size_t kScatterSmem = sizeof(ScatterStage) * kScatterWarps;

// Test the first cnt candidates (piece_classify), queue the accepted pairs and those left to
// the FP64 tests, and drop the candidates.
__device__ __forceinline__ void scatter_test(ScatterStage &S, int lane, int cnt, int &cn, int &qn)
{
    bool ok = false;
    uint32_t code = 0u;
    if (lane < cnt) {
        const uint32_t e = S.cq[lane];
        const int c = (int)(e & 31u);
        const int cls = piece_classify(S.rec[c >> 3], c & 7, (int)((e >> 5) & 255u), (int)((e >> 13) & 255u),
                                       (int)((e >> 21) & 255u));
        ok = cls != 0;
        code = e | (cls == 2 ? kSQDecide : 0u);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, ok);
    if (ok) S.q[qn + __popc(bal & ((1u << lane) - 1u))] = code;
    qn += __popc(bal);
    const int rem = cn - cnt;
    const uint32_t keep = lane < rem ? S.cq[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rem) S.cq[lane] = keep;
    __syncwarp();
    cn = rem;
}

// Evaluate the first cnt queued pairs, one per lane, and add them into the side accumulator;
// the pairs left to FP64 (kSQDecide, or a curved-branch amplification above kRedoCond) are
// deferred.  Points outside the context's planes (a z-slab context) are dropped.
template <bool General>
__device__ __forceinline__ void scatter_drain(ScatterStage &S, int lane, int cnt, int &qn, int64_t p0, int N, int zs,
                                              int nz, float fscale, unsigned long long *__restrict__ side,
                                              int *__restrict__ err, const DeferList &D, unsigned long long &nacc)
{
    bool flag = false, counted = false;
    uint32_t rrec = 0;
    int gx = 0, gy = 0, gz = 0;
    if (lane < cnt) {
        const uint32_t e = S.q[lane];
        const int c = (int)(e & 31u), k = c >> 3, j = c & 7;
        const int rx = (int)((e >> 5) & 255u), ry = (int)((e >> 13) & 255u), rz = (int)((e >> 21) & 255u);
        const PieceRec &R = S.rec[k];
        // unwrapped 0-based indices lie within one period of the domain (checked with the chord
        // boxes): one conditional shift wraps them, no integer division
        gx = R.box_lo[0] - 1 + rx;
        gy = R.box_lo[1] - 1 + ry;
        gz = R.box_lo[2] - 1 + rz;
        gx += gx < 0 ? N : (gx >= N ? -N : 0);
        gy += gy < 0 ? N : (gy >= N ? -N : 0);
        gz += gz < 0 ? N : (gz >= N ? -N : 0);
        const bool inslab = gz >= zs && gz < zs + nz;
        const uint32_t id = ((uint32_t)(p0 + k) & ((1u << 26) - 1u)) | ((uint32_t)j << 26);
        if (inslab && (e & kSQDecide)) {
            flag = true;
            rrec = id | kDeferDecide;
        } else if (inslab && (General || !D.emit_only)) {
            counted = true;
            const float4 cp = R.po[j], cq = R.chq[j], pn = R.pl[j];
            const float ex = fmaf((float)rx, R.dx, cp.x);
            const float ey = fmaf((float)ry, R.dx, cp.y);
            const float ez = fmaf((float)rz, R.dx, cp.z);
            const float t0 = fmaf(ez, pn.z, fmaf(ey, pn.y, ex * pn.x));
            float vv[3], cond;
            vort_w<General, true>(R, ex, ey, ez, cp.w, t0 * cq.x, cq.y, vv, cond);
            flag = General && !(cond <= kRedoCond);
            if (flag) {
                rrec = id;
            } else if (!D.emit_only) {
                const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * (size_t)(gz - zs));
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float sv = vv[d] * fscale;
                    if (!(fabsf(sv) < 4.0e18f)) {
                        atomicOr(err, 4);
                        sv = sv != sv ? 0.0f : copysignf(4.0e18f, sv);
                    }
                    atomicAdd(side + kSideStride * g + d, (unsigned long long)__float2ll_rn(sv));
                }
            }
        }
    }
    nacc += (unsigned long long)__popc(__ballot_sync(0xffffffffu, counted));
    defer_push(D, lane, flag, rrec, gx, gy, gz);
    __syncwarp();
    const int rem = qn - cnt;
    const uint32_t keep = lane < rem ? S.q[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rem) S.q[lane] = keep;
    __syncwarp();
    qn = rem;
}

template <bool General>
__global__ void __launch_bounds__(kScatterWarps * 32, 3) scatter_piece_kernel(
    const PieceRec *__restrict__ rec, int64_t npieces, int N, int zs, int nz, float fscale,
    unsigned long long *__restrict__ side, int *__restrict__ err, const DeferList D,
    unsigned long long *__restrict__ tally)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    ScatterStage &S = reinterpret_cast<ScatterStage *>(dsm)[warp];
    const int64_t nchunks = (npieces + kPChunk - 1) / kPChunk;
    const int64_t nw = (int64_t)gridDim.x * kScatterWarps;
    unsigned long long nacc = 0;   // pairs evaluated by this warp (warp-uniform)
    const int64_t chend = min(nchunks, (int64_t)D.w1);
    for (int64_t ch = (int64_t)D.w0 + (int64_t)blockIdx.x * kScatterWarps + warp; ch < chend; ch += nw) {
        const int64_t p0 = ch * kPChunk;
        const int nc = (int)min((int64_t)kPChunk, npieces - p0);
        {   // stage the chunk's records: coalesced 16-byte loads
            const uint4 *src = reinterpret_cast<const uint4 *>(rec + p0);
            uint4 *dst = reinterpret_cast<uint4 *>(S.rec);
            const int n16 = nc * (int)(sizeof(PieceRec) / 16);
            for (int t = lane; t < n16; t += 32) dst[t] = __ldg(src + t);
        }
        __syncwarp();
        // lane = (piece k, chord j): the chord's whole box and its rows
        int nrows = 0;
        {
            const int k = lane >> 3, j = lane & 7;
            if (k < nc && j < S.rec[k].nch) {
                const PieceRec &R = S.rec[k];
                const uint32_t blo = __float_as_uint(R.chq[j].z), bhi = __float_as_uint(R.chq[j].w);
                int co[3], cnn[3];
                bool nonempty = true, fits = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    co[d] = unpack3(blo, d);
                    const int hi = unpack3(bhi, d);
                    cnn[d] = max(0, hi - co[d] + 1);
                    nonempty = nonempty && cnn[d] > 0;
                    // 8-bit offsets, and unwrapped indices within one period of the domain
                    const int u0 = R.box_lo[d] - 1 + co[d], u1 = R.box_lo[d] - 1 + hi;
                    fits = fits && hi <= kScatterMaxOff && u0 >= -N && u1 < 2 * N;
                }
                if (!fits) {   // the host sends only pieces whose boxes fit: never expected
                    atomicOr(err, 64);
                    nonempty = false;
                }
                nrows = chord_row_table(R, j, co, cnn, nonempty, S.cr, lane);
            }
        }
        int incl = nrows;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int roff = incl - nrows;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        __syncwarp();
        int cn = 0, qn = 0;   // queued candidates and pairs (warp-uniform)
        for (int r0 = 0; r0 < total; r0 += 32) {
            const int r = r0 + lane;
            int c = 0;   // chord lane of row r: last lane whose first row is <= r
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int t = c + step;
                const int ot = __shfl_sync(0xffffffffu, roff, t);
                if (ot <= r) c = t;
            }
            const int rc = __shfl_sync(0xffffffffu, roff, c);
            int i = 1, ihi = 0, a = 0, bx = 0, by = 0, bz = 0;
            if (r < total) chord_row_span(S.rec[c >> 3], S.cr, c, c & 7, r - rc, bx, by, bz, a, i, ihi);
            while (__any_sync(0xffffffffu, i <= ihi)) {
                const bool has = i <= ihi;
                uint32_t code = 0u;
                if (has) {
                    code = (uint32_t)c | ((uint32_t)(bx + (a == 0 ? i : 0)) << 5) |
                           ((uint32_t)(by + (a == 1 ? i : 0)) << 13) | ((uint32_t)(bz + (a == 2 ? i : 0)) << 21);
                    ++i;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, has);
                if (has) S.cq[cn + __popc(bal & ((1u << lane) - 1u))] = code;
                cn += __popc(bal);
                __syncwarp();
                if (cn >= 32) {
                    scatter_test(S, lane, 32, cn, qn);
                    if (qn >= 32) scatter_drain<General>(S, lane, 32, qn, p0, N, zs, nz, fscale, side, err, D, nacc);
                }
            }
        }
        while (cn > 0) {
            scatter_test(S, lane, min(cn, 32), cn, qn);
            if (qn >= 32) scatter_drain<General>(S, lane, 32, qn, p0, N, zs, nz, fscale, side, err, D, nacc);
        }
        while (qn > 0) scatter_drain<General>(S, lane, min(qn, 32), qn, p0, N, zs, nz, fscale, side, err, D, nacc);
        __syncwarp();   // the warp's stage is reused by its next chunk
    }
    if (lane == 0 && tally && !D.emit_only && nacc) atomicAdd(tally, nacc);
}

// ------------------------------------------------------------------------------ host
int piece_raster(Ctx *c, CenterlineBatch &B, int *d_err);

// Set-up of the batch's pieces (after the section pass of centerline_setup).
int piece_setup(Ctx *c, CenterlineBatch &B)
{
    Ctx &C = *c;
    const int64_t slots = B.nslots;
    FWT_TRY(buf_reserve(c, C.scratch[14], sizeof(int64_t) * (size_t)(slots + 1) + 64));
    int64_t *d_poff = (int64_t *)C.scratch[14].p;
    int *d_err = (int *)(d_poff + slots + 1);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    int km = kt_begin(c, KT_CENTERLINE);
    piece_counts_kernel<<<(unsigned)((slots + 255) / 256), 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf,
                                                                                 d_poff);
    FWT_TRY(scan_exclusive_i64(c, d_poff, slots, d_poff + slots, C.scratch[12]));
    kt_end(c, km);
    int64_t np_ = 0;
    FWT_CUDA(cudaMemcpyAsync(&np_, d_poff + slots, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    B.npieces = np_;
    FWT_TRY(buf_reserve(c, C.scratch[15], sizeof(int) * (size_t)std::max<int64_t>(np_, 1)));
    FWT_TRY(buf_reserve(c, C.scratch[18], sizeof(PieceRec) * (size_t)std::max<int64_t>(np_, 1)));
    int *d_map = (int *)C.scratch[15].p;
    B.piece = (PieceRec *)C.scratch[18].p;
    B.rec_map = d_map;
    B.rec_first = d_poff;
    km = kt_begin(c, KT_CENTERLINE);
    piece_map_kernel<<<(unsigned)((slots + 255) / 256), 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf,
                                                                              d_poff, d_map);
    if (np_ > 0)
        piece_build_kernel<<<(unsigned)((np_ + kBuildThreads - 1) / kBuildThreads), kBuildThreads, 0, c->stream>>>(
            B.lp, B.slot_line, d_map, np_, c->d_x, c->d_y, c->d_z, B.cze, B.node_base, B.coe, B.ntf, B.dtf, d_poff,
            c->p.N, c->p.Rtube_ratio, c->p.dzeta_sup, c->p.eta_t, B.piece, d_err);
    kt_end(c, km);
    c->launches += 5;
    FWT_CUDA(cudaGetLastError());
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 8) return fail(FWT_E_RANGE, "piece box wider than 1023 grid points");
    if (herr & 64) B.scatter = false;   // a piece too wide for the scatter kernel's offsets
    if (B.scatter) B.raster = false;
    if (B.raster && np_ > 0) FWT_TRY(piece_raster(c, B, d_err));
    return 0;
}

// Rasterise the batch's pieces (piece_raster_kernel): count, scan, write.  A batch whose chord
// boxes exceed the 9-bit offsets, or whose point list would exceed the memory budget, is
// deposited by the row search instead (B.raster = false).
int piece_raster(Ctx *c, CenterlineBatch &B, int *d_err)
{
    Ctx &C = *c;
    const int64_t np_ = B.npieces;
    const bool wide = c->p.precision == 64;
    FWT_TRY(buf_reserve(c, C.scratch[25], sizeof(int64_t) * (size_t)(np_ + 1)));
    int64_t *d_off = (int64_t *)C.scratch[25].p;
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const unsigned g = (unsigned)((np_ + 127) / 128);
    int km = kt_begin(c, KT_CENTERLINE);
    if (wide) piece_raster_kernel<true, false><<<g, 128, 0, c->stream>>>(B.piece, np_, d_off, nullptr, d_err);
    else piece_raster_kernel<false, false><<<g, 128, 0, c->stream>>>(B.piece, np_, d_off, nullptr, d_err);
    FWT_TRY(scan_exclusive_i64(c, d_off, np_, d_off + np_, C.scratch[12]));
    kt_end(c, km);
    int64_t total = 0;
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&total, d_off + np_, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    const int64_t budget = (int64_t)1 << 32;   // points (16 GB of codes)
    if ((herr & 16) || total > budget) {
        B.raster = false;
        return 0;
    }
    FWT_TRY(buf_reserve(c, C.scratch[26], sizeof(uint32_t) * (size_t)std::max<int64_t>(total, 1)));
    uint32_t *d_pts = (uint32_t *)C.scratch[26].p;
    km = kt_begin(c, KT_CENTERLINE);
    if (wide) piece_raster_kernel<true, true><<<g, 128, 0, c->stream>>>(B.piece, np_, d_off, d_pts, d_err);
    else piece_raster_kernel<false, true><<<g, 128, 0, c->stream>>>(B.piece, np_, d_off, d_pts, d_err);
    kt_end(c, km);
    c->launches += 5;
    FWT_CUDA(cudaGetLastError());
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 32) return fail(FWT_E_STATE, "piece raster: the two passes disagreed on a piece's points");
    B.ras_off = d_off;
    B.ras_pts = d_pts;
    return 0;
}

int launch_piece(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out)
{
    const int N = c->p.N;
    const int ntx = (N + TX - 1) / TX, nty = (N + TY - 1) / TY;
    // tiles of the context's planes: the whole grid, or its z-slab (whole tiles)
    const int tz0 = c->slab_nz ? c->slab_z0 / TZ : 0;
    const int ntz = c->slab_nz ? c->slab_nz / TZ : (N + TZ - 1) / TZ;
    const int64_t ntiles = (int64_t)ntx * nty * ntz;
    const int64_t nrec = B.npieces;
    if (nrec >= ((int64_t)1 << 26)) return fail(FWT_E_RANGE, "piece batch exceeds 2^26");
    Ctx &C = *c;
    FWT_TRY(buf_reserve(c, C.scratch[20], sizeof(int64_t) * (size_t)(nrec + 2) + 64));
    int64_t *d_cnt = (int64_t *)C.scratch[20].p;
    int *d_err = (int *)(d_cnt + nrec + 1);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const unsigned bq = (unsigned)((nrec + 255) / 256);
    int km = kt_begin(c, KT_BINNING);
    if (nrec > 0) pair_count_kernel<PieceRec><<<bq, 256, 0, c->stream>>>(B.piece, nrec, N, tz0, ntz, d_cnt, d_err);
    FWT_TRY(scan_exclusive_i64(c, d_cnt, nrec, d_cnt + nrec, C.scratch[12]));
    kt_end(c, km);
    int64_t npairs = 0;
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&npairs, d_cnt + nrec, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr) return fail(FWT_E_RANGE, "piece box wider than one periodic image (Rtube too large)");
    *pairs_out = npairs;
    FWT_TRY(buf_reserve(c, C.scratch[21], sizeof(uint32_t) * 2 * (size_t)std::max<int64_t>(npairs, 1)));
    uint32_t *d_key = (uint32_t *)C.scratch[21].p, *d_val = d_key + npairs;
    const size_t tb = sizeof(uint32_t) * (size_t)ntiles;
    FWT_TRY(buf_reserve(c, C.scratch[22], tb * 2 + sizeof(int64_t) * (size_t)(ntiles + 1) + 64));
    uint32_t *d_tcnt = (uint32_t *)C.scratch[22].p, *d_cur = d_tcnt + ntiles;
    int64_t *d_toff = (int64_t *)(((uintptr_t)(d_cur + ntiles) + 15) & ~(uintptr_t)15);
    FWT_CUDA(cudaMemsetAsync(d_tcnt, 0, tb * 2, c->stream));
    km = kt_begin(c, KT_BINNING);
    if (nrec > 0)
        pair_emit_kernel<PieceRec><<<bq, 256, 0, c->stream>>>(B.piece, nrec, N, ntx, nty, tz0, ntz, d_cnt, d_key, d_val,
                                                                d_tcnt);
    u32_to_i64_kernel<<<(unsigned)((ntiles + 255) / 256), 256, 0, c->stream>>>(d_tcnt, ntiles, d_toff);
    FWT_TRY(scan_exclusive_i64(c, d_toff, ntiles, d_toff + ntiles, C.scratch[13]));
    FWT_TRY(buf_reserve(c, C.scratch[23], sizeof(uint32_t) * (size_t)(npairs + 8)));
    uint32_t *d_list = (uint32_t *)C.scratch[23].p;
    if (npairs > 0)
        tile_scatter_kernel<<<(unsigned)((npairs + 255) / 256), 256, 0, c->stream>>>(d_key, d_val, npairs, d_toff,
                                                                                     d_cur, d_list);
    kt_end(c, km);
    c->launches += 5;
    FWT_CUDA(cudaGetLastError());
    if (std::getenv("FWT_SYNC_CHECK")) {
        int64_t emitted = 0;
        FWT_CUDA(cudaMemcpyAsync(&emitted, d_toff + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
        if (emitted != npairs)
            std::fprintf(stderr, "libfwt: binning emitted %lld of %lld pairs\n", (long long)emitted, (long long)npairs);
    }

    const size_t n3 = field_elems(c);
    const bool f64 = c->p.precision == 64;
    const size_t rb = f64 ? 8 : 4;
    char *w = (char *)c->b_w.p;
    void *wx = w, *wy = w + n3 * rb, *wz = w + 2 * n3 * rb;
    FWT_TRY(buf_reserve(c, C.scratch[19], 128));   // deposit_lines cleared the tallies at 64
    const bool general = !(c->p.sigma_ratio == 1.0 && c->p.eta_t == 0.0);
    const bool accumulate = c->w_written;
    const double scale = fixed_point_scale(c);
    RedoCtx rctx = redo_ctx(c, B, scale, true);
    rctx.tally = (unsigned long long *)((char *)C.scratch[19].p + 64);
    DeferList D{};
    if (!f64) FWT_TRY(defer_list(c, npairs, c->defer_per_pair, D));
    auto launch = [&](const DeferList &L) -> int {
#define FWT_PIECE_LAUNCH(G, A, F, R)                                                                       \
    do {                                                                                                   \
        FWT_CUDA(cudaFuncSetAttribute(deposit_piece_kernel<G, A, F, R>,                                    \
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPieceSmem));      \
        deposit_piece_kernel<G, A, F, R><<<grid, kDepThreads, kPieceSmem, c->stream>>>(                   \
            B.piece, N, ntx, nty, tz0, d_toff, d_list, scale, wx, wy, wz, d_err, rctx, L, B.ras_off, B.ras_pts); \
        FWT_CUDA(cudaGetLastError());                                                                      \
    } while (0)
#define FWT_PIECE_LAUNCH_R(G, A, F)                                                                        \
    do {                                                                                                   \
        if (B.raster) FWT_PIECE_LAUNCH(G, A, F, true); else FWT_PIECE_LAUNCH(G, A, F, false);              \
    } while (0)
        const unsigned grid = (unsigned)(std::min<int64_t>(ntiles, L.w1) - L.w0);
        const int m = kt_begin(c, KT_DEPOSIT);
        if (f64) {
            if (accumulate) FWT_PIECE_LAUNCH_R(true, true, true); else FWT_PIECE_LAUNCH_R(true, false, true);
        } else if (general) {
            if (accumulate) FWT_PIECE_LAUNCH_R(true, true, false); else FWT_PIECE_LAUNCH_R(true, false, false);
        } else {
            if (accumulate) FWT_PIECE_LAUNCH_R(false, true, false); else FWT_PIECE_LAUNCH_R(false, false, false);
        }
#undef FWT_PIECE_LAUNCH_R
#undef FWT_PIECE_LAUNCH
        kt_end(c, m);
        c->launches += 1;
        return 0;
    };
    FWT_TRY(launch(D));
    c->launches += 1;
    c->w_written = true;
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    // tiles without candidates keep their values, so the field's range is taken when it is
    // needed (stats_minmax)
    c->wmm_valid = false;
    if (herr & 2) return fail(FWT_E_TIMEOUT, "deposit: bulk copy wait ran out");
    if (herr & 4) return fail(FWT_E_RANGE, "deposit: contribution outside the fixed-point range");
    if (!f64) FWT_TRY(defer_finish(c, rctx, D, npairs, c->defer_per_pair, ntiles, launch));
    return 0;
}

int launch_scatter(Ctx *c, const CenterlineBatch &B)
{
    if (B.npieces == 0) return 0;
    if (B.npieces >= ((int64_t)1 << 26)) return fail(FWT_E_RANGE, "piece batch exceeds 2^26");
    Ctx &C = *c;
    const int N = c->p.N;
    FWT_TRY(side_ensure(c));
    FWT_TRY(buf_reserve(c, C.scratch[19], 128));   // deposit_lines cleared the tallies at 64
    int *d_err = (int *)((char *)C.scratch[19].p + 104);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const bool general = !(c->p.sigma_ratio == 1.0 && c->p.eta_t == 0.0);
    const double scale = fixed_point_scale(c);
    RedoCtx rctx = redo_ctx(c, B, scale, true);
    rctx.tally = (unsigned long long *)((char *)C.scratch[19].p + 64);
    const int zs = c->slab_nz ? c->slab_z0 : 0, nz = c->slab_nz ? c->slab_nz : N;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int64_t nchunks = (B.npieces + kPChunk - 1) / kPChunk;
    unsigned long long *side = (unsigned long long *)c->b_side.p;
    DeferList D{};
    FWT_TRY(defer_list(c, B.npieces, c->defer_per_piece, D));
    auto launch = [&](const DeferList &L) -> int {
        const int64_t nch = std::min<int64_t>(nchunks, L.w1) - L.w0;
        const unsigned grid = (unsigned)std::min<int64_t>((int64_t)sms * 3, (nch + kScatterWarps - 1) / kScatterWarps);
        const int m = kt_begin(c, KT_DEPOSIT);
        if (general) {
            FWT_CUDA(cudaFuncSetAttribute(scatter_piece_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kScatterSmem));
            scatter_piece_kernel<true><<<grid, kScatterWarps * 32, kScatterSmem, c->stream>>>(
                B.piece, B.npieces, N, zs, nz, (float)scale, side, d_err, L, rctx.tally);
        } else {
            FWT_CUDA(cudaFuncSetAttribute(scatter_piece_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kScatterSmem));
            scatter_piece_kernel<false><<<grid, kScatterWarps * 32, kScatterSmem, c->stream>>>(
                B.piece, B.npieces, N, zs, nz, (float)scale, side, d_err, L, rctx.tally);
        }
        FWT_CUDA(cudaGetLastError());
        kt_end(c, m);
        c->launches += 1;
        return 0;
    };
    FWT_TRY(launch(D));
    c->side_dirty = true;
    c->w_written = true;
    c->wmm_valid = false;
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 64) return fail(FWT_E_STATE, "scatter: a chord box beyond the candidate codes or one period");
    if (herr & 4) return fail(FWT_E_RANGE, "deposit: contribution outside the fixed-point range");
    return defer_finish(c, rctx, D, B.npieces, c->defer_per_piece, nchunks, launch);
}

}  // namespace fwt
