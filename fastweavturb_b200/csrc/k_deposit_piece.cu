// k_deposit_piece.cu -- tile-owned deposition of thin tubes by chord pieces.
//
// The reference deposits sub-segment by sub-segment (tube.f90:762-904): chord j of a section
// accepts a mesh point x when t_j(x) = (x - ci_j) . tci_j >= 0, t_{j+1}(x) < 0 (the next
// chord's plane) and the distance to chord line j is below Rtube, inside chord j's box.
// Consecutive chords share their planes (tube.f90:721-723,740-751), so a run of chords of one
// section can be tested together: one scan of the run's planes per mesh point finds the
// accepting chords as the sign changes of t_k.  For tubes a few grid spacings thick, where a
// sub-segment holds only a handful of points but its box and rows cost far more, this cuts
// the set-up, the binning and the per-point work by the run length.
//
// A piece is up to kPieceMax consecutive chords of one section.  Its record holds the
// section's quintic Taylor-shifted to the piece start, the planes (normal, offset), per sample
// the offset of the box origin in that sample's own frame, and per chord the spline slope,
// Rtube^2 and the chord's own box.  Pieces are binned into tiles like sub-segments; the kernel
// stages a warp's pieces with bulk asynchronous copies, scans every point of piece box x tile
// against the planes, queues the accepted (point, chord) pairs and evaluates them 32 at a time
// with the vorticity code of the sub-segment kernel, into the same int64 fixed-point cells.
#include <cstdio>
#include <cstdlib>

#include "k_deposit.cuh"
#include "k_tile_common.cuh"

namespace fwt {

constexpr int kPieceMax = 8;   // chords per piece

struct __align__(16) PieceRec {
    float off[3], dx;       // mesh point at box_lo minus the origin o (the piece's first sample)
    float b[15], smin;      // c(z0 + W) - c(z0) = sum_k b[k-1] W^k about the piece start z0
    float thi[3], A;        // wrap thresholds pi - c(z0) (see SegF); core amplitude
    float tlo[3], om;
    int kq[3];
    float ph0;
    float inv2s2, ftd, amp, Gamma;   // constant-core profile (tube.f90:845-847)
    float Linv, eta, q, guard;       // guard: half-width of the band around a plane where the
                                     // piece-frame plane test is redone in the sample's frame
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

// slot of every piece (one warp per section slot)
__global__ void piece_map_kernel(const LineParam *__restrict__ lp, const int *__restrict__ slot_line, int64_t nslots,
                                 const int *__restrict__ ntf, const int64_t *__restrict__ poff, int *__restrict__ map)
{
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nslots) return;
    const LineParam &P = lp[slot_line[warp]];
    if ((int)(warp - P.slot_off) >= P.n_sec) return;
    const int n = (ntf[warp] + kPieceMax - 1) / kPieceMax;
    for (int j = lane; j < n; j += 32) map[poff[warp] + j] = (int)warp;
}

// One thread per piece: FP64 samples, chords and boxes as the sub-segment set-up
// (tube.f90:703-798), then the FP32 record in the piece's frame.  err bit 8: a piece box
// wider than 1023 points (the 10-bit chord box offsets).
__global__ void __launch_bounds__(128) piece_build_kernel(
    const LineParam *__restrict__ lp, const int *__restrict__ slot_line, const int *__restrict__ map, int64_t npieces,
    const double *__restrict__ X, const double *__restrict__ Y, const double *__restrict__ Z,
    const double *__restrict__ cze, int64_t node_base, const double *__restrict__ coe, const int *__restrict__ ntf,
    const double *__restrict__ dtf, const int64_t *__restrict__ poff, int N, double Rtube_ratio, double dzeta_sup,
    double eta, PieceRec *__restrict__ rec, int *__restrict__ err)
{
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
    const double *cf = coe + 18 * (size_t)slot;
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
    // pass 1: the piece box (union of the chord boxes), the largest Rtube, extent and bend
    int blo[3] = {1 << 30, 1 << 30, 1 << 30}, bhi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    double Rmax = 0.0, dlen = 0.0;
    float bendmin = 1.0f;
    double tprev[3] = {0.0, 0.0, 0.0};
    walk([&](int jj, const double *ch, double nd, const double *pj, const int *lo3, const int *hi3, double, double,
             double Rt) {
        const double inv = 1.0 / nd;
        const double tc[3] = {ch[0] * inv, ch[1] * inv, ch[2] * inv};
        if (jj > 0) bendmin = fminf(bendmin, (float)(tc[0] * tprev[0] + tc[1] * tprev[1] + tc[2] * tprev[2]));
        tprev[0] = tc[0];
        tprev[1] = tc[1];
        tprev[2] = tc[2];
        dlen = fmax(dlen, sqrt(pj[0] * pj[0] + pj[1] * pj[1] + pj[2] * pj[2]));
        if (jj == n) return;
        Rmax = fmax(Rmax, Rt);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            blo[k] = min(blo[k], lo3[k]);
            bhi[k] = max(bhi[k], hi3[k]);
        }
    });
    PieceRec &R = rec[pc];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (bhi[k] - blo[k] > 1023) atomicOr(err, 8);
        R.box_lo[k] = blo[k];
        R.box_hi[k] = bhi[k];
        // mesh coordinate of the 1-based unwrapped index box_lo: (i - 1) dx + xstart
        const double X0 = dadd(dmul((double)blo[k] - 1.0, dev_pi2() / N), xstart);
        R.off[k] = (float)(X0 - o[k]);
    }
    R.dx = (float)(dev_pi2() / N);
    R.nch = n;
    // pass 2: planes, per-sample frames and chords
    float Wm = 0.0f, cmax = 0.0f;
    walk([&](int jj, const double *ch, double nd, const double *pj, const int *lo3, const int *hi3, double s0,
             double s1, double Rt) {
        const double inv = 1.0 / nd;
        const double tc[3] = {ch[0] * inv, ch[1] * inv, ch[2] * inv};
        const float ck = (float)(tc[0] * pj[0] + tc[1] * pj[1] + tc[2] * pj[2]);
        R.pl[jj] = make_float4((float)tc[0], (float)tc[1], (float)tc[2], ck);
        cmax = fmaxf(cmax, fabsf(ck));
        // mesh point at box_lo minus sample jj (FP64, then FP32): the sample's own local frame,
        // as accurate as a sub-segment record's
        float offj[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double X0 = dadd(dmul((double)blo[k] - 1.0, dev_pi2() / N), xstart);
            offj[k] = (float)(X0 - (o[k] + pj[k]));
        }
        const float zoff = (float)((s0 - zj0) * L);
        R.po[jj] = make_float4(offj[0], offj[1], offj[2], zoff);
        if (jj == n) return;
        const float g = (float)((s1 - s0) * L * inv);
        R.chq[jj] = make_float4(g, (float)(Rt * Rt),
                                __uint_as_float(pack3(lo3[0] - blo[0], lo3[1] - blo[1], lo3[2] - blo[2])),
                                __uint_as_float(pack3(hi3[0] - blo[0], hi3[1] - blo[1], hi3[2] - blo[2])));
        Wm = fmaxf(Wm, (zoff + (float)(nd + Rt) * fabsf(g)) * 1.01f);
    });
    // FP32 rounding of the piece-frame plane test d . tci_k - c_k stays well below
    // 1e-6 (|d|_1 + |c_k|); |d|_1 is bounded by the box corners' offsets
    float dmax = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        dmax += fmaxf(fabsf(R.off[k]), fabsf(R.off[k] + (float)(bhi[k] - blo[k]) * R.dx));
    R.guard = 1.0e-6f * (dmax + cmax) + 1.0e-30f;
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
    R.ftd = expf(-(float)(rt * rt) * R.inv2s2);
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
constexpr int kPChunk = 8;        // pieces staged per warp chunk
constexpr int kPQueue = 64;       // accepted (point, chord) queue of a warp

// A piece's box clipped to the tile (one periodic image).
struct PBox {
    int lo[3];      // clipped origin, tile-local
    int n[3];       // clipped extent
    int dl[3];      // clipped origin relative to the piece's box_lo, minus lo
    int vol;
    float inx, inxy;   // (1 + 1e-6) / n[0], (1 + 1e-6) / (n[0] n[1])
    int pad[2];
};

struct PieceStage {
    PieceRec rec[kPChunk];
    PBox box[kPChunk];
    uint32_t q[kPQueue];   // piece | chord << 3 | x << 6 | y << 10 | z << 13 (tile-local)
    uint64_t bar;
    uint64_t pad;
};
constexpr size_t kPieceSmem = kAccBytes + sizeof(PieceStage) * kDepWarps;

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
    B.inx = nonempty ? 1.000001f / (float)B.n[0] : 0.0f;
    B.inxy = nonempty ? 1.000001f / (float)(B.n[0] * B.n[1]) : 0.0f;
}

// Evaluate the first `cnt` queued (point, chord) pairs, one per lane, into the tile cells.
template <bool General>
__device__ __forceinline__ void drain_pieces(PieceStage &S, long long (*acc)[kAccN], int lane, int cnt, int &qn,
                                             float fscale, float fmaxq, int *__restrict__ err)
{
    if (lane < cnt) {
        const uint32_t e = S.q[lane];
        const int k = (int)(e & 7u), j = (int)((e >> 3) & 7u);
        const int lx = (int)((e >> 6) & 15u), ly = (int)((e >> 10) & 7u), lz = (int)(e >> 13);
        const PBox &B = S.box[k];
        const PieceRec &R = S.rec[k];
        const float4 cp = R.po[j], cq = R.chq[j], pn = R.pl[j];
        const float ex = fmaf((float)(lx + B.dl[0]), R.dx, cp.x);
        const float ey = fmaf((float)(ly + B.dl[1]), R.dx, cp.y);
        const float ez = fmaf((float)(lz + B.dl[2]), R.dx, cp.z);
        const float t0 = fmaf(ez, pn.z, fmaf(ey, pn.y, ex * pn.x));
        float vv[3];
        vort_w<General, true>(R, ex, ey, ez, cp.w, t0 * cq.x, cq.y, vv);
        const int p = lx + kSY * ly + kSZ * lz;
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
    __syncwarp();
    const int rem = qn - cnt;
    const uint32_t keep = lane < rem ? S.q[cnt + lane] : 0u;
    __syncwarp();
    if (lane < rem) S.q[lane] = keep;
    __syncwarp();
    qn = rem;
}

// One CTA per tile.  Each warp claims chunks of kPChunk pieces, stages their records with one
// bulk asynchronous copy each, then scans the points of every piece box x tile, 32 at a time
// across the lanes: the plane scan gives the chords whose slab holds the point, the chord's
// box and the cylinder test (tube.f90:793-818) decide, and the accepted pairs are queued and
// evaluated 32 at a time.
template <bool General, bool Accumulate>
__global__ void __launch_bounds__(kDepThreads, 3) deposit_piece_kernel(
    const PieceRec *__restrict__ rec, int N, int ntx, int nty, const int64_t *__restrict__ tile_off,
    const uint32_t *__restrict__ list, double scale, float *__restrict__ wx, float *__restrict__ wy,
    float *__restrict__ wz, uint32_t *__restrict__ mm, int *__restrict__ err)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    long long(*acc)[kAccN] = reinterpret_cast<long long(*)[kAccN]>(dsm);
    const int tile = blockIdx.x;
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    PieceStage &S = reinterpret_cast<PieceStage *>(dsm + kAccBytes)[warp];
    if (lane == 0) mbar_init(&S.bar);
    // chunks are handed out through a shared counter: a warp that finishes early takes the
    // next one, so the warps of a tile end close together at the epilogue's barrier
    __shared__ int next_chunk;
    if (threadIdx.x == 0) next_chunk = kDepWarps;
    tile_acc_init<Accumulate>(acc, N, x0, y0, z0, scale, wx, wy, wz);
    __syncthreads();
    const int64_t c0 = tile_off[tile], c1 = tile_off[tile + 1];
    const int nchunks = (int)((c1 - c0 + kPChunk - 1) / kPChunk);
    const float fscale = (float)scale;
    const float fmaxq = 4.0e18f;
    uint32_t phase = 0;
    bool failed = false;
    int qn = 0;
    for (int ch = warp; ch < nchunks && !failed;) {
        const int64_t base = c0 + (int64_t)ch * kPChunk;
        const int nc = (c1 - base < kPChunk) ? (int)(c1 - base) : kPChunk;
        const uint32_t v = lane < nc ? __ldg(list + base + lane) : 0u;
        if (lane == 0) mbar_expect(&S.bar, (uint32_t)(nc * sizeof(PieceRec)));
        __syncwarp();
        if (lane < nc) bulk_g2s(&S.rec[lane], rec + (v & ((1u << 26) - 1u)), (uint32_t)sizeof(PieceRec), &S.bar);
        if (!mbar_wait(&S.bar, phase)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        int vol = 0;
        if (lane < nc) {
            PBox B;
            pclip(S.rec[lane], v >> 26, N, x0, y0, z0, B);
            S.box[lane] = B;
            vol = B.vol;
        }
        int incl = vol;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int voff = incl - vol;
        const int total = __shfl_sync(0xffffffffu, incl, kPChunk - 1);
        __syncwarp();
        for (int r0 = 0; r0 < total; r0 += 32) {
            const int r = r0 + lane;
            int k = 0;
#pragma unroll
            for (int step = kPChunk / 2; step > 0; step >>= 1) {
                const int t = k + step;
                const int ot = __shfl_sync(0xffffffffu, voff, t);
                if (t < nc && ot <= r) k = t;
            }
            const int rk = __shfl_sync(0xffffffffu, voff, k);
            uint32_t amask = 0u;   // accepted chords of this lane's point
            int lx = 0, ly = 0, lz = 0;
            if (r < total) {
                const PBox &B = S.box[k];
                const PieceRec &R = S.rec[k];
                const int li = r - rk;
                const int nxy = B.n[0] * B.n[1];
                int iz = (int)((float)li * B.inxy);
                if (iz * nxy > li) --iz;
                else if ((iz + 1) * nxy <= li) ++iz;
                const int rxy = li - iz * nxy;
                int iy = (int)((float)rxy * B.inx);
                if (iy * B.n[0] > rxy) --iy;
                else if ((iy + 1) * B.n[0] <= rxy) ++iy;
                const int ix = rxy - iy * B.n[0];
                lx = B.lo[0] + ix;
                ly = B.lo[1] + iy;
                lz = B.lo[2] + iz;
                const int rx = lx + B.dl[0], ry = ly + B.dl[1], rz = lz + B.dl[2];   // offsets from box_lo
                const float dxv = fmaf((float)rx, R.dx, R.off[0]);
                const float dyv = fmaf((float)ry, R.dx, R.off[1]);
                const float dzv = fmaf((float)rz, R.dx, R.off[2]);
                const int nch = R.nch;
                // plane scan: bit k of sgn = (t_k >= 0), in the piece frame; a point within the
                // rounding band of a plane is re-tested in that sample's own frame
                uint32_t sgn = 0u;
                const float guard = R.guard;
                for (int kk = 0; kk <= nch; ++kk) {
                    const float4 pl = R.pl[kk];
                    float tk = fmaf(dzv, pl.z, fmaf(dyv, pl.y, fmaf(dxv, pl.x, -pl.w)));
                    if (fabsf(tk) < guard) {
                        const float4 po = R.po[kk];
                        const float ex = fmaf((float)rx, R.dx, po.x);
                        const float ey = fmaf((float)ry, R.dx, po.y);
                        const float ez = fmaf((float)rz, R.dx, po.z);
                        tk = fmaf(ez, pl.z, fmaf(ey, pl.y, ex * pl.x));
                    }
                    sgn |= (tk >= 0.0f ? 1u : 0u) << kk;
                }
                uint32_t cand = sgn & ~(sgn >> 1) & ((1u << nch) - 1u);
                while (cand) {
                    const int j = __ffs(cand) - 1;
                    cand &= cand - 1u;
                    const float4 cp = R.po[j], cq = R.chq[j], pn = R.pl[j];
                    const uint32_t blo = __float_as_uint(cq.z), bhi = __float_as_uint(cq.w);
                    if (rx < unpack3(blo, 0) || rx > unpack3(bhi, 0) || ry < unpack3(blo, 1) || ry > unpack3(bhi, 1) ||
                        rz < unpack3(blo, 2) || rz > unpack3(bhi, 2))
                        continue;
                    // distance to chord line j (tube.f90:806-818), in the chord's frame
                    const float ex = fmaf((float)rx, R.dx, cp.x);
                    const float ey = fmaf((float)ry, R.dx, cp.y);
                    const float ez = fmaf((float)rz, R.dx, cp.z);
                    const float t0 = fmaf(ez, pn.z, fmaf(ey, pn.y, ex * pn.x));
                    const float r2 = fmaf(-t0, t0, fmaf(ez, ez, fmaf(ey, ey, ex * ex)));
                    if (r2 < cq.y) amask |= 1u << j;
                }
            }
            // queue the accepted pairs (a point may pass for more than one chord)
            while (__any_sync(0xffffffffu, amask != 0u)) {
                const bool ok = amask != 0u;
                uint32_t code = 0u;
                if (ok) {
                    const int j = __ffs(amask) - 1;
                    amask &= amask - 1u;
                    code = (uint32_t)k | ((uint32_t)j << 3) | ((uint32_t)lx << 6) | ((uint32_t)ly << 10) |
                           ((uint32_t)lz << 13);
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) S.q[qn + __popc(bal & ((1u << lane) - 1u))] = code;
                qn += __popc(bal);
                __syncwarp();
                if (qn >= 32) drain_pieces<General>(S, acc, lane, 32, qn, fscale, fmaxq, err);
            }
        }
        if (qn > 0) drain_pieces<General>(S, acc, lane, qn, qn, fscale, fmaxq, err);
        __syncwarp();   // the warp's stage is reused by its next chunk
        int nxt = 0;
        if (lane == 0) nxt = atomicAdd(&next_chunk, 1);
        ch = __shfl_sync(0xffffffffu, nxt, 0);
    }
    if (failed && lane == 0) atomicOr(err, 2);
    __syncthreads();
    tile_epilogue(acc, N, x0, y0, z0, scale, wx, wy, wz, mm);
}

// ------------------------------------------------------------------------------ host
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
    km = kt_begin(c, KT_CENTERLINE);
    piece_map_kernel<<<(unsigned)((slots * 32 + 255) / 256), 256, 0, c->stream>>>(B.lp, B.slot_line, slots, B.ntf,
                                                                                   d_poff, d_map);
    if (np_ > 0)
        piece_build_kernel<<<(unsigned)((np_ + 127) / 128), 128, 0, c->stream>>>(
            B.lp, B.slot_line, d_map, np_, c->d_x, c->d_y, c->d_z, B.cze, B.node_base, B.coe, B.ntf, B.dtf, d_poff,
            c->p.N, c->p.Rtube_ratio, c->p.dzeta_sup, c->p.eta_t, B.piece, d_err);
    kt_end(c, km);
    c->launches += 5;
    FWT_CUDA(cudaGetLastError());
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 8) return fail(FWT_E_RANGE, "piece box wider than 1023 grid points");
    return 0;
}

int launch_piece(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out)
{
    const int N = c->p.N;
    const int ntx = (N + TX - 1) / TX, nty = (N + TY - 1) / TY, ntz = (N + TZ - 1) / TZ;
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
    if (nrec > 0) pair_count_kernel<PieceRec><<<bq, 256, 0, c->stream>>>(B.piece, nrec, N, d_cnt, d_err);
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
        pair_emit_kernel<PieceRec><<<bq, 256, 0, c->stream>>>(B.piece, nrec, N, ntx, nty, d_cnt, d_key, d_val, d_tcnt);
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
    float *w = (float *)c->b_w.p;
    FWT_TRY(buf_reserve(c, C.scratch[19], 64));
    uint32_t *d_mm = (uint32_t *)((char *)C.scratch[19].p + 16);
    mm_init_kernel<<<1, 32, 0, c->stream>>>(d_mm, 6);
    const bool general = !(c->p.sigma_ratio == 1.0 && c->p.eta_t == 0.0);
    const bool accumulate = c->w_written;
    const double scale = fixed_point_scale(c);
    km = kt_begin(c, KT_DEPOSIT);
#define FWT_PIECE_LAUNCH(G, A)                                                                              \
    do {                                                                                                    \
        FWT_CUDA(cudaFuncSetAttribute(deposit_piece_kernel<G, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                      (int)kPieceSmem));                                                    \
        deposit_piece_kernel<G, A><<<(unsigned)ntiles, kDepThreads, kPieceSmem, c->stream>>>(              \
            B.piece, N, ntx, nty, d_toff, d_list, scale, w, w + n3, w + 2 * n3, d_mm, d_err);                \
    } while (0)
    if (general) {
        if (accumulate) FWT_PIECE_LAUNCH(true, true); else FWT_PIECE_LAUNCH(true, false);
    } else {
        if (accumulate) FWT_PIECE_LAUNCH(false, true); else FWT_PIECE_LAUNCH(false, false);
    }
#undef FWT_PIECE_LAUNCH
    kt_end(c, km);
    // algorithmic bytes: omega written once (read too when accumulating), one list entry and
    // one record per (tile, piece) pair
    c->kbytes[KT_DEPOSIT] += (int64_t)(3 * n3 * 4 * (accumulate ? 2 : 1)) + npairs * (int64_t)(4 + sizeof(PieceRec));
    c->launches += 2;
    FWT_CUDA(cudaGetLastError());
    c->w_written = true;
    uint32_t hmm[6];
    FWT_CUDA(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 2) return fail(FWT_E_TIMEOUT, "deposit: bulk copy wait ran out");
    if (herr & 4) return fail(FWT_E_RANGE, "deposit: contribution outside the fixed-point range");
    c->wmin.assign(3, 0.f);
    c->wmax.assign(3, 0.f);
    for (int d = 0; d < 3; ++d) {
        c->wmin[d] = ord2f(hmm[2 * d]);
        c->wmax[d] = ord2f(hmm[2 * d + 1]);
    }
    c->wmm_valid = true;
    return 0;
}

}  // namespace fwt
