// k_deposit_tile.cu -- tile-owned Burgers-tube deposition with integer cell lists.
//
// 1. pair_count / pair_emit: every sub-segment's box (tube.f90:793-798) is cut into the
//    grid tiles it overlaps (periodic images kept apart), giving (tile, sub-segment|image)
//    pairs in sub-segment order.
// 2. counting sort by tile: integer histogram, exclusive scan, scatter (warp-aggregated
//    atomics) -> per-tile candidate lists holding exactly the sub-segments whose box meets
//    the tile.
// 3. deposit_tile_kernel: one CTA per tile, accumulating the tile in shared int64 fixed-point
//    cells.  Integer addition is associative, so the tile sum is bit-exact whatever the order
//    of candidates.  Each warp claims chunks of candidates and stages their FP32 records with
//    one bulk asynchronous copy each (cp.async.bulk, the TMA engine's 1-D form, completing on
//    the warp's mbarrier).  A chunk's work is flattened into grid rows along each candidate's
//    best-aligned axis; each row solves the two half-space tests and the cylinder test of
//    tube.f90:806-818 for its index interval (one-point margin) and evaluates the reference
//    predicate and vorticity only there, where the reference walks the whole box (about 11
//    points per accepted one at these sub-segment lengths).  A point whose plane test lies
//    within its FP32 rounding bound of zero is decided by the reference's FP64 tests, and
//    evaluated in FP64 if accepted: the field jumps across the plane two consecutive chords
//    share.  The tile is written once with coalesced float4 stores.
#include <cstdio>
#include <cstdlib>

#include "k_deposit.cuh"
#include "k_tile_common.cuh"

namespace fwt {

// Can the tile's points (unwrapped grid offsets o0..o0+n-1 from the record's box origin) pass
// t0 >= 0, t1 < 0 and rho < Rtube (tube.f90:806-818)?  Conservative: extremes of the linear
// tests over the tile's bounding box, and the box's distance to the chord line.
__device__ __forceinline__ bool tile_may_hit(const SegRec &R, int ox, int oy, int oz, int nx, int ny, int nz)
{
    // Every operation is spelled out (fmaf, __fmul_rn, __fadd_rn): the counting and the
    // emitting kernel of the binning inline this test separately and must decide each tile
    // identically, which free contraction by the compiler would not guarantee.
    const float dx = R.dx;
    const float hx = __fmul_rn(0.5f * (float)(nx - 1), dx), hy = __fmul_rn(0.5f * (float)(ny - 1), dx),
                hz = __fmul_rn(0.5f * (float)(nz - 1), dx);
    const float cx = __fadd_rn(fmaf((float)ox, dx, R.off[0]), hx), cy = __fadd_rn(fmaf((float)oy, dx, R.off[1]), hy),
                cz = __fadd_rn(fmaf((float)oz, dx, R.off[2]), hz);
    const float hn = sqrtf(fmaf(hz, hz, fmaf(hy, hy, __fmul_rn(hx, hx))));
    const float Rt = sqrtf(R.R2);
    const float e = __fmul_rn(1e-3f, __fadd_rn(__fadd_rn(hn, Rt), dx));   // slack for the rounding of the bounds
    const float t0c = fmaf(cz, R.tc0[2], fmaf(cy, R.tc0[1], __fmul_rn(cx, R.tc0[0])));
    const float t0h = fmaf(hz, fabsf(R.tc0[2]), fmaf(hy, fabsf(R.tc0[1]), __fmul_rn(hx, fabsf(R.tc0[0]))));
    if (__fadd_rn(t0c, t0h) < -e) return false;
    const float t1c = fmaf(__fadd_rn(cz, -R.dci[2]), R.tc1[2],
                           fmaf(__fadd_rn(cy, -R.dci[1]), R.tc1[1], __fmul_rn(__fadd_rn(cx, -R.dci[0]), R.tc1[0])));
    const float t1h = fmaf(hz, fabsf(R.tc1[2]), fmaf(hy, fabsf(R.tc1[1]), __fmul_rn(hx, fabsf(R.tc1[0]))));
    if (__fadd_rn(t1c, -t1h) > e) return false;
    const float d2 = fmaxf(fmaf(-t0c, t0c, fmaf(cz, cz, fmaf(cy, cy, __fmul_rn(cx, cx)))), 0.0f);
    const float rr = __fadd_rn(__fadd_rn(Rt, hn), e);
    return d2 <= __fmul_rn(rr, rr);
}

// Visit every (tile, image) of record S's box that may hold accepted points.
template <typename F>
__device__ __forceinline__ void for_each_tile(const SegRec &S, int N, F &&f)
{
    for_each_box_tile(S.box_lo, S.box_hi, N,
                      [&](int ox, int oy, int oz, int nx, int ny, int nz) {
                          return tile_may_hit(S, ox, oy, oz, nx, ny, nz);
                      },
                      f);
}

// Counting sort, last step: every emitted pair to its tile's list.  Slots left unfilled by
// the emitting pass (key kNoTile) are skipped.
__global__ void tile_scatter_kernel(const uint32_t *__restrict__ key, const uint32_t *__restrict__ val, int64_t n,
                                    const int64_t *__restrict__ tile_off, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ list)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t t = i < n ? key[i] : kNoTile;
    const bool live = t != kNoTile;
    // warp-aggregated cursor: lanes with the same tile take consecutive slots
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const unsigned peers = __match_any_sync(act, t);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(cursor + t, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    const uint32_t r = base + __popc(peers & ((1u << lane) - 1u));
    list[tile_off[t] + r] = val[i];
}

__global__ void u32_to_i64_kernel(const uint32_t *__restrict__ a, int64_t n, int64_t *__restrict__ b)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// -------------------------------------------------------------------------------- deposit
struct CandBox {
    int lo[3];      // clipped box origin, tile-local
    int n[3];       // clipped box extent
    int dorg[3];    // clipped origin minus the record's box_lo (grid points)
    int axis;       // walk axis: largest |tc0|
    int nrows;      // n[(axis+1)%3] * n[(axis+2)%3]
    float isa;      // 1 / (dx tc0[axis])
    float isb;      // 1 / (dx tc1[axis]), 0 when |tc1[axis]| <= 0.05 (no bound from t1)
    float q2;       // dx^2 (1 - tc0[axis]^2), 0 when the cylinder bound is not used
    float i2q;      // 1 / (2 q2)
    float rnb;      // (1 + 1e-6) / n[(axis+1)%3]: row -> (jb, jc) without an integer divide
    int dl[3];      // dorg - lo: tile-local coordinate -> grid offset from the record's box_lo
    float pe;       // rounding bound of the record's plane tests (plane_eps)
};

// Index interval [ilo, ihi] (clamped to [0, n-1]) of the grid row d0 + i dx e_a that can pass
// t0 >= 0, t1 < 0 and rho^2 < R2; a one-point margin covers the FP32 rounding of the bounds.
// [clo, chi] is the row's core, where all three tests hold for certain: two points inside every
// bound (the bounds' rounding is far below a point, and a plane two points away is far beyond
// its rounding bound pe), and only when the row is bounded by both planes and the cylinder.
__device__ __forceinline__ void row_interval(const SegRec &R, const CandBox &B, float d0x, float d0y, float d0z, int a,
                                             int n, int &ilo, int &ihi, int &clo, int &chi)
{
    clo = 1;
    chi = 0;
    const float dx = R.dx;
    const float T0 = d0x * R.tc0[0] + d0y * R.tc0[1] + d0z * R.tc0[2];
    const float ta = R.tc0[a];
    float lo = -2.0f, hi = (float)n + 1.0f;
    // t0(i) = T0 + i dx ta >= 0  (|ta| >= 1/sqrt3 on the best-aligned axis)
    const float r0 = -T0 * B.isa;
    if (ta > 0.f) lo = fmaxf(lo, r0);
    else hi = fminf(hi, r0);
    // t1(i) = T1 + i dx tb < 0
    if (B.isb != 0.0f) {
        const float T1 = (d0x - R.dci[0]) * R.tc1[0] + (d0y - R.dci[1]) * R.tc1[1] + (d0z - R.dci[2]) * R.tc1[2];
        const float r1 = -T1 * B.isb;
        if (B.isb > 0.f) hi = fminf(hi, r1);
        else lo = fmaxf(lo, r1);
    }
    // rho^2(i) = Q0 + Q1 i + Q2 i^2 < R2 (the distance to the chord line)
    if (B.q2 > 0.0f) {
        const float da = a == 0 ? d0x : (a == 1 ? d0y : d0z);
        const float Q1 = 2.0f * dx * (da - T0 * ta);
        const float Q0 = d0x * d0x + d0y * d0y + d0z * d0z - T0 * T0;
        const float rmin = Q0 - Q1 * Q1 * (0.5f * B.i2q);
        if (rmin > R.R2 * 1.001f + 1e-30f) {
            ilo = 1;
            ihi = 0;
            return;
        }
        const float sq = sqrtf(fmaxf(Q1 * Q1 - 4.0f * B.q2 * (Q0 - R.R2), 0.0f));
        lo = fmaxf(lo, (-Q1 - sq) * B.i2q);
        hi = fminf(hi, (-Q1 + sq) * B.i2q);
        if (B.isb != 0.0f) {
            clo = max(0, (int)ceilf(lo) + 2);
            chi = min(n - 1, (int)floorf(hi) - 2);
        }
    }
    ilo = max(0, (int)ceilf(lo) - 1);
    ihi = min(n - 1, (int)floorf(hi) + 1);
}

// Clip record R's box (image code img) to the tile at tl.
__device__ __forceinline__ void clip_box(const SegRec &R, uint32_t img, int N, int tx0, int ty0, int tz0, CandBox &B)
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
        B.dorg[d] = lo - (R.box_lo[d] - 1);
        B.dl[d] = B.dorg[d] - B.lo[d];
        nonempty = nonempty && B.n[d] > 0;
    }
    const float ax = fabsf(R.tc0[0]), ay = fabsf(R.tc0[1]), az = fabsf(R.tc0[2]);
    const int a = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    B.axis = a;
    // per-axis picks by selects: a runtime index would put B in local memory
    const int nbv = a == 0 ? B.n[1] : (a == 1 ? B.n[2] : B.n[0]);
    const int ncv = a == 0 ? B.n[2] : (a == 1 ? B.n[0] : B.n[1]);
    B.nrows = nonempty ? nbv * ncv : 0;
    const float ta = a == 0 ? R.tc0[0] : (a == 1 ? R.tc0[1] : R.tc0[2]);
    const float tb = a == 0 ? R.tc1[0] : (a == 1 ? R.tc1[1] : R.tc1[2]);
    const float dx = R.dx;
    B.isa = 1.0f / (dx * ta);
    B.isb = fabsf(tb) > 0.05f ? 1.0f / (dx * tb) : 0.0f;
    const float q2 = dx * dx * (1.0f - ta * ta);
    B.q2 = q2 > 0.01f * dx * dx ? q2 : 0.0f;
    B.i2q = B.q2 > 0.0f ? 0.5f / B.q2 : 0.0f;
    B.rnb = nonempty ? 1.000001f / (float)nbv : 0.0f;
    const int ext[3] = {R.box_hi[0] - R.box_lo[0], R.box_hi[1] - R.box_lo[1], R.box_hi[2] - R.box_lo[2]};
    B.pe = plane_eps(R.off, ext, dx, R.dci);
}

// Warp-autonomous tile deposition.  Each warp claims chunks of up to kWarpChunk candidates of the
// tile, stages their records in its own slice of shared memory with one bulk asynchronous
// copy per record (cp.async.bulk, completion on the warp's mbarrier), flattens the chunk's
// grid rows across its lanes, and adds into the CTA's fixed-point accumulators.  Only the
// accumulator set-up and the epilogue synchronise the whole CTA.
constexpr int kWarpChunk = 8;
constexpr int kQueue = 64;       // accepted-point queue of a warp (< 32 left over + 32 new)
struct WarpStage {
    SegRec rec[kWarpChunk];
    CandBox box[kWarpChunk];
    uint32_t q[kQueue];         // accepted points: candidate | x << 4 | y << 8 | z << 11 (tile-local)
                                // | kQDecide (a plane test within its rounding bound)
    uint32_t id[kWarpChunk];    // global record ids of the staged candidates
    uint64_t bar;
    uint64_t pad;
};
constexpr size_t kDepSmem = kAccBytes + sizeof(WarpStage) * kDepWarps;
constexpr uint32_t kQDecide = 1u << 15;

// Evaluate the first `cnt` queued points of the warp, one per lane (t0 again, then the
// vorticity), add them into the tile's fixed-point cells and drop them from the queue.
// Pairs whose curved-branch amplification exceeds kRedoCond, and pairs with a plane test
// within its rounding bound (kQDecide), are deferred to FP64 (DeferList) instead.  In the
// emit-only pass (D.emit_only) nothing is added and only the deferred pairs are listed again.
template <bool General, bool F64>
__device__ __forceinline__ void drain_queue(WarpStage &S, long long (*acc)[kAccN], int lane, int cnt, int &qn,
                                            unsigned &nacc, float fscale, float fmaxq, int *__restrict__ err,
                                            const RedoCtx &redo, const DeferList &D, int x0, int y0, int z0)
{
    bool flag = false, ok64 = false, counted = false;
    uint32_t rrec = 0;
    int lx = 0, ly = 0, lz = 0;
    if (F64 && lane < cnt) {
        // FP64 tile path: the candidate passed the widened FP32 tests; the reference's FP64
        // tests decide, at its index in the sub-segment's own box
        const uint32_t e = S.q[lane];
        const int k = (int)(e & 15u);
        lx = (int)((e >> 4) & 15u), ly = (int)((e >> 8) & 7u), lz = (int)((e >> 11) & 7u);
        const CandBox &B = S.box[k];
        const SegRec &R = S.rec[k];
        ok64 = eval_pair_f64(redo, (int64_t)(S.id[k] & ((1u << 26) - 1u)), R.box_lo[0] + lx + B.dl[0],
                      R.box_lo[1] + ly + B.dl[1], R.box_lo[2] + lz + B.dl[2], reinterpret_cast<double(*)[kAccN]>(acc),
                      lx + kSY * ly + kSZ * lz);
    } else if (lane < cnt) {
        const uint32_t e = S.q[lane];
        const int k = (int)(e & 15u);
        lx = (int)((e >> 4) & 15u), ly = (int)((e >> 8) & 7u), lz = (int)((e >> 11) & 7u);
        if (e & kQDecide) {
            flag = true;
            rrec = (S.id[k] & ((1u << 26) - 1u)) | kDeferDecide;
        } else if (General || !D.emit_only) {
            counted = true;
            const CandBox &B = S.box[k];
            const SegRec &R = S.rec[k];
            const float d0x = fmaf((float)(lx + B.dl[0]), R.dx, R.off[0]);
            const float d0y = fmaf((float)(ly + B.dl[1]), R.dx, R.off[1]);
            const float d0z = fmaf((float)(lz + B.dl[2]), R.dx, R.off[2]);
            // the pair passed rec_classify: only t0 (the spline argument) is needed again
            const float t0 = fmaf(d0z, R.tc0[2], fmaf(d0y, R.tc0[1], d0x * R.tc0[0]));
            float vv[3], cond;
            rec_vorticity<General>(R, d0x, d0y, d0z, t0, vv, cond);
            const int p = lx + kSY * ly + kSZ * lz;
            flag = General && !(cond <= kRedoCond);
            if (flag) {
                rrec = S.id[k] & ((1u << 26) - 1u);
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

// The candidate test of the FP64 tile path: the three tests of tube.f90:806-818 widened by far
// more than their FP32 rounding (about 1e-7 of the offsets), so that every point the
// reference's FP64 tests accept is queued; the FP64 tests then decide.
__device__ __forceinline__ bool rec_tests_wide(const SegRec &R, float d0x, float d0y, float d0z)
{
    const float e = 1e-3f * R.dx;
    const float t0 = fmaf(d0z, R.tc0[2], fmaf(d0y, R.tc0[1], d0x * R.tc0[0]));
    if (!(t0 >= -e)) return false;
    const float ex = d0x - R.dci[0], ey = d0y - R.dci[1], ez = d0z - R.dci[2];
    const float t1 = fmaf(ez, R.tc1[2], fmaf(ey, R.tc1[1], ex * R.tc1[0]));
    if (!(t1 < e)) return false;
    const float d2 = fmaf(d0z, d0z, fmaf(d0y, d0y, d0x * d0x));
    return fmaf(-t0, t0, d2) < R.R2 + 1e-5f * (d2 + R.R2) + e * e;
}

template <bool General, bool Accumulate, bool F64>
__global__ void __launch_bounds__(kDepThreads, F64 ? 2 : 3) deposit_tile_kernel(
    const SegRec *__restrict__ rec, int N, int ntx, int nty, int tz0, const int64_t *__restrict__ tile_off,
    const uint32_t *__restrict__ list, double scale, void *__restrict__ wx, void *__restrict__ wy,
    void *__restrict__ wz, int *__restrict__ err, const RedoCtx redo, const DeferList D)
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
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    WarpStage &S = reinterpret_cast<WarpStage *>(dsm + kAccBytes)[warp];
    if (lane == 0) mbar_init(&S.bar);
    // chunks are handed out through a shared counter: a warp that finishes early takes the
    // next one, so the warps of a tile end close together at the epilogue's barrier
    __shared__ int next_rec;
    if (threadIdx.x == 0) next_rec = kDepWarps * kWarpChunk;
    if constexpr (F64)
        tile_acc_init_f64<Accumulate>(reinterpret_cast<double(*)[kAccN]>(acc), N, x0, y0, z0, zs, zlim, (const double *)wx,
                                      (const double *)wy, (const double *)wz);
    else if (!D.emit_only)
        tile_acc_init<Accumulate>(acc, N, x0, y0, z0, zs, zlim, scale, (const float *)wx, (const float *)wy,
                                  (const float *)wz);
    __syncthreads();

    const int nrec = (int)(c1 - c0);
    const float fscale = (float)scale;
    const float fmaxq = 4.0e18f;
    uint32_t phase = 0;
    bool failed = false;
    int qn = 0;   // queued points of this warp (warp-uniform)
    unsigned nacc = 0;   // pairs evaluated by this warp (warp-uniform)
    int csz = kWarpChunk;   // candidates in this warp's current chunk
    for (int start = warp * kWarpChunk; start < nrec && !failed;) {
        const int64_t base = c0 + start;
        const int nc = min(csz, nrec - start);
        const uint32_t v = lane < nc ? __ldg(list + base + lane) : 0u;
        if (lane < nc) S.id[lane] = v;
        // stage the records: expect nc * sizeof(SegRec) bytes, then one bulk copy per record
        if (lane == 0) mbar_expect(&S.bar, (uint32_t)(nc * sizeof(SegRec)));
        __syncwarp();
        if (lane < nc) bulk_g2s(&S.rec[lane], rec + (v & ((1u << 26) - 1u)), (uint32_t)sizeof(SegRec), &S.bar);
        if (!mbar_wait(&S.bar, phase)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        int nrows = 0;
        if (lane < nc) {
            CandBox B;
            clip_box(S.rec[lane], v >> 26, N, x0, y0, z0, B);
            S.box[lane] = B;
            nrows = B.nrows;
        }
        // warp exclusive scan of the row counts; lane k holds the first row of candidate k
        int incl = nrows;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int rowoff = incl - nrows;
        const int total = __shfl_sync(0xffffffffu, incl, kWarpChunk - 1);
        __syncwarp();
        // Rows, one per lane: solve the row's index interval, test its points (rec_classify) in
        // lock step and queue the accepted ones and those left to the FP64 tests; every 32
        // queued points are evaluated with all lanes busy.
        for (int r0 = 0; r0 < total; r0 += 32) {
            const int r = r0 + lane;
            // candidate of row r: last k with rowoff_k <= r (binary search over the lanes)
            int k = 0;
#pragma unroll
            for (int step = kWarpChunk / 2; step > 0; step >>= 1) {
                const int t = k + step;
                const int ot = __shfl_sync(0xffffffffu, rowoff, t);
                if (t < nc && ot <= r) k = t;
            }
            const int rk = __shfl_sync(0xffffffffu, rowoff, k);
            int i = 1, ihi = 0, clo = 1, chi = 0;
            int a = 0, lb0 = 0, lb1 = 0, lb2 = 0;
            if (r < total) {
                const CandBox &B = S.box[k];
                const SegRec &R = S.rec[k];
                a = B.axis;
                const int rr = r - rk;
                // rows run over (b, c) = ((a+1)%3, (a+2)%3); per-axis offsets by selects
                const int nb = a == 0 ? B.n[1] : (a == 1 ? B.n[2] : B.n[0]);
                const int jc = (int)((float)rr * B.rnb), jb = rr - jc * nb;
                const int ex = a == 0 ? 0 : (a == 1 ? jc : jb);
                const int ey = a == 0 ? jb : (a == 1 ? 0 : jc);
                const int ez = a == 0 ? jc : (a == 1 ? jb : 0);
                lb0 = B.lo[0] + ex;
                lb1 = B.lo[1] + ey;
                lb2 = B.lo[2] + ez;
                const float d0x = fmaf((float)(B.dorg[0] + ex), R.dx, R.off[0]);
                const float d0y = fmaf((float)(B.dorg[1] + ey), R.dx, R.off[1]);
                const float d0z = fmaf((float)(B.dorg[2] + ez), R.dx, R.off[2]);
                const int na = a == 0 ? B.n[0] : (a == 1 ? B.n[1] : B.n[2]);
                int ilo;
                row_interval(R, B, d0x, d0y, d0z, a, na, ilo, ihi, clo, chi);
                i = ilo;
            }
            while (__any_sync(0xffffffffu, i <= ihi)) {
                bool ok = false;
                uint32_t code = 0;
                if (i <= ihi) {
                    const CandBox &B = S.box[k];
                    const SegRec &R = S.rec[k];
                    const int lx = lb0 + (a == 0 ? i : 0), ly = lb1 + (a == 1 ? i : 0), lz = lb2 + (a == 2 ? i : 0);
                    int cls = 1;   // the row's core passes for certain
                    if (F64 || i < clo || i > chi) {
                        const float d0x = fmaf((float)(lx + B.dl[0]), R.dx, R.off[0]);
                        const float d0y = fmaf((float)(ly + B.dl[1]), R.dx, R.off[1]);
                        const float d0z = fmaf((float)(lz + B.dl[2]), R.dx, R.off[2]);
                        if constexpr (F64) cls = rec_tests_wide(R, d0x, d0y, d0z) ? 1 : 0;
                        else cls = rec_classify(R, d0x, d0y, d0z, B.pe);
                    }
                    ok = cls != 0;
                    code = (uint32_t)k | ((uint32_t)lx << 4) | ((uint32_t)ly << 8) | ((uint32_t)lz << 11) |
                           (cls == 2 ? kQDecide : 0u);
                    ++i;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) S.q[qn + __popc(bal & ((1u << lane) - 1u))] = code;
                qn += __popc(bal);
                __syncwarp();
                if (qn >= 32) drain_queue<General, F64>(S, acc, lane, 32, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
            }
        }
        if (qn > 0) drain_queue<General, F64>(S, acc, lane, qn, qn, nacc, fscale, fmaxq, err, redo, D, x0, y0, z0);
        __syncwarp();   // the warp's stage is reused by its next chunk
        // the next chunk, guided self-scheduling: kWarpChunk candidates while many remain,
        // down to two near the end of the list, so that the warps reach the epilogue's
        // barrier close together (a thick tube's candidates cost a whole tile each)
        int nxt = 0, cs = 0;
        if (lane == 0) {
            const int rem = nrec - *(volatile int *)&next_rec;
            cs = max(2, min(kWarpChunk, rem / (2 * kDepWarps)));
            nxt = atomicAdd(&next_rec, cs);
        }
        start = __shfl_sync(0xffffffffu, nxt, 0);
        csz = __shfl_sync(0xffffffffu, cs, 0);
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


RedoCtx redo_ctx(const Ctx *c, const CenterlineBatch &B, double scale, bool pieces)
{
    RedoCtx r;
    r.lp = B.lp;
    r.slot_line = B.slot_line;
    r.map = B.rec_map;
    r.ntf = B.ntf;
    r.first = B.rec_first;
    r.qoff = B.qoff;
    r.seg = B.seg;
    r.tally = nullptr;
    r.X = c->d_x;
    r.Y = c->d_y;
    r.Z = c->d_z;
    r.cze = B.cze;
    r.coe = B.coe;
    r.dtf = B.dtf;
    r.node_base = B.node_base;
    r.N = c->p.N;
    r.pieces = pieces ? 1 : 0;
    r.zs = c->slab_nz ? c->slab_z0 : 0;
    r.nz = c->slab_nz ? c->slab_nz : c->p.N;
    r.Rtube_ratio = c->p.Rtube_ratio;
    r.dzeta_sup = c->p.dzeta_sup;
    r.eta = c->p.eta_t;
    r.scale = scale;
    return r;
}

double fixed_point_scale(const Ctx *c)
{
    // bound of one contribution: |Gamma| / (2 pi sigma_min^2), times a margin for the
    // curvature and core-variation terms; the sum of ~10^4 contributions still fits 2^63
    double b = 1e-30;
    for (int l = 0; l < c->nline; ++l) {
        const double s = c->sigma[l];
        if (s > 0) b = std::max(b, std::fabs(c->Gamma[l]) / (kPi2 * s * s));
    }
    b *= 16.0;
    const int e = (int)std::floor(48.0 - std::log2(b));
    return std::ldexp(1.0, e);
}

// ------------------------------------------------------------------ deferred pairs
// One thread per deferred pair: the reference's FP64 tests (decided pairs) and vorticity
// (redo_pair_f64), added as int64 fixed point into the side accumulator (kSideStride int64 per
// grid point: x, y, z and a pad, one 32-byte sector).
__global__ void __launch_bounds__(128) redo_apply_kernel(const RedoCtx R, const Deferred *__restrict__ e, int64_t n,
                                                         unsigned long long *__restrict__ side,
                                                         int *__restrict__ err)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool taken = false;
    if (i < n) {
        const Deferred d = e[i];
        const bool decide = (d.rec & kDeferDecide) != 0u;
        const int gx = (int)(d.gxy & 0xffffu), gy = (int)(d.gxy >> 16), gz = (int)d.gz;
        long long q[3];
        const int r = redo_pair_f64(R, d.rec & ((1u << 26) - 1u), (int)((d.rec >> 26) & 7u), decide, gx, gy, gz, q);
        if (r < 0) atomicOr(err, 4);
        if (r != 0) {
            const size_t g = (size_t)gx + (size_t)R.N * ((size_t)gy + (size_t)R.N * (size_t)(gz - R.zs));
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (q[k] != 0) atomicAdd(side + kSideStride * g + k, (unsigned long long)q[k]);
        }
        taken = decide && r != 0;
    }
    // tallies: decided pairs the FP64 tests accept (the cond pairs were counted by the tile
    // kernel), and every pair evaluated here
    const unsigned nt = __popc(__ballot_sync(0xffffffffu, taken));
    const unsigned nv = __popc(__ballot_sync(0xffffffffu, i < n));
    if ((threadIdx.x & 31) == 0 && R.tally) {
        if (nt) atomicAdd(R.tally, (unsigned long long)nt);
        if (nv) atomicAdd(R.tally + 1, (unsigned long long)nv);
    }
}

// omega += side / scale where side holds a sum (n3 grid points, three components of omega
// n3 apart), and side back to zero.
__global__ void side_fold_kernel(float *__restrict__ w, unsigned long long *__restrict__ side, size_t n3, double inv)
{
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < n3; g += (size_t)gridDim.x * blockDim.x) {
        ulonglong2 *s2 = reinterpret_cast<ulonglong2 *>(side + kSideStride * g);
        const ulonglong2 a = s2[0], b = s2[1];
        const long long v[3] = {(long long)a.x, (long long)a.y, (long long)b.x};
        if ((v[0] | v[1] | v[2]) == 0) continue;
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (v[d] != 0) w[(size_t)d * n3 + g] = (float)((double)w[(size_t)d * n3 + g] + (double)v[d] * inv);
        s2[0] = make_ulonglong2(0ull, 0ull);
        s2[1] = make_ulonglong2(0ull, 0ull);
    }
}

int defer_list(Ctx *c, int64_t units, double rate, DeferList &D)
{
    // 1.5 times the last launch's rate, between 1 Mi and 16 Mi pairs (256 MB) unless a larger
    // list is already held; an overflow is refilled in windows of work units (defer_finish)
    const double want = std::min(std::max(1.0 * (1 << 20), 1.5 * rate * (double)units), 1.0 * (1 << 24));
    const unsigned long long cap = std::min((unsigned long long)want, defer_max(c));
    FWT_TRY(buf_reserve(c, c->b_defer, 16 + sizeof(Deferred) * (size_t)cap));
    D.count = (unsigned long long *)c->b_defer.p;
    D.e = (Deferred *)((char *)c->b_defer.p + 16);
    D.cap = (c->b_defer.bytes - 16) / sizeof(Deferred);
    D.emit_only = 0;
    D.w0 = 0;
    D.w1 = ~0u;
    FWT_CUDA(cudaMemsetAsync(D.count, 0, sizeof(unsigned long long), c->stream));
    return 0;
}

int defer_grow(Ctx *c, unsigned long long n, DeferList &D)
{
    // the list's old entries are rewritten by the refill pass: a fresh buffer will do
    buf_free(c, c->b_defer);
    FWT_TRY(buf_reserve(c, c->b_defer, 16 + sizeof(Deferred) * (size_t)n));
    D.count = (unsigned long long *)c->b_defer.p;
    D.e = (Deferred *)((char *)c->b_defer.p + 16);
    D.cap = (c->b_defer.bytes - 16) / sizeof(Deferred);
    FWT_CUDA(cudaMemsetAsync(D.count, 0, sizeof(unsigned long long), c->stream));
    return 0;
}

void defer_rate(double &rate, unsigned long long n, int64_t units)
{
    if (units > 0) rate = std::max(1e-3, (double)n / (double)units);
}

int side_ensure(Ctx *c)
{
    const size_t bytes = kSideStride * field_elems(c) * sizeof(unsigned long long);
    if (!c->b_side.p || c->b_side.bytes < bytes) {
        buf_free(c, c->b_side);
        FWT_TRY(buf_reserve(c, c->b_side, bytes));
        FWT_CUDA(cudaMemsetAsync(c->b_side.p, 0, c->b_side.bytes, c->stream));
        c->side_dirty = false;
    }
    return 0;
}

int defer_apply(Ctx *c, const RedoCtx &R, const DeferList &D, unsigned long long n)
{
    if (n == 0) return 0;
    const size_t n3 = field_elems(c);
    FWT_TRY(side_ensure(c));
    FWT_TRY(buf_reserve(c, c->scratch[19], 128));
    int *d_err = (int *)((char *)c->scratch[19].p + 96);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const int km = kt_begin(c, KT_DEPOSIT);
    redo_apply_kernel<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(R, D.e, (int64_t)n,
                                                                          (unsigned long long *)c->b_side.p, d_err);
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    c->side_dirty = true;
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 4) return fail(FWT_E_RANGE, "deposit: FP64 contribution outside the fixed-point range");
    return 0;
}

int side_fold(Ctx *c)
{
    if (!c->side_dirty) return 0;
    const size_t n = field_elems(c);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int km = kt_begin(c, KT_DEPOSIT);
    side_fold_kernel<<<(unsigned)(sms * 8), 256, 0, c->stream>>>((float *)c->b_w.p, (unsigned long long *)c->b_side.p,
                                                                n, 1.0 / fixed_point_scale(c));
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    c->side_dirty = false;
    c->wmm_valid = false;
    return 0;
}

int launch_tile(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out)
{
    const int N = c->p.N;
    const int ntx = (N + TX - 1) / TX, nty = (N + TY - 1) / TY;
    // tiles of the context's planes: the whole grid, or its z-slab (whole tiles)
    const int tz0 = c->slab_nz ? c->slab_z0 / TZ : 0;
    const int ntz = c->slab_nz ? c->slab_nz / TZ : (N + TZ - 1) / TZ;
    const int64_t ntiles = (int64_t)ntx * nty * ntz;
    if (B.nsub >= ((int64_t)1 << 26)) return fail(FWT_E_RANGE, "sub-segment batch exceeds 2^26");
    if (!B.rec) return fail(FWT_E_STATE, "tile deposition needs the FP32 sub-segment records");
    Ctx &C = *c;
    // scratch[20]: pair counts/offsets (nsub+1 int64), [21]: key,val (2 x npairs u32),
    // [22]: tile counts u32 + cursor u32 + tile offsets i64, [23]: list u32
    FWT_TRY(buf_reserve(c, C.scratch[20], sizeof(int64_t) * (size_t)(B.nsub + 2) + 64));
    int64_t *d_cnt = (int64_t *)C.scratch[20].p;
    int *d_err = (int *)(d_cnt + B.nsub + 1);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const unsigned bq = (unsigned)((B.nsub + 255) / 256);
    int km = kt_begin(c, KT_BINNING);
    if (B.nsub > 0) pair_count_kernel<SegRec><<<bq, 256, 0, c->stream>>>(B.rec, B.nsub, N, tz0, ntz, d_cnt, d_err);
    FWT_TRY(scan_exclusive_i64(c, d_cnt, B.nsub, d_cnt + B.nsub, C.scratch[12]));
    kt_end(c, km);
    int64_t npairs = 0;
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&npairs, d_cnt + B.nsub, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr) return fail(FWT_E_RANGE, "sub-segment box wider than one periodic image (Rtube too large)");
    *pairs_out = npairs;
    FWT_TRY(buf_reserve(c, C.scratch[21], sizeof(uint32_t) * 2 * (size_t)std::max<int64_t>(npairs, 1)));
    uint32_t *d_key = (uint32_t *)C.scratch[21].p, *d_val = d_key + npairs;
    const size_t tb = sizeof(uint32_t) * (size_t)ntiles;
    FWT_TRY(buf_reserve(c, C.scratch[22], tb * 2 + sizeof(int64_t) * (size_t)(ntiles + 1) + 64));
    uint32_t *d_tcnt = (uint32_t *)C.scratch[22].p, *d_cur = d_tcnt + ntiles;
    int64_t *d_toff = (int64_t *)(((uintptr_t)(d_cur + ntiles) + 15) & ~(uintptr_t)15);
    FWT_CUDA(cudaMemsetAsync(d_tcnt, 0, tb * 2, c->stream));
    km = kt_begin(c, KT_BINNING);
    if (B.nsub > 0)
        pair_emit_kernel<SegRec><<<bq, 256, 0, c->stream>>>(B.rec, B.nsub, N, ntx, nty, tz0, ntz, d_cnt, d_key, d_val,
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
    RedoCtx rctx = redo_ctx(c, B, scale, false);
    rctx.tally = (unsigned long long *)((char *)C.scratch[19].p + 64);
    DeferList D{};
    if (!f64) FWT_TRY(defer_list(c, npairs, c->defer_per_pair, D));
    auto launch = [&](const DeferList &L) -> int {
#define FWT_TILE_LAUNCH(G, A, F)                                                                          \
    do {                                                                                                  \
        FWT_CUDA(cudaFuncSetAttribute(deposit_tile_kernel<G, A, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                      (int)kDepSmem));                                                    \
        deposit_tile_kernel<G, A, F><<<grid, kDepThreads, kDepSmem, c->stream>>>(                         \
            B.rec, N, ntx, nty, tz0, d_toff, d_list, scale, wx, wy, wz, d_err, rctx, L);                  \
        FWT_CUDA(cudaGetLastError());                                                                     \
    } while (0)
        const unsigned grid = (unsigned)(std::min<int64_t>(ntiles, L.w1) - L.w0);
        const int m = kt_begin(c, KT_DEPOSIT);
        if (f64) {
            // the FP64 path evaluates every pair in FP64: the General distinction is only the FP32 one
            if (accumulate) FWT_TILE_LAUNCH(true, true, true); else FWT_TILE_LAUNCH(true, false, true);
        } else if (general) {
            if (accumulate) FWT_TILE_LAUNCH(true, true, false); else FWT_TILE_LAUNCH(true, false, false);
        } else {
            if (accumulate) FWT_TILE_LAUNCH(false, true, false); else FWT_TILE_LAUNCH(false, false, false);
        }
#undef FWT_TILE_LAUNCH
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

}  // namespace fwt
