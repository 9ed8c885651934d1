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
//    of candidates.  Candidates are processed in double-buffered chunks: the ids of chunk i+2
//    arrive by a bulk asynchronous copy (cp.async.bulk, the TMA engine's 1-D form) and the
//    FP32 records of chunk i+1 by cp.async while chunk i is evaluated.  A chunk's work is
//    flattened into grid rows along each candidate's best-aligned axis; each row solves the
//    two half-space tests and the cylinder test of tube.f90:806-818 for its index interval
//    (one-point margin) and evaluates the reference predicate and vorticity only there, where
//    the reference walks the whole box (about 11 points per accepted one at these
//    sub-segment lengths).  The tile is written once with coalesced float4 stores; its
//    component min/max are folded into the epilogue.
#include "k_deposit.cuh"

namespace fwt {

constexpr int TX = 16, TY = 8, TZ = 8, TP = TX * TY * TZ;
constexpr int kCandChunk = 32;   // candidates per chunk (two chunks staged: ~44 KB of shared memory)
constexpr int kDepThreads = 256;
constexpr int kMaxRows = kCandChunk * 128;   // a clipped cross-section has at most 16 x 8 rows
constexpr int kRecVec = (int)(sizeof(SegRec) / 16);

__device__ __forceinline__ int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

__device__ __forceinline__ int axis_entries(int glo, int ghi, int N, int T)
{
    int cnt = 0;
    const int m0 = floordiv(glo, N), m1 = floordiv(ghi, N);
    for (int m = m0; m <= m1; ++m) {
        const int a = max(glo, m * N) - m * N, b = min(ghi, m * N + N - 1) - m * N;
        cnt += b / T - a / T + 1;
    }
    return cnt;
}

// Can the tile's points (unwrapped grid offsets o0..o0+n-1 from the record's box origin) pass
// t0 >= 0, t1 < 0 and rho < Rtube (tube.f90:806-818)?  Conservative: extremes of the linear
// tests over the tile's bounding box, and the box's distance to the chord line.
__device__ __forceinline__ bool tile_may_hit(const SegRec &R, int ox, int oy, int oz, int nx, int ny, int nz)
{
    const float dx = R.dx;
    const float hx = 0.5f * (nx - 1) * dx, hy = 0.5f * (ny - 1) * dx, hz = 0.5f * (nz - 1) * dx;
    const float cx = fmaf((float)ox, dx, R.off[0]) + hx, cy = fmaf((float)oy, dx, R.off[1]) + hy,
                cz = fmaf((float)oz, dx, R.off[2]) + hz;
    const float hn = sqrtf(hx * hx + hy * hy + hz * hz);
    const float Rt = sqrtf(R.R2);
    const float e = 1e-3f * (hn + Rt + dx);   // slack for the FP32 rounding of these bounds
    const float t0c = cx * R.tc0[0] + cy * R.tc0[1] + cz * R.tc0[2];
    const float t0h = hx * fabsf(R.tc0[0]) + hy * fabsf(R.tc0[1]) + hz * fabsf(R.tc0[2]);
    if (t0c + t0h < -e) return false;
    const float t1c = (cx - R.dci[0]) * R.tc1[0] + (cy - R.dci[1]) * R.tc1[1] + (cz - R.dci[2]) * R.tc1[2];
    const float t1h = hx * fabsf(R.tc1[0]) + hy * fabsf(R.tc1[1]) + hz * fabsf(R.tc1[2]);
    if (t1c - t1h > e) return false;
    const float d2 = fmaxf(cx * cx + cy * cy + cz * cz - t0c * t0c, 0.0f);
    const float rr = Rt + hn + e;
    return d2 <= rr * rr;
}

// Visit every (tile, image) of record S's box that may hold accepted points.
template <typename F>
__device__ __forceinline__ void for_each_tile(const SegRec &S, int N, F &&f)
{
    const int glo0 = S.box_lo[0] - 1, ghi0 = S.box_hi[0] - 1;
    const int glo1 = S.box_lo[1] - 1, ghi1 = S.box_hi[1] - 1;
    const int glo2 = S.box_lo[2] - 1, ghi2 = S.box_hi[2] - 1;
    for (int mz = floordiv(glo2, N); mz <= floordiv(ghi2, N); ++mz) {
        const int az = max(glo2, mz * N) - mz * N, bz = min(ghi2, mz * N + N - 1) - mz * N;
        for (int tz = az / TZ; tz <= bz / TZ; ++tz) {
            const int uz0 = max(tz * TZ + mz * N, glo2), uz1 = min(min(tz * TZ + TZ, N) - 1 + mz * N, ghi2);
            for (int my = floordiv(glo1, N); my <= floordiv(ghi1, N); ++my) {
                const int ay = max(glo1, my * N) - my * N, by = min(ghi1, my * N + N - 1) - my * N;
                for (int ty = ay / TY; ty <= by / TY; ++ty) {
                    const int uy0 = max(ty * TY + my * N, glo1), uy1 = min(min(ty * TY + TY, N) - 1 + my * N, ghi1);
                    for (int mx = floordiv(glo0, N); mx <= floordiv(ghi0, N); ++mx) {
                        const int ax = max(glo0, mx * N) - mx * N, bx = min(ghi0, mx * N + N - 1) - mx * N;
                        for (int tx = ax / TX; tx <= bx / TX; ++tx) {
                            const int ux0 = max(tx * TX + mx * N, glo0), ux1 = min(min(tx * TX + TX, N) - 1 + mx * N, ghi0);
                            if (!tile_may_hit(S, ux0 - glo0, uy0 - glo1, uz0 - glo2, ux1 - ux0 + 1, uy1 - uy0 + 1,
                                              uz1 - uz0 + 1))
                                continue;
                            f(tx, ty, tz, (uint32_t)((mx + 1) + 3 * (my + 1) + 9 * (mz + 1)));
                        }
                    }
                }
            }
        }
    }
}

template <typename Rec>
__global__ void pair_count_kernel(const Rec *__restrict__ seg, int64_t nsub, int N, int64_t *__restrict__ cnt,
                                  int *__restrict__ err)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub) return;
    const Rec &S = seg[q];
    int64_t c = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int glo = S.box_lo[d] - 1, ghi = S.box_hi[d] - 1;
        if (floordiv(glo, N) < -1 || floordiv(ghi, N) > 1 || ghi < glo) atomicOr(err, 1);
    }
    for_each_tile(S, N, [&](int, int, int, uint32_t) { ++c; });
    cnt[q] = c;
}

// warp-aggregated increment of tile_cnt[key]: consecutive sub-segments share tiles
__device__ __forceinline__ void agg_inc(uint32_t *cnt, uint32_t key, bool active)
{
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned peers = __match_any_sync(act, key);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(cnt + key, (uint32_t)__popc(peers));
}

template <typename Rec>
__global__ void pair_emit_kernel(const Rec *__restrict__ seg, int64_t nsub, int N, int ntx, int nty,
                                 const int64_t *__restrict__ off, uint32_t *__restrict__ key,
                                 uint32_t *__restrict__ val, uint32_t *__restrict__ tile_cnt)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = q < nsub;
    const Rec &S = seg[live ? q : 0];
    int64_t o = live ? off[q] : 0;
    // the first pair of each thread is counted through a warp-aggregated atomic below
    bool first = true;
    uint32_t k0 = 0;
    if (live)
        for_each_tile(S, N, [&](int tx, int ty, int tz, uint32_t img) {
            const uint32_t tile = (uint32_t)(tx + ntx * (ty + nty * tz));
            key[o] = tile;
            val[o] = (uint32_t)q | (img << 26);
            ++o;
            if (first) {
                first = false;
                k0 = tile;
                return;
            }
            atomicAdd(tile_cnt + tile, 1u);
        });
    agg_inc(tile_cnt, k0, live && !first);
}

__global__ void tile_scatter_kernel(const uint32_t *__restrict__ key, const uint32_t *__restrict__ val, int64_t n,
                                    const int64_t *__restrict__ tile_off, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ list)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const uint32_t t = live ? key[i] : 0u;
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
};

__device__ __forceinline__ void bulk_copy_g2s(void *smem, const void *gmem, uint32_t bytes, uint64_t *bar)
{
    // 1-D bulk asynchronous copy through the TMA engine, completion on an mbarrier
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s),
                 "l"(gmem), "r"(bytes), "r"(b)
                 : "memory");
}

// Wait for the mbarrier phase with a bounded spin; returns false if it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase)
{
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Index interval [ilo, ihi] (clamped to [0, n-1]) of the grid row d0 + i dx e_a that can pass
// t0 >= 0, t1 < 0 and rho^2 < R2; a one-point margin covers the FP32 rounding of the bounds.
__device__ __forceinline__ void row_interval(const SegRec &R, const CandBox &B, float d0x, float d0y, float d0z, int a,
                                             int n, int &ilo, int &ihi)
{
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
        nonempty = nonempty && B.n[d] > 0;
    }
    const float ax = fabsf(R.tc0[0]), ay = fabsf(R.tc0[1]), az = fabsf(R.tc0[2]);
    B.axis = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    B.nrows = nonempty ? B.n[(B.axis + 1) % 3] * B.n[(B.axis + 2) % 3] : 0;
    const float ta = R.tc0[B.axis], tb = R.tc1[B.axis], dx = R.dx;
    B.isa = 1.0f / (dx * ta);
    B.isb = fabsf(tb) > 0.05f ? 1.0f / (dx * tb) : 0.0f;
    const float q2 = dx * dx * (1.0f - ta * ta);
    B.q2 = q2 > 0.01f * dx * dx ? q2 : 0.0f;
    B.i2q = B.q2 > 0.0f ? 0.5f / B.q2 : 0.0f;
    B.rnb = nonempty ? 1.000001f / (float)B.n[(B.axis + 1) % 3] : 0.0f;
}

// Warp-autonomous tile deposition.  Each warp claims chunks of kWarpChunk candidates of the
// tile, stages their records in its own slice of shared memory with one bulk asynchronous
// copy per record (cp.async.bulk, completion on the warp's mbarrier), flattens the chunk's
// grid rows across its lanes, and adds into the CTA's fixed-point accumulators.  Only the
// accumulator set-up and the epilogue synchronise the whole CTA.
constexpr int kWarpChunk = 16;
constexpr int kDepWarps = kDepThreads / 32;
struct WarpStage {
    SegRec rec[kWarpChunk];
    CandBox box[kWarpChunk];
    uint64_t bar;
    uint64_t pad;
};
// Accumulator cell of tile point (x, y, z): x + kSY y + kSZ z.  A warp's lanes take adjacent
// rows, so along a y- or z-walk they hit cells kSY or kSZ apart; with both strides odd in
// 8-byte words the lanes spread over all shared-memory banks.
constexpr int kSY = TX + 1, kSZ = kSY * TY + 1, kAccN = kSZ * TZ;
constexpr size_t kDepSmem = sizeof(long long) * 3 * kAccN + sizeof(WarpStage) * kDepWarps;

template <bool General, bool Accumulate>
__global__ void __launch_bounds__(kDepThreads, 3) deposit_tile_kernel(
    const SegRec *__restrict__ rec, int N, int ntx, int nty, const int64_t *__restrict__ tile_off,
    const uint32_t *__restrict__ list, double scale, float *__restrict__ wx, float *__restrict__ wy,
    float *__restrict__ wz, uint32_t *__restrict__ mm, int *__restrict__ err)
{
    extern __shared__ __align__(16) unsigned char dsm[];
    long long(*acc)[kAccN] = reinterpret_cast<long long(*)[kAccN]>(dsm);
    const int tile = blockIdx.x;
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    WarpStage &S = reinterpret_cast<WarpStage *>(dsm + sizeof(long long) * 3 * kAccN)[warp];
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int p = tid; p < TP; p += kDepThreads) {
        const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
        const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
        long long a0 = 0, a1 = 0, a2 = 0;
        if (Accumulate && gx < N && gy < N && gz < N) {
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * gz);
            a0 = __double2ll_rn((double)wx[g] * scale);
            a1 = __double2ll_rn((double)wy[g] * scale);
            a2 = __double2ll_rn((double)wz[g] * scale);
        }
        const int pa = lx + kSY * ly + kSZ * lz;
        acc[0][pa] = a0;
        acc[1][pa] = a1;
        acc[2][pa] = a2;
    }
    __syncthreads();
    const int64_t c0 = tile_off[tile], c1 = tile_off[tile + 1];
    const int nchunks = (int)((c1 - c0 + kWarpChunk - 1) / kWarpChunk);
    const float fscale = (float)scale;
    const float fmaxq = 4.0e18f;
    uint32_t phase = 0;
    bool failed = false;
    for (int ch = warp; ch < nchunks && !failed; ch += kDepWarps) {
        const int64_t base = c0 + (int64_t)ch * kWarpChunk;
        const int nc = (c1 - base < kWarpChunk) ? (int)(c1 - base) : kWarpChunk;
        const uint32_t v = lane < nc ? __ldg(list + base + lane) : 0u;
        // stage the records: expect nc * sizeof(SegRec) bytes, then one bulk copy per record
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"((uint32_t)(nc * sizeof(SegRec)))
                         : "memory");
        __syncwarp();
        if (lane < nc) {
            const uint32_t q = v & ((1u << 26) - 1u);
            const uint32_t s = (uint32_t)__cvta_generic_to_shared(&S.rec[lane]);
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s),
                "l"(rec + q), "r"((uint32_t)sizeof(SegRec)), "r"(bar)
                : "memory");
        }
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
            if (r >= total) continue;
            const CandBox &B = S.box[k];
            const SegRec &R = S.rec[k];
            const int a = B.axis;
            const int rr = r - rk;
            // rows run over (b, c) = ((a+1)%3, (a+2)%3); per-axis offsets by selects (no
            // runtime-indexed local arrays)
            const int nb = a == 0 ? B.n[1] : (a == 1 ? B.n[2] : B.n[0]);
            const int jc = (int)((float)rr * B.rnb), jb = rr - jc * nb;
            const int ex = a == 0 ? 0 : (a == 1 ? jc : jb);
            const int ey = a == 0 ? jb : (a == 1 ? 0 : jc);
            const int ez = a == 0 ? jc : (a == 1 ? jb : 0);
            const float d0x = fmaf((float)(B.dorg[0] + ex), R.dx, R.off[0]);
            const float d0y = fmaf((float)(B.dorg[1] + ey), R.dx, R.off[1]);
            const float d0z = fmaf((float)(B.dorg[2] + ez), R.dx, R.off[2]);
            const int na = a == 0 ? B.n[0] : (a == 1 ? B.n[1] : B.n[2]);
            int ilo, ihi;
            row_interval(R, B, d0x, d0y, d0z, a, na, ilo, ihi);
            const int pstride = a == 0 ? 1 : (a == 1 ? kSY : kSZ);
            const int p0 = (B.lo[0] + ex) + kSY * (B.lo[1] + ey) + kSZ * (B.lo[2] + ez);
            const float sx = a == 0 ? R.dx : 0.f, sy = a == 1 ? R.dx : 0.f, sz = a == 2 ? R.dx : 0.f;
            for (int ii = ilo; ii <= ihi; ++ii) {
                float vv[3];
                const float fi = (float)ii;
                if (!point_rec<General>(R, fmaf(fi, sx, d0x), fmaf(fi, sy, d0y), fmaf(fi, sz, d0z), vv)) continue;
                const int p = p0 + ii * pstride;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float s = vv[d] * fscale;
                    if (!(fabsf(s) < fmaxq)) {
                        atomicOr(err, 4);
                        s = s != s ? 0.0f : copysignf(fmaxq, s);
                    }
                    atomicAdd((unsigned long long *)&acc[d][p], (unsigned long long)__float2ll_rn(s));
                }
            }
        }
        __syncwarp();   // the warp's stage is reused by its next chunk
    }
    if (failed && lane == 0) atomicOr(err, 2);
    __syncthreads();
    // epilogue: fixed point -> float, coalesced float4 stores, tile min/max per component
    const double inv = 1.0 / scale;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
    const bool full = (x0 + TX <= N) && (y0 + TY <= N) && (z0 + TZ <= N);
    float *w[3] = {wx, wy, wz};
    if (full) {
        for (int q4 = tid; q4 < TP / 4; q4 += kDepThreads) {
            const int p = 4 * q4;
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const size_t g = (size_t)(x0 + lx) + (size_t)N * ((size_t)(y0 + ly) + (size_t)N * (z0 + lz));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                float4 v4;
                const int pa = lx + kSY * ly + kSZ * lz;
                v4.x = (float)((double)acc[d][pa] * inv);
                v4.y = (float)((double)acc[d][pa + 1] * inv);
                v4.z = (float)((double)acc[d][pa + 2] * inv);
                v4.w = (float)((double)acc[d][pa + 3] * inv);
                *reinterpret_cast<float4 *>(w[d] + g) = v4;
                mn[d] = fminf(mn[d], fminf(fminf(v4.x, v4.y), fminf(v4.z, v4.w)));
                mx[d] = fmaxf(mx[d], fmaxf(fmaxf(v4.x, v4.y), fmaxf(v4.z, v4.w)));
            }
        }
    } else {
        for (int p = tid; p < TP; p += kDepThreads) {
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
            if (gx >= N || gy >= N || gz >= N) continue;
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * gz);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float v1 = (float)((double)acc[d][lx + kSY * ly + kSZ * lz] * inv);
                w[d][g] = v1;
                mn[d] = fminf(mn[d], v1);
                mx[d] = fmaxf(mx[d], v1);
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        for (int o2 = 16; o2 > 0; o2 >>= 1) {
            mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o2));
            mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o2));
        }
        if (lane == 0) {
            atomicMin(mm + 2 * d, f2ord(mn[d]));
            atomicMax(mm + 2 * d + 1, f2ord(mx[d]));
        }
    }
}


__global__ void mm_init_kernel(uint32_t *mm, int n)
{
    const int i = threadIdx.x;
    if (i < n) mm[i] = (i & 1) ? 0u : 0xffffffffu;
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

int launch_tile(Ctx *c, const CenterlineBatch &B, int64_t *pairs_out)
{
    const int N = c->p.N;
    const int ntx = (N + TX - 1) / TX, nty = (N + TY - 1) / TY, ntz = (N + TZ - 1) / TZ;
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
    if (B.nsub > 0) pair_count_kernel<SegRec><<<bq, 256, 0, c->stream>>>(B.rec, B.nsub, N, d_cnt, d_err);
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
        pair_emit_kernel<SegRec><<<bq, 256, 0, c->stream>>>(B.rec, B.nsub, N, ntx, nty, d_cnt, d_key, d_val, d_tcnt);
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

    const size_t n3 = field_elems(c);
    float *w = (float *)c->b_w.p;
    FWT_TRY(buf_reserve(c, C.scratch[19], 64));
    uint32_t *d_mm = (uint32_t *)((char *)C.scratch[19].p + 16);
    mm_init_kernel<<<1, 32, 0, c->stream>>>(d_mm, 6);
    const bool general = !(c->p.sigma_ratio == 1.0 && c->p.eta_t == 0.0);
    const bool accumulate = c->w_written;
    const double scale = fixed_point_scale(c);
    km = kt_begin(c, KT_DEPOSIT);
#define FWT_TILE_LAUNCH(G, A)                                                                              \
    do {                                                                                                   \
        FWT_CUDA(cudaFuncSetAttribute(deposit_tile_kernel<G, A>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                      (int)kDepSmem));                                                     \
        deposit_tile_kernel<G, A><<<(unsigned)ntiles, kDepThreads, kDepSmem, c->stream>>>(                \
            B.rec, N, ntx, nty, d_toff, d_list, scale, w, w + n3, w + 2 * n3, d_mm, d_err);                 \
    } while (0)
    if (general) {
        if (accumulate) FWT_TILE_LAUNCH(true, true); else FWT_TILE_LAUNCH(true, false);
    } else {
        if (accumulate) FWT_TILE_LAUNCH(false, true); else FWT_TILE_LAUNCH(false, false);
    }
#undef FWT_TILE_LAUNCH
    kt_end(c, km);
    // algorithmic bytes: omega written once (read too when accumulating), one candidate id
    // and one record per (tile, sub-segment) pair
    c->kbytes[KT_DEPOSIT] += (int64_t)(3 * n3 * 4 * (accumulate ? 2 : 1)) + npairs * (int64_t)(4 + sizeof(SegRec));
    c->launches += 2;
    FWT_CUDA(cudaGetLastError());
    c->w_written = true;
    uint32_t hmm[6];
    FWT_CUDA(cudaMemcpyAsync(hmm, d_mm, sizeof(hmm), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    if (herr & 2) return fail(FWT_E_TIMEOUT, "deposit: bulk copy wait ran out");
    if (herr & 4) return fail(FWT_E_RANGE, "deposit: contribution outside the fixed-point range");
    // every tile is rewritten in every batch, so the last batch's range is the field's range
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
