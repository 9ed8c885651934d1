// k_tile_common.cuh -- pieces shared by the tile-owned deposition kernels: the tile shape, the
// periodic tile walk of a record's box, the binning kernels, warp-aggregated counters, bulk
// asynchronous copies with bounded mbarrier waits, and the tile's int64 fixed-point
// accumulator (set-up and the coalesced epilogue).
#pragma once

#include "k_deposit.cuh"

namespace fwt {

constexpr int TX = 16, TY = 8, TZ = 8, TP = TX * TY * TZ;
constexpr int kDepThreads = 256;
constexpr int kDepWarps = kDepThreads / 32;

// Accumulator cell of tile point (x, y, z): x + kSY y + kSZ z.  Lanes working on adjacent
// rows hit cells kSY or kSZ apart; with both strides odd in 8-byte words the lanes spread
// over all shared-memory banks.
constexpr int kSY = TX + 1, kSZ = kSY * TY + 1, kAccN = kSZ * TZ;
constexpr size_t kAccBytes = sizeof(long long) * 3 * kAccN;

__device__ __forceinline__ int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Visit every (tile, periodic image) that the box [box_lo, box_hi] (1-based, unwrapped grid
// indices, at most one period beyond the domain on either side) overlaps and that `cull`
// does not rule out.  cull(ox, oy, oz, nx, ny, nz) receives the clipped part as offsets from
// box_lo and extents; f(tx, ty, tz, image) receives the tile and the image code
// (mx+1) + 3 (my+1) + 9 (mz+1).
template <typename C, typename F>
__device__ __forceinline__ void for_each_box_tile(const int *box_lo, const int *box_hi, int N, C &&cull, F &&f)
{
    const int glo0 = box_lo[0] - 1, ghi0 = box_hi[0] - 1;
    const int glo1 = box_lo[1] - 1, ghi1 = box_hi[1] - 1;
    const int glo2 = box_lo[2] - 1, ghi2 = box_hi[2] - 1;
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
                            if (!cull(ux0 - glo0, uy0 - glo1, uz0 - glo2, ux1 - ux0 + 1, uy1 - uy0 + 1, uz1 - uz0 + 1))
                                continue;
                            f(tx, ty, tz, (uint32_t)((mx + 1) + 3 * (my + 1) + 9 * (mz + 1)));
                        }
                    }
                }
            }
        }
    }
}

// warp-aggregated increment of cnt[key]: consecutive records share tiles
__device__ __forceinline__ void agg_inc(uint32_t *cnt, uint32_t key, bool active)
{
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned peers = __match_any_sync(act, key);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(cnt + key, (uint32_t)__popc(peers));
}

// Binning, step 1: number of (tile, image) pairs of every record (for_each_tile is overloaded
// per record type).  Boxes wider than one period beyond the domain set err bit 1.
template <typename Rec>
__global__ void pair_count_kernel(const Rec *__restrict__ seg, int64_t nsub, int N, int tz0, int ntz,
                                  int64_t *__restrict__ cnt, int *__restrict__ err)
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
    // tiles of the context's z-slab only (tz0 .. tz0 + ntz - 1; the whole grid by default)
    for_each_tile(S, N, [&](int, int, int tz, uint32_t) {
        if (tz >= tz0 && tz < tz0 + ntz) ++c;
    });
    cnt[q] = c;
}

constexpr uint32_t kNoTile = 0xffffffffu;   // key of a pair slot that the emitting pass left empty

// Binning, step 2: the (tile, record | image << 26) pairs at the record's offset, and the
// per-tile counts (warp-aggregated for the first tile of each record).  The pass writes only
// inside the record's slots [off[q], off[q+1]) reserved by step 1 and marks any slot it leaves
// empty, so the sort stays in bounds even if the two passes ever decided a tile differently.
template <typename Rec>
__global__ void pair_emit_kernel(const Rec *__restrict__ seg, int64_t nsub, int N, int ntx, int nty, int tz0, int ntz,
                                 const int64_t *__restrict__ off, uint32_t *__restrict__ key,
                                 uint32_t *__restrict__ val, uint32_t *__restrict__ tile_cnt)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = q < nsub;
    const Rec &S = seg[live ? q : 0];
    int64_t o = live ? off[q] : 0;
    const int64_t end = live ? off[q + 1] : 0;
    // the first pair of each thread is counted through a warp-aggregated atomic below
    bool first = true;
    uint32_t k0 = 0;
    if (live)
        for_each_tile(S, N, [&](int tx, int ty, int tz, uint32_t img) {
            if (o >= end || tz < tz0 || tz >= tz0 + ntz) return;
            const uint32_t tile = (uint32_t)(tx + ntx * (ty + nty * (tz - tz0)));
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
    for (; o < end; ++o) key[o] = kNoTile;
    agg_inc(tile_cnt, k0, live && !first);
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

__device__ __forceinline__ void mbar_init(uint64_t *bar)
{
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes)
{
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
}

// 1-D bulk asynchronous copy (TMA engine) of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *smem, const void *gmem, uint32_t bytes, uint64_t *bar)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(s),
                 "l"(gmem), "r"(bytes), "r"(b)
                 : "memory");
}

// Load the tile's current values into the fixed-point cells (Accumulate) or zero them.
// The field holds planes zs .. zlim - 1 (the whole grid: zs = 0, zlim = N; a z-slab context:
// its slab), plane gz stored at gz - zs.
template <bool Accumulate>
__device__ __forceinline__ void tile_acc_init(long long (*acc)[kAccN], int N, int x0, int y0, int z0, int zs,
                                              int zlim, double scale, const float *__restrict__ wx,
                                              const float *__restrict__ wy, const float *__restrict__ wz)
{
    for (int p = threadIdx.x; p < TP; p += blockDim.x) {
        const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
        const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
        long long a0 = 0, a1 = 0, a2 = 0;
        if (Accumulate && gx < N && gy < N && gz < zlim) {
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * (gz - zs));
            a0 = __double2ll_rn((double)wx[g] * scale);
            a1 = __double2ll_rn((double)wy[g] * scale);
            a2 = __double2ll_rn((double)wz[g] * scale);
        }
        const int pa = lx + kSY * ly + kSZ * lz;
        acc[0][pa] = a0;
        acc[1][pa] = a1;
        acc[2][pa] = a2;
    }
}

// Fixed point -> float, coalesced float4 stores of the tile.
__device__ __forceinline__ void tile_epilogue(long long (*acc)[kAccN], int N, int x0, int y0, int z0, int zs, int zlim,
                                              double scale, float *__restrict__ wx, float *__restrict__ wy,
                                              float *__restrict__ wz)
{
    const int tid = threadIdx.x;
    const double inv = 1.0 / scale;
    const bool full = (x0 + TX <= N) && (y0 + TY <= N) && (z0 + TZ <= zlim);
    if (full) {
        for (int q4 = tid; q4 < TP / 4; q4 += blockDim.x) {
            const int p = 4 * q4;
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const size_t g = (size_t)(x0 + lx) + (size_t)N * ((size_t)(y0 + ly) + (size_t)N * (z0 + lz - zs));
            const int pa = lx + kSY * ly + kSZ * lz;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                float4 v4;
                v4.x = (float)((double)acc[d][pa] * inv);
                v4.y = (float)((double)acc[d][pa + 1] * inv);
                v4.z = (float)((double)acc[d][pa + 2] * inv);
                v4.w = (float)((double)acc[d][pa + 3] * inv);
                float *w = d == 0 ? wx : (d == 1 ? wy : wz);
                *reinterpret_cast<float4 *>(w + g) = v4;
            }
        }
    } else {
        for (int p = tid; p < TP; p += blockDim.x) {
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
            if (gx >= N || gy >= N || gz >= zlim) continue;
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * (gz - zs));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float v1 = (float)((double)acc[d][lx + kSY * ly + kSZ * lz] * inv);
                float *w = d == 0 ? wx : (d == 1 ? wy : wz);
                w[g] = v1;
            }
        }
    }
}

// FP64 tile cells (the FP64 tile path): load the tile's current values or zero them.
template <bool Accumulate>
__device__ __forceinline__ void tile_acc_init_f64(double (*acc)[kAccN], int N, int x0, int y0, int z0, int zs, int zlim,
                                                  const double *__restrict__ wx, const double *__restrict__ wy,
                                                  const double *__restrict__ wz)
{
    for (int p = threadIdx.x; p < TP; p += blockDim.x) {
        const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
        const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        if (Accumulate && gx < N && gy < N && gz < zlim) {
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * (gz - zs));
            a0 = wx[g];
            a1 = wy[g];
            a2 = wz[g];
        }
        const int pa = lx + kSY * ly + kSZ * lz;
        acc[0][pa] = a0;
        acc[1][pa] = a1;
        acc[2][pa] = a2;
    }
}

// FP64 tile store (coalesced double2 stores).
__device__ __forceinline__ void tile_epilogue_f64(double (*acc)[kAccN], int N, int x0, int y0, int z0, int zs, int zlim,
                                                  double *__restrict__ wx, double *__restrict__ wy,
                                                  double *__restrict__ wz)
{
    const int tid = threadIdx.x;
    const bool full = (x0 + TX <= N) && (y0 + TY <= N) && (z0 + TZ <= zlim);
    if (full) {
        for (int q2 = tid; q2 < TP / 2; q2 += blockDim.x) {
            const int p = 2 * q2;
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const size_t g = (size_t)(x0 + lx) + (size_t)N * ((size_t)(y0 + ly) + (size_t)N * (z0 + lz - zs));
            const int pa = lx + kSY * ly + kSZ * lz;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                double2 v2;
                v2.x = acc[d][pa];
                v2.y = acc[d][pa + 1];
                double *w = d == 0 ? wx : (d == 1 ? wy : wz);
                *reinterpret_cast<double2 *>(w + g) = v2;
            }
        }
    } else {
        for (int p = tid; p < TP; p += blockDim.x) {
            const int lx = p % TX, ly = (p / TX) % TY, lz = p / (TX * TY);
            const int gx = x0 + lx, gy = y0 + ly, gz = z0 + lz;
            if (gx >= N || gy >= N || gz >= zlim) continue;
            const size_t g = (size_t)gx + (size_t)N * ((size_t)gy + (size_t)N * (gz - zs));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const double v1 = acc[d][lx + kSY * ly + kSZ * lz];
                double *w = d == 0 ? wx : (d == 1 ? wy : wz);
                w[g] = v1;
            }
        }
    }
}

// The FP64 tile path's evaluation of a candidate pair: the reference's FP64 tests of
// tube.f90:806-818 at the 1-based unwrapped grid index (ip, jp, kp) of sub-segment q's own box,
// and, if it passes, the reference's FP64 vorticity (tube.f90:819-892) added into the double
// cell p.
__device__ __forceinline__ bool eval_pair_f64(const RedoCtx &R, int64_t q, int ip, int jp, int kp,
                                              double (*acc)[kAccN], int p)
{
    const SubSeg &S = R.seg[q];
    double m[3], t0, t1;
    ref_mesh_f64(dev_pi2() / R.N, ip, jp, kp, m);
    if (!ref_tests_f64(S, m, t0, t1)) return false;
    const int slot = S.slot;
    const LineParam P = R.lp[R.slot_line[slot]];
    double v[3];
    ref_value_f64(S, P, R.coe + 18 * (size_t)slot, R.dtf[slot], R.dzeta_sup, R.eta, m, t0, t1, v);
#pragma unroll
    for (int d = 0; d < 3; ++d) atomicAdd(&acc[d][p], v[d]);
    return true;
}

// Index along one axis in the box of a sub-segment whose lower corner is lo, of the grid
// point with unwrapped index i in another frame (the two differ by whole periods).
__device__ __forceinline__ int box_index(int i, int lo, int N)
{
    int o = (i - lo) % N;
    if (o < 0) o += N;
    return lo + o;
}




// ---------------------------------------------------------------- pairs deferred to FP64
// Two kinds of (point, chord) pairs are not evaluated by the FP32 tile kernels:
// * accepted pairs whose curved-branch amplification |1/(1 - kappa rho cos theta)| exceeds
//   kRedoCond (tube.f90:876-879: the FP32 value carries the amplified rounding of kappa, rho and
//   cos theta); only tubes with a varying core or a twist have that term;
// * pairs with a plane test within its FP32 rounding bound of zero (the decide bit), which the
//   reference's FP64 tests decide.
// The kernels append them to a global list (a warp-aggregated counter; every pair is counted,
// stored or not); after the kernel, redo_apply_kernel evaluates each in the reference's FP64
// arithmetic (redo_pair_f64) and adds its int64 fixed-point contribution into a side
// accumulator, which side_fold adds into omega once the batch loop is done.  Integer sums make
// the field independent of the order; no FP64 code, and so no call, sits in the FP32 kernels.
// A list that overflows is refilled by a second, emit-only pass of the same kernel at the
// counted size.
struct Deferred {
    uint32_t rec;   // record id | chord << 26 | kDeferDecide
    uint32_t gxy;   // grid point x | y << 16 (0-based, wrapped)
    uint32_t gz;    // grid plane z (0-based, global)
    uint32_t pad;
};
constexpr uint32_t kDeferDecide = 1u << 31;
// int64 words per grid point of the side accumulator: x, y, z and a pad, so that the three
// reductions of a pair meet one 32-byte sector (three arrays would touch three, each a DRAM
// read-modify-write when the accumulator is larger than L2)
constexpr size_t kSideStride = 4;

struct DeferList {
    Deferred *e = nullptr;
    unsigned long long *count = nullptr;   // pairs pushed (may exceed cap)
    unsigned long long cap = 0;
    int emit_only = 0;                     // 1: a refill pass after an overflow (no field update)
    // the refill pass's window of work units [w0, w1) (tiles, or chunks of pieces); the
    // first pass covers every unit
    uint32_t w0 = 0, w1 = ~0u;
};

// Append the lanes' flagged pairs (warp-uniform call).
__device__ __forceinline__ void defer_push(const DeferList &D, int lane, bool flag, uint32_t rec, int gx, int gy,
                                           int gz)
{
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    if (bal == 0u) return;
    const int leader = __ffs(bal) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(D.count, (unsigned long long)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (flag) {
        const unsigned long long i = base + (unsigned long long)__popc(bal & ((1u << lane) - 1u));
        if (i < D.cap) D.e[i] = Deferred{rec, (uint32_t)gx | ((uint32_t)gy << 16), (uint32_t)gz, 0u};
    }
}

// The redo context of a batch (records: sub-segments, or chord pieces when `pieces`).
RedoCtx redo_ctx(const Ctx *c, const CenterlineBatch &B, double scale, bool pieces);

// The deferred-pair list of a launch over `units` work units ((tile, record) pairs, or pieces),
// sized from the running rate of deferred pairs per unit (k_deposit_tile.cu).
int defer_list(Ctx *c, int64_t units, double rate, DeferList &D);
// The side accumulator (kSideStride int64 per grid point), allocated and zeroed on first use.
int side_ensure(Ctx *c);

// Evaluate the first n pairs of the list in FP64 into the side accumulator (k_deposit_tile.cu).
int defer_apply(Ctx *c, const RedoCtx &R, const DeferList &D, unsigned long long n);
// Replace the list by one of n entries (its old entries are not kept) and reset its count.
int defer_grow(Ctx *c, unsigned long long n, DeferList &D);
void defer_rate(double &rate, unsigned long long n, int64_t units);
// Entries of the largest list an overflow grows to (1 GiB, or the context's tuning): a launch
// that defers more pairs refills its list in windows of work units.
constexpr unsigned long long kDeferMaxEntries = 1ull << 26;
inline unsigned long long defer_max(const Ctx *c)
{
    if (c->defer_max_pairs >= 1.0) return (unsigned long long)c->defer_max_pairs;
    // under a memory cap: a sixteenth of it
    if (c->p.mem_cap) return std::max(1ull << 16, std::min(kDeferMaxEntries, (unsigned long long)(c->p.mem_cap / 256)));
    return kDeferMaxEntries;
}

// After a launch over `units` work units (the rate's denominator) of which `wunits` can be
// windowed (tiles, or chunks of pieces): read the list's count and, when nothing overflowed,
// evaluate every deferred pair in FP64 into the side accumulator.  After an overflow the list
// is grown (up to kDeferMaxEntries) and refilled by rescan(D), the same launch in emit-only
// mode over a window of units at a time; each window's pairs are evaluated before the next is
// listed.  A unit's pairs are listed in the same order-independent way by every pass, so the
// windows together hold each counted pair once.
template <typename F>
int defer_finish(Ctx *c, const RedoCtx &R, DeferList &D, int64_t units, double &rate, int64_t wunits, F &&rescan)
{
    auto read_count = [&](unsigned long long &n) -> int {
        FWT_CUDA(cudaMemcpyAsync(&n, D.count, sizeof(n), cudaMemcpyDeviceToHost, c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
        return 0;
    };
    unsigned long long n = 0;
    FWT_TRY(read_count(n));
    defer_rate(rate, n, units);
    if (n == 0) return 0;
    if (n <= D.cap) return defer_apply(c, R, D, n);
    const unsigned long long want = std::min(n + n / 8, defer_max(c));
    if (want > D.cap) FWT_TRY(defer_grow(c, want, D));
    D.emit_only = 1;
    unsigned long long done = 0;
    int64_t u = 0;
    // window width in units, from the mean count per unit, for a list three quarters full
    double width = std::max(1.0, (double)wunits * 0.75 * (double)D.cap / (double)n);
    int rc = 0;
    while (u < wunits && rc == 0) {
        const int64_t w1 = std::min<int64_t>(wunits, u + (int64_t)width);
        D.w0 = (uint32_t)u;
        D.w1 = (uint32_t)w1;
        FWT_CUDA(cudaMemsetAsync(D.count, 0, sizeof(unsigned long long), c->stream));
        if ((rc = rescan(D)) != 0) break;
        unsigned long long m = 0;
        if ((rc = read_count(m)) != 0) break;
        if (m > D.cap) {
            if (w1 - u > 1) {   // narrower window: the counted pairs scaled to half the list
                width = std::max(1.0, (double)(w1 - u) * 0.5 * (double)D.cap / (double)m);
                continue;
            }
            // one unit holds more pairs than the list: make room for them and list it again
            if ((rc = defer_grow(c, m + m / 8, D)) != 0) break;
            continue;
        }
        if ((rc = defer_apply(c, R, D, m)) != 0) break;
        done += m;
        const double scaled = (double)(w1 - u) * 0.75 * (double)D.cap / (double)std::max(m, 1ull);
        width = std::max(1.0, std::min(2.0 * (double)(w1 - u), scaled));
        u = w1;
    }
    D.emit_only = 0;
    D.w0 = 0;
    D.w1 = ~0u;
    if (rc) return rc;
    if (done != n) return fail(FWT_E_STATE, "deferred pairs: the refill passes counted a different number");
    return 0;
}

// Shared kernels of the binning (defined in k_deposit_tile.cu).
__global__ void tile_scatter_kernel(const uint32_t *__restrict__ key, const uint32_t *__restrict__ val, int64_t n,
                                    const int64_t *__restrict__ tile_off, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ list);
__global__ void u32_to_i64_kernel(const uint32_t *__restrict__ a, int64_t n, int64_t *__restrict__ b);

// Scale of the int64 fixed-point tile sums for the context's lines.
double fixed_point_scale(const Ctx *c);

}  // namespace fwt
