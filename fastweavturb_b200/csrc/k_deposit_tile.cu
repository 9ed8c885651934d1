// k_deposit_tile.cu -- tile-owned Burgers-tube deposition with integer cell lists.
//
// 1. pair_count / pair_emit: every sub-segment's box (tube.f90:793-798) is cut into the
//    grid tiles it overlaps (periodic images kept apart), giving (tile, sub-segment|image)
//    pairs in sub-segment order.
// 2. counting sort by tile: integer histogram, exclusive scan, scatter -> per-tile
//    candidate lists (each list holds exactly the sub-segments whose box meets the tile).
// 3. deposit_tile_kernel: one CTA per tile.  Candidate ids are staged in shared memory with
//    a bulk asynchronous copy (cp.async.bulk, the TMA engine's 1-D form); per chunk each
//    candidate's FP32 local frame is built once, then warps walk the candidates' boxes
//    clipped to the tile and add contributions into shared int64 fixed-point accumulators.
//    Integer addition is associative, so the tile sum is bit-exact whatever the order of
//    candidates.  The tile is written once with coalesced float4 stores, and the tile's
//    component min/max are folded into the epilogue for the PDFs.
#include "k_deposit.cuh"

namespace fwt {

constexpr int TX = 16, TY = 8, TZ = 8, TP = TX * TY * TZ;
constexpr int kCandChunk = 64;
constexpr int kDepThreads = 256;

__device__ __forceinline__ int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

struct AxisSpan {
    int n;           // number of (image, tile) entries along this axis
};

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

__global__ void pair_count_kernel(const SubSeg *__restrict__ seg, int64_t nsub, int N, int64_t *__restrict__ cnt,
                                  int *__restrict__ err)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub) return;
    const SubSeg &S = seg[q];
    int64_t c = 1;
    const int T[3] = {TX, TY, TZ};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int glo = S.box_lo[d] - 1, ghi = S.box_hi[d] - 1;
        if (floordiv(glo, N) < -1 || floordiv(ghi, N) > 1 || ghi < glo) atomicOr(err, 1);
        c *= axis_entries(glo, ghi, N, T[d]);
    }
    cnt[q] = c;
}

__global__ void pair_emit_kernel(const SubSeg *__restrict__ seg, int64_t nsub, int N, int ntx, int nty,
                                 const int64_t *__restrict__ off, uint32_t *__restrict__ key,
                                 uint32_t *__restrict__ val, uint32_t *__restrict__ tile_cnt)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub) return;
    const SubSeg &S = seg[q];
    int64_t o = off[q];
    const int glo0 = S.box_lo[0] - 1, ghi0 = S.box_hi[0] - 1;
    const int glo1 = S.box_lo[1] - 1, ghi1 = S.box_hi[1] - 1;
    const int glo2 = S.box_lo[2] - 1, ghi2 = S.box_hi[2] - 1;
    for (int mz = floordiv(glo2, N); mz <= floordiv(ghi2, N); ++mz) {
        const int az = max(glo2, mz * N) - mz * N, bz = min(ghi2, mz * N + N - 1) - mz * N;
        for (int tz = az / TZ; tz <= bz / TZ; ++tz)
            for (int my = floordiv(glo1, N); my <= floordiv(ghi1, N); ++my) {
                const int ay = max(glo1, my * N) - my * N, by = min(ghi1, my * N + N - 1) - my * N;
                for (int ty = ay / TY; ty <= by / TY; ++ty)
                    for (int mx = floordiv(glo0, N); mx <= floordiv(ghi0, N); ++mx) {
                        const int ax = max(glo0, mx * N) - mx * N, bx = min(ghi0, mx * N + N - 1) - mx * N;
                        for (int tx = ax / TX; tx <= bx / TX; ++tx) {
                            const uint32_t tile = (uint32_t)(tx + ntx * (ty + nty * tz));
                            const uint32_t img = (uint32_t)((mx + 1) + 3 * (my + 1) + 9 * (mz + 1));
                            key[o] = tile;
                            val[o] = (uint32_t)q | (img << 26);
                            ++o;
                            atomicAdd(tile_cnt + tile, 1u);
                        }
                    }
            }
    }
}

__global__ void tile_scatter_kernel(const uint32_t *__restrict__ key, const uint32_t *__restrict__ val, int64_t n,
                                    const int64_t *__restrict__ tile_off, uint32_t *__restrict__ cursor,
                                    uint32_t *__restrict__ list)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = key[i];
    const uint32_t r = atomicAdd(cursor + t, 1u);
    list[tile_off[t] + r] = val[i];
}

__global__ void u32_to_i64_kernel(const uint32_t *__restrict__ a, int64_t n, int64_t *__restrict__ b)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

// -------------------------------------------------------------------------------- deposit
struct CandBox {
    int lo[3];    // clipped box origin, tile-local coordinates
    int n[3];     // clipped box extent
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

template <bool General, bool Accumulate>
__global__ void __launch_bounds__(kDepThreads) deposit_tile_kernel(
    const SubSeg *__restrict__ seg, const LineParam *__restrict__ lp, int line_base, const double *__restrict__ coe,
    const double *__restrict__ dtf, int N, int ntx, int nty, double dzeta_sup, double eta,
    const int64_t *__restrict__ tile_off, const uint32_t *__restrict__ list, double scale, float *__restrict__ wx,
    float *__restrict__ wy, float *__restrict__ wz, uint32_t *__restrict__ mm, int *__restrict__ err)
{
    __shared__ long long acc[3][TP];
    __shared__ SegF cand[kCandChunk];
    __shared__ CandBox cbox[kCandChunk];
    __shared__ __align__(16) uint32_t ids[kCandChunk + 4];
    __shared__ __align__(8) uint64_t bar;
    const int tile = blockIdx.x;
    const int tx = tile % ntx, ty = (tile / ntx) % nty, tz = tile / (ntx * nty);
    const int x0 = tx * TX, y0 = ty * TY, z0 = tz * TZ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // initialise accumulators
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
        acc[0][p] = a0;
        acc[1][p] = a1;
        acc[2][p] = a2;
    }
    __syncthreads();
    const int64_t c0 = tile_off[tile], c1 = tile_off[tile + 1];
    uint32_t phase = 0;
    const float fscale = (float)scale;
    const float fmaxq = 4.0e18f;
    for (int64_t cb = c0; cb < c1; cb += kCandChunk) {
        const int nc = (c1 - cb < kCandChunk) ? (int)(c1 - cb) : kCandChunk;
        // stage the candidate ids: bulk copy of the 16-byte aligned window, else plain loads
        const int64_t a16 = cb & ~(int64_t)3;          // 4 uint32 = 16 bytes
        const int skip = (int)(cb - a16);
        const int nw = (skip + nc + 3) & ~3;
        if (tid == 0) bulk_copy_g2s(ids, list + a16, (uint32_t)(nw * 4), &bar);
        const bool ok = mbar_wait(&bar, phase);
        if (__syncthreads_or(!ok)) {   // every thread leaves together if any wait ran out
            if (tid == 0) atomicOr(err, 2);
            return;
        }
        phase ^= 1u;
        // per-candidate set-up: FP64 -> FP32 local frame and the box clipped to the tile
        if (tid < nc) {
            const uint32_t v = ids[skip + tid];
            const uint32_t q = v & ((1u << 26) - 1u), img = v >> 26;
            const int m[3] = {(int)(img % 3) - 1, (int)((img / 3) % 3) - 1, (int)(img / 9) - 1};
            const SubSeg S = seg[q];
            const int tl[3] = {x0, y0, z0}, te[3] = {TX, TY, TZ};
            CandBox B;
            int org[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                // unwrapped 0-based span of the tile for image m: [tl + mN, tl + te - 1 + mN]
                const int ulo = tl[d] + m[d] * N, uhi = min(tl[d] + te[d] - 1, N - 1) + m[d] * N;
                const int lo = max(ulo, S.box_lo[d] - 1), hi = min(uhi, S.box_hi[d] - 1);
                B.lo[d] = lo - ulo;
                B.n[d] = max(0, hi - lo + 1);
                org[d] = lo + 1;   // 1-based unwrapped index of the clipped box origin
            }
            cbox[tid] = B;
            seg_setup_f32(S, lp[S.line - line_base], coe, dtf[S.slot], dzeta_sup, eta, N, org[0], org[1], org[2],
                          cand[tid]);
        }
        __syncthreads();
        for (int k = warp; k < nc; k += kDepThreads / 32) {
            const CandBox B = cbox[k];
            const int tot = B.n[0] * B.n[1] * B.n[2];
            for (int idx = lane; idx < tot; idx += 32) {
                const int ii = idx % B.n[0], r = idx / B.n[0];
                const int jj = r % B.n[1], kk = r / B.n[1];
                float o[3];
                if (!point_f32<General>(cand[k], ii, jj, kk, o)) continue;
                const int p = (B.lo[0] + ii) + TX * ((B.lo[1] + jj) + TY * (B.lo[2] + kk));
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    float s = o[d] * fscale;
                    if (!(fabsf(s) < fmaxq)) {
                        atomicOr(err, 4);
                        s = s != s ? 0.0f : copysignf(fmaxq, s);
                    }
                    atomicAdd((unsigned long long *)&acc[d][p], (unsigned long long)__float2ll_rn(s));
                }
            }
        }
        __syncthreads();
    }
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
                float4 v;
                v.x = (float)((double)acc[d][p] * inv);
                v.y = (float)((double)acc[d][p + 1] * inv);
                v.z = (float)((double)acc[d][p + 2] * inv);
                v.w = (float)((double)acc[d][p + 3] * inv);
                *reinterpret_cast<float4 *>(w[d] + g) = v;
                mn[d] = fminf(mn[d], fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
                mx[d] = fmaxf(mx[d], fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
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
                const float v = (float)((double)acc[d][p] * inv);
                w[d][g] = v;
                mn[d] = fminf(mn[d], v);
                mx[d] = fmaxf(mx[d], v);
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
    Ctx &C = *c;
    // scratch[20]: pair counts/offsets (nsub+1 int64), [21]: key,val (2 x npairs u32),
    // [22]: tile counts u32 + tile offsets i64 + cursor u32, [23]: list u32
    FWT_TRY(buf_reserve(c, C.scratch[20], sizeof(int64_t) * (size_t)(B.nsub + 2) + 64));
    int64_t *d_cnt = (int64_t *)C.scratch[20].p;
    int *d_err = (int *)(d_cnt + B.nsub + 1);
    FWT_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), c->stream));
    const unsigned bq = (unsigned)((B.nsub + 255) / 256);
    if (B.nsub > 0) pair_count_kernel<<<bq, 256, 0, c->stream>>>(B.seg, B.nsub, N, d_cnt, d_err);
    FWT_TRY(scan_exclusive_i64(c, d_cnt, B.nsub, d_cnt + B.nsub, C.scratch[12]));
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
    if (B.nsub > 0)
        pair_emit_kernel<<<bq, 256, 0, c->stream>>>(B.seg, B.nsub, N, ntx, nty, d_cnt, d_key, d_val, d_tcnt);
    u32_to_i64_kernel<<<(unsigned)((ntiles + 255) / 256), 256, 0, c->stream>>>(d_tcnt, ntiles, d_toff);
    FWT_TRY(scan_exclusive_i64(c, d_toff, ntiles, d_toff + ntiles, C.scratch[13]));
    FWT_TRY(buf_reserve(c, C.scratch[23], sizeof(uint32_t) * (size_t)(npairs + 8)));
    uint32_t *d_list = (uint32_t *)C.scratch[23].p;
    if (npairs > 0)
        tile_scatter_kernel<<<(unsigned)((npairs + 255) / 256), 256, 0, c->stream>>>(d_key, d_val, npairs, d_toff,
                                                                                     d_cur, d_list);
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
#define FWT_TILE_LAUNCH(G, A)                                                                              \
    deposit_tile_kernel<G, A><<<(unsigned)ntiles, kDepThreads, 0, c->stream>>>(                           \
        B.seg, B.lp, B.la, B.coe, B.dtf, N, ntx, nty, c->p.dzeta_sup, c->p.eta_t, d_toff, d_list, scale, w, \
        w + n3, w + 2 * n3, d_mm, d_err)
    if (general) {
        if (accumulate) FWT_TILE_LAUNCH(true, true); else FWT_TILE_LAUNCH(true, false);
    } else {
        if (accumulate) FWT_TILE_LAUNCH(false, true); else FWT_TILE_LAUNCH(false, false);
    }
#undef FWT_TILE_LAUNCH
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
