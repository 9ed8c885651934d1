// k_deposit.cu -- Burgers vortex-tube deposition (tube.f90:762-904).
//
// Two kernels share the per-point arithmetic:
//   * deposit_walk_kernel  -- the reference's box walk, one warp per sub-segment, global
//     atomics.  Templated on FP64 (the plain FP64 GPU path, statement-for-statement the
//     reference arithmetic) and FP32.
//   * deposit_tile_kernel  -- (k_deposit_tile.cu) tile-owned: sub-segments binned into
//     integer cell lists, each CTA owns a grid tile, accumulates in shared memory and writes
//     the tile once with coalesced vector stores.
//
// FP32 arithmetic is done in a frame local to the sub-segment start ci0: grid-point offsets
// x - ci0, and the spline re-expanded around the start, c(z0 + W) - c(z0) = sum_k b_k W^k
// (Taylor shift of the quintic in FP64), so no FP32 quantity carries the absolute position.
#include <cstdio>
#include <cstdlib>

#include "k_deposit.cuh"

namespace fwt {

// Reference box walk: one warp per sub-segment; lanes stride the box points in the
// reference's loop order (k outer, i inner); contributions added with global atomics.
template <typename Real, bool General>
__global__ void __launch_bounds__(256) deposit_walk_kernel(const SubSeg *__restrict__ seg, int64_t nsub,
                                                           const LineParam *__restrict__ lp, int line_base,
                                                           const double *__restrict__ coe,
                                                           const double *__restrict__ dtf, int N, double dzeta_sup,
                                                           double eta, Real *__restrict__ wx, Real *__restrict__ wy,
                                                           Real *__restrict__ wz, unsigned long long *accepted)
{
    const int lane = threadIdx.x & 31;
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long acc = 0;
    for (int64_t q = w0; q < nsub; q += nw) {
        const SubSeg S = seg[q];
        const LineParam P = lp[S.line - line_base];
        const int nx = S.box_hi[0] - S.box_lo[0] + 1, ny = S.box_hi[1] - S.box_lo[1] + 1,
                  nz = S.box_hi[2] - S.box_lo[2] + 1;
        const int64_t total = (int64_t)nx * ny * nz;
        const double dt = dtf[S.slot];
        if constexpr (sizeof(Real) == 8) {
            const double dx = dev_pi2() / N;
            const double *cf = coe + 18 * (size_t)S.slot;
            for (int64_t idx = lane; idx < total; idx += 32) {
                const int ii = (int)(idx % nx);
                const int64_t r = idx / nx;
                const int jj = (int)(r % ny), kk = (int)(r / ny);
                const int ip = S.box_lo[0] + ii, jp = S.box_lo[1] + jj, kp = S.box_lo[2] + kk;
                double o[3];
                if (!point_ref_f64(S, P, cf, dt, dzeta_sup, eta, dx, ip, jp, kp, o)) continue;
                const size_t id = (size_t)wrap_idx(ip - 1, N) +
                                  (size_t)N * ((size_t)wrap_idx(jp - 1, N) + (size_t)N * (size_t)wrap_idx(kp - 1, N));
                atomicAdd((double *)wx + id, o[0]);
                atomicAdd((double *)wy + id, o[1]);
                atomicAdd((double *)wz + id, o[2]);
                ++acc;
            }
        } else {
            SegF G;
            seg_setup_f32(S, P, coe, dt, dzeta_sup, eta, N, S.box_lo[0], S.box_lo[1], S.box_lo[2], G);
            for (int64_t idx = lane; idx < total; idx += 32) {
                const int ii = (int)(idx % nx);
                const int64_t r = idx / nx;
                const int jj = (int)(r % ny), kk = (int)(r / ny);
                float o[3], cond;
                const int pass = point_f32<General>(G, ii, jj, kk, o, cond);
                if (pass == 0) continue;
                const int ip = S.box_lo[0] + ii, jp = S.box_lo[1] + jj, kp = S.box_lo[2] + kk;
                if (pass == 2 || (General && !(cond <= kRedoCond))) {
                    // a plane test within its rounding bound, or an ill-conditioned
                    // curved-branch point: the reference's FP64 tests and arithmetic
                    double o64[3];
                    if (!point_ref_f64(S, P, coe + 18 * (size_t)S.slot, dt, dzeta_sup, eta, dev_pi2() / N, ip, jp, kp,
                                       o64))
                        continue;
                    o[0] = (float)o64[0];
                    o[1] = (float)o64[1];
                    o[2] = (float)o64[2];
                }
                const size_t id = (size_t)wrap_idx(ip - 1, N) +
                                  (size_t)N * ((size_t)wrap_idx(jp - 1, N) + (size_t)N * (size_t)wrap_idx(kp - 1, N));
                atomicAdd((float *)wx + id, o[0]);
                atomicAdd((float *)wy + id, o[1]);
                atomicAdd((float *)wz + id, o[2]);
                ++acc;
            }
        }
    }
    acc = warp_sum(acc);
    if (lane == 0 && accepted) atomicAdd(accepted, acc);
}

// ---------------------------------------------------------------------------- driver
int launch_walk(Ctx *c, const CenterlineBatch &B, unsigned long long *d_acc)
{
    if (B.nsub == 0) return 0;
    const int N = c->p.N;
    const size_t n3 = field_elems(c);
    const bool general = !(c->p.sigma_ratio == 1.0 && c->p.eta_t == 0.0);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const int64_t want = (B.nsub * 32 + 255) / 256;
    const unsigned blocks = (unsigned)std::min<int64_t>(want, (int64_t)sms * 64);
    const int km = kt_begin(c, KT_DEPOSIT);
    if (c->p.precision == 64) {
        double *w = (double *)c->b_w.p;
        deposit_walk_kernel<double, true><<<blocks, 256, 0, c->stream>>>(
            B.seg, B.nsub, B.lp, B.la, B.coe, B.dtf, N, c->p.dzeta_sup, c->p.eta_t, w, w + n3, w + 2 * n3, d_acc);
    } else {
        float *w = (float *)c->b_w.p;
        if (general)
            deposit_walk_kernel<float, true><<<blocks, 256, 0, c->stream>>>(
                B.seg, B.nsub, B.lp, B.la, B.coe, B.dtf, N, c->p.dzeta_sup, c->p.eta_t, w, w + n3, w + 2 * n3, d_acc);
        else
            deposit_walk_kernel<float, false><<<blocks, 256, 0, c->stream>>>(
                B.seg, B.nsub, B.lp, B.la, B.coe, B.dtf, N, c->p.dzeta_sup, c->p.eta_t, w, w + n3, w + 2 * n3, d_acc);
    }
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    return 0;
}

static int64_t batch_node_cap(const Ctx *c)
{
    // sub-segment records are ~200 B, with samples and tile lists ~300 B, and there are ~10-50
    // per node: keep a batch's set-up arrays within a few GB, and under a memory cap within
    // about half of it (24 KB per node)
    int64_t cap = (int64_t)1 << 22;
    if (c->p.mem_cap) cap = std::min(cap, std::max<int64_t>((int64_t)1 << 15, (int64_t)(c->p.mem_cap / 24576)));
    return cap;
}

int deposit_lines(Ctx *c, int line_s, int line_e)
{
    if (!c->have_lines) return fail(FWT_E_STATE, "no centerlines set");
    if (c->slab_nz && c->p.deposit_mode != 0) return fail(FWT_E_STATE, "a z-slab context deposits with deposit_mode 0");
    if (line_s < 1 || line_e > c->nline || line_s > line_e)
        return fail(FWT_E_ARG, "line range outside 1..nline");
    const size_t n3 = field_elems(c);
    FWT_TRY(buf_reserve(c, c->b_w, 3 * n3 * real_bytes(c)));
    if (!c->have_w) {
        FWT_CUDA(cudaMemsetAsync(c->b_w.p, 0, 3 * n3 * real_bytes(c), c->stream));
        if (c->side_dirty) {   // sums left by a deposition that failed part-way
            FWT_CUDA(cudaMemsetAsync(c->b_side.p, 0, c->b_side.bytes, c->stream));
            c->side_dirty = false;
        }
        c->have_w = true;
        c->line_ntf_sum.assign(c->nline, 0);
        c->line_ntf_max.assign(c->nline, 0);
        c->line_len.assign(c->nline, 0.0);
    }
    c->have_u = false;
    c->normalised = false;
    // scratch[19]: [0, 8) accepted points of the box walk, [16, 64) the component range of a
    // tile deposition, [64, 80) the tile kernels' tallies (accepted pairs, FP64 redone pairs),
    // [96, 100) the error flag of the deferred pairs' FP64 pass
    FWT_TRY(buf_reserve(c, c->scratch[19], 128));
    unsigned long long *d_acc = (unsigned long long *)c->scratch[19].p;
    FWT_CUDA(cudaMemsetAsync(d_acc, 0, 128, c->stream));
    int64_t sections = 0, subsegs = 0, pairs = 0;
    const int64_t cap = batch_node_cap(c);
    // deposit_mode 0: the tile-owned kernels (FP32 evaluation, or in the FP64 path FP32
    // candidate tests and the reference's FP64 tests and arithmetic); 1: the reference's box walk
    const bool tile_path = c->p.deposit_mode == 0;
    const double dxg = kPi2 / c->p.N;
    // radius limit of the piece kernel in grid spacings: fwt_set_tuning, else the environment
    // variable FWT_PIECE_RT_CELLS, else the default
    const char *env = std::getenv("FWT_PIECE_RT_CELLS");
    const double rt_cells = c->piece_rt_cells >= 0.0 ? c->piece_rt_cells : (env ? std::atof(env) : kPieceMaxRtCells);
    auto thin = [&](int l) {
        return tile_path && c->p.Rtube_ratio * c->p.sigma_ratio * c->sigma[l] <= rt_cells * dxg;
    };
    // radius limit of rasterised pieces: fwt_set_tuning, else FWT_RASTER_RT_CELLS, else the default
    const char *renv = std::getenv("FWT_RASTER_RT_CELLS");
    const double ras_cells =
        c->raster_rt_cells >= 0.0 ? c->raster_rt_cells : (renv ? std::atof(renv) : kRasterMaxRtCells);
    auto rasterised = [&](int l) {
        return thin(l) && c->p.Rtube_ratio * c->p.sigma_ratio * c->sigma[l] <= ras_cells * dxg;
    };
    // radius limit of the scatter path (FP32 piece lines without tiles): fwt_set_tuning, else
    // FWT_SCATTER_RT_CELLS, else the default
    const char *senv = std::getenv("FWT_SCATTER_RT_CELLS");
    const double sca_cells =
        c->scatter_rt_cells >= 0.0 ? c->scatter_rt_cells : (senv ? std::atof(senv) : kScatterMaxRtCells);
    auto scattered = [&](int l) {
        return thin(l) && c->p.precision == 32 && !rasterised(l) &&
               c->p.Rtube_ratio * c->p.sigma_ratio * c->sigma[l] <= sca_cells * dxg;
    };
    int la = line_s - 1;
    while (la < line_e) {
        // batch: consecutive lines up to the node cap, ending after a filtered line and where
        // the lines change between the sub-segment and the piece kernel
        int lb = la;
        int64_t nodes = 0;
        while (lb < line_e) {
            nodes += c->npoint[lb];
            ++lb;
            if (c->if_filter[lb - 1]) break;
            if (lb < line_e && nodes + c->npoint[lb] > cap) break;
            if (lb < line_e && (thin(lb) != thin(la) || rasterised(lb) != rasterised(la) ||
                                scattered(lb) != scattered(la)))
                break;
        }
        const BatchRecords mode =
            !tile_path ? BatchRecords::Walk : (thin(la) ? BatchRecords::Pieces : BatchRecords::SubSeg);
        if (std::getenv("FWT_SYNC_CHECK"))
            std::fprintf(stderr, "libfwt: batch lines %d..%d records %d\n", la + 1, lb, (int)mode);
        // the batch's nodes, when an asynchronous upload is still bringing them
        FWT_TRY(wait_nodes(c, c->node_off[lb]));
        CenterlineBatch B;
        B.raster = mode == BatchRecords::Pieces && rasterised(la);
        B.scatter = mode == BatchRecords::Pieces && scattered(la);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, c->stream);
        const int rc_setup = centerline_setup(c, la, lb, B, mode);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms_setup = 0;
        cudaEventElapsedTime(&ms_setup, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        FWT_TRY(rc_setup);
        c->t_setup_acc += ms_setup;
        for (int i = 0; i < B.nl; ++i) {
            c->line_ntf_sum[la + i] = B.line_ntf_sum[2 * i];
            c->line_ntf_max[la + i] = B.line_ntf_sum[2 * i + 1];
            c->line_len[la + i] = B.Lens[i] * kPi2;
        }
        sections += B.nslots - B.nl;
        subsegs += B.nsub;
        if (mode == BatchRecords::Walk) {
            FWT_TRY(launch_walk(c, B, d_acc));
        } else {
            int64_t np_ = 0;
            if (mode == BatchRecords::Pieces && B.scatter) FWT_TRY(launch_scatter(c, B));
            else if (mode == BatchRecords::Pieces) FWT_TRY(launch_piece(c, B, &np_));
            else FWT_TRY(launch_tile(c, B, &np_));
            pairs += np_;
        }
        if (c->if_filter[lb - 1]) {
            // the filter acts on the whole field deposited so far
            FWT_TRY(side_fold(c));
            const double kc = std::ceil(4.0 / c->sigma[lb - 1]);
            FWT_TRY(spectral_filter(c, kc));
        }
        la = lb;
    }
    FWT_TRY(side_fold(c));
    c->counters[0] = line_e - line_s + 1;
    c->counters[1] = sections;
    c->counters[2] = subsegs;
    c->counters[3] = pairs;
    unsigned long long tally[3];
    FWT_CUDA(cudaMemcpyAsync(tally, d_acc, sizeof(tally), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaMemcpyAsync(tally + 1, d_acc + 8, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    c->counters[5] = (int64_t)(tile_path ? tally[1] : tally[0]);
    c->counters[6] = (int64_t)tally[2];
    // an asynchronous upload is complete once this call returns (its caller's array is free)
    return finish_upload(c);
}

}  // namespace fwt
