// k_iso.cu -- isosurface extraction of |omega| with the helicity omega.u as its colour, the
// compute part of the reference's rendering script (output/field_wh_norm.py:56-89: read
// field_wh.dat, iso value 3 rms(|omega|) / sqrt 2, contour of |omega|, helicity as the point
// scalar).  The rendering itself (an off-screen GL window) has no place on a headless device;
// the mesh is returned as a buffer of triangles.
//
// Method: marching tetrahedra on the field_wh data box, a published alternative to marching
// cubes that needs no case table.  The box is the script's structured grid: n^3 points at
// x_i = 2 pi i / (n - 1) (numpy.linspace(0, 2 pi, n)), not periodic.  Every cube is split into
// six tetrahedra around its diagonal from corner 0 to corner 7 (one per order in which the three
// axes are stepped), a split that neighbouring cubes share on their common faces, so the surface
// is closed.  A vertex is inside when its value exceeds the iso value; a tetrahedron with one or
// three vertices inside gives one triangle, with two inside two.  A crossing point is
// interpolated along its edge from the edge's lower-indexed end, so both tetrahedra that share
// an edge compute the same point bit for bit.  Triangles are wound so that their normal points
// from the inside vertices to the outside ones.
//
// Two passes and a scan: triangles per cube, exclusive scan, emission at the cube's offset;
// the triangle order is the cube order (x fastest), deterministic.
#include "k_centerline.cuh"

namespace fwt {

namespace {

// corner c = x | y << 1 | z << 2; tetrahedron t of the Kuhn split: 0 -> a -> a|b -> 7
__constant__ int kTetAxes[6][2] = {{1, 2}, {1, 4}, {2, 1}, {2, 4}, {4, 1}, {4, 2}};

struct IsoBox {
    const float *v;   // |omega| at the box points, x fastest
    const float *h;   // omega . u
    int n;
    float iso, step;  // iso value, grid step 2 pi / (n - 1)
};

__device__ __forceinline__ void tet_corners(int t, int c[4])
{
    const int a = kTetAxes[t][0], b = kTetAxes[t][1];
    c[0] = 0;
    c[1] = a;
    c[2] = a | b;
    c[3] = 7;
}

__device__ __forceinline__ int tet_tris(int mask)
{
    const int k = __popc(mask);
    return (k == 1 || k == 3) ? 1 : (k == 2 ? 2 : 0);
}

// triangles of cube (i, j, k) (lower corner) and the corner values
__device__ __forceinline__ int cube_mask(const IsoBox &B, int i, int j, int k, size_t gi[8], float val[8])
{
    const size_t n = (size_t)B.n;
    int m = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        gi[c] = (size_t)(i + (c & 1)) + n * ((size_t)(j + ((c >> 1) & 1)) + n * (size_t)(k + ((c >> 2) & 1)));
        val[c] = B.v[gi[c]];
        if (val[c] > B.iso) m |= 1 << c;
    }
    return m;
}

__global__ void iso_count_kernel(IsoBox B, int64_t *__restrict__ cnt)
{
    const int64_t nc = (int64_t)(B.n - 1) * (B.n - 1) * (B.n - 1);
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nc) return;
    const int m1 = B.n - 1;
    const int i = (int)(q % m1), j = (int)((q / m1) % m1), k = (int)(q / ((int64_t)m1 * m1));
    size_t gi[8];
    float val[8];
    const int m = cube_mask(B, i, j, k, gi, val);
    int t = 0;
    if (m != 0 && m != 0xff) {
#pragma unroll
        for (int tt = 0; tt < 6; ++tt) {
            int c[4];
            tet_corners(tt, c);
            const int tm = ((m >> c[0]) & 1) | (((m >> c[1]) & 1) << 1) | (((m >> c[2]) & 1) << 2) | (((m >> c[3]) & 1) << 3);
            t += tet_tris(tm);
        }
    }
    cnt[q] = t;
}

// crossing point of edge (a, b) of the cube, interpolated from its lower-indexed end
__device__ __forceinline__ void crossing(const IsoBox &B, int i, int j, int k, int a, int b, const size_t gi[8],
                                         const float val[8], float p[4])
{
    if (gi[a] > gi[b]) {
        const int t = a;
        a = b;
        b = t;
    }
    const float t = __fdiv_rn(__fsub_rn(B.iso, val[a]), __fsub_rn(val[b], val[a]));
    const float xa[3] = {(float)(i + (a & 1)), (float)(j + ((a >> 1) & 1)), (float)(k + ((a >> 2) & 1))};
    const float xb[3] = {(float)(i + (b & 1)), (float)(j + ((b >> 1) & 1)), (float)(k + ((b >> 2) & 1))};
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = __fmul_rn(__fadd_rn(xa[d], __fmul_rn(t, __fsub_rn(xb[d], xa[d]))), B.step);
    const float ha = B.h[gi[a]], hb = B.h[gi[b]];
    p[3] = __fadd_rn(ha, __fmul_rn(t, __fsub_rn(hb, ha)));
}

// one triangle (p, q, r) wound so that its normal points along `out` (inside -> outside)
__device__ __forceinline__ void put_tri(float *__restrict__ dst, const float p[4], const float q[4], const float r[4],
                                        const float out[3])
{
    // every operation rounded on its own (no contraction), so a host restatement decides alike
    const float e1[3] = {__fsub_rn(q[0], p[0]), __fsub_rn(q[1], p[1]), __fsub_rn(q[2], p[2])};
    const float e2[3] = {__fsub_rn(r[0], p[0]), __fsub_rn(r[1], p[1]), __fsub_rn(r[2], p[2])};
    const float nx = __fsub_rn(__fmul_rn(e1[1], e2[2]), __fmul_rn(e1[2], e2[1]));
    const float ny = __fsub_rn(__fmul_rn(e1[2], e2[0]), __fmul_rn(e1[0], e2[2]));
    const float nz = __fsub_rn(__fmul_rn(e1[0], e2[1]), __fmul_rn(e1[1], e2[0]));
    const float dot = __fadd_rn(__fadd_rn(__fmul_rn(nx, out[0]), __fmul_rn(ny, out[1])), __fmul_rn(nz, out[2]));
    const bool flip = dot < 0.0f;
    const float *v[3] = {p, flip ? r : q, flip ? q : r};
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
        for (int d = 0; d < 4; ++d) dst[4 * s + d] = v[s][d];
}

__global__ void iso_emit_kernel(IsoBox B, const int64_t *__restrict__ off, float *__restrict__ tri)
{
    const int64_t nc = (int64_t)(B.n - 1) * (B.n - 1) * (B.n - 1);
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nc) return;
    int64_t o = off[q];
    if (off[q + 1] == o) return;
    const int m1 = B.n - 1;
    const int i = (int)(q % m1), j = (int)((q / m1) % m1), k = (int)(q / ((int64_t)m1 * m1));
    size_t gi[8];
    float val[8];
    const int m = cube_mask(B, i, j, k, gi, val);
    for (int tt = 0; tt < 6; ++tt) {
        int c[4];
        tet_corners(tt, c);
        int in[4], out[4], ni = 0, no = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if ((m >> c[s]) & 1) in[ni++] = c[s];
            else out[no++] = c[s];
        }
        if (ni == 0 || no == 0) continue;
        // direction from the inside corners' centroid to the outside ones'
        // (small integer sums and quotients of 1..3: exact or correctly rounded alike anywhere)
        float dir[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            int si = 0, so = 0;
            for (int s = 0; s < ni; ++s) si += (in[s] >> d) & 1;
            for (int s = 0; s < no; ++s) so += (out[s] >> d) & 1;
            dir[d] = __fsub_rn(__fdiv_rn((float)so, (float)no), __fdiv_rn((float)si, (float)ni));
        }
        float p[4][4];
        if (ni == 1 || no == 1) {
            const int lone = ni == 1 ? in[0] : out[0];
            const int *oth = ni == 1 ? out : in;
            for (int s = 0; s < 3; ++s) crossing(B, i, j, k, lone, oth[s], gi, val, p[s]);
            put_tri(tri + 12 * o, p[0], p[1], p[2], dir);
            ++o;
        } else {
            // quad in[0]-out[0], in[0]-out[1], in[1]-out[1], in[1]-out[0], split on one diagonal
            crossing(B, i, j, k, in[0], out[0], gi, val, p[0]);
            crossing(B, i, j, k, in[0], out[1], gi, val, p[1]);
            crossing(B, i, j, k, in[1], out[1], gi, val, p[2]);
            crossing(B, i, j, k, in[1], out[0], gi, val, p[3]);
            put_tri(tri + 12 * o, p[0], p[1], p[2], dir);
            put_tri(tri + 12 * (o + 1), p[0], p[2], p[3], dir);
            o += 2;
        }
    }
}

// sum of |omega|^2 over the box (for the iso value 3 rms / sqrt 2)
__global__ void iso_sumsq_kernel(const float *__restrict__ v, size_t n, double *__restrict__ s)
{
    double a = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        a += (double)v[i] * (double)v[i];
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) atomicAdd(s, a);
}

}  // namespace

int iso_extract(Ctx *c, float iso, float *host_tris, int64_t max_tris, int64_t *ntris, float *iso_used)
{
    // the field_wh box of the normalised fields (tube.f90:1055-1071) into scratch[8]
    FWT_TRY(stats_field_wh(c, nullptr));
    const int n = c->p.N_downsample;
    if (n < 2) return fail(FWT_E_ARG, "isosurface: the field box needs at least 2 points per side");
    const size_t m3 = (size_t)n * n * n;
    const float *box = (const float *)c->scratch[8].p;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    if (!(iso > 0.0f)) {
        FWT_TRY(buf_reserve(c, c->scratch[9], 64));
        double *d_s = (double *)c->scratch[9].p;
        FWT_CUDA(cudaMemsetAsync(d_s, 0, sizeof(double), c->stream));
        iso_sumsq_kernel<<<(unsigned)std::min<size_t>((m3 + 255) / 256, (size_t)sms * 8), 256, 0, c->stream>>>(box, m3,
                                                                                                             d_s);
        double s = 0.0;
        FWT_CUDA(cudaMemcpyAsync(&s, d_s, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        FWT_CUDA(cudaStreamSynchronize(c->stream));
        // output/field_wh_norm.py:71-73: rms_vor = sqrt(mean(vor^2)); iso_w = rms_vor * 3 / sqrt(2)
        iso = (float)(std::sqrt(s / (double)m3) * 3.0 / std::sqrt(2.0));
        c->launches += 1;
    }
    if (iso_used) *iso_used = iso;
    IsoBox B{box, box + m3, n, iso, (float)(kPi2 / (double)(n - 1))};
    const int64_t nc = (int64_t)(n - 1) * (n - 1) * (n - 1);
    FWT_TRY(buf_reserve(c, c->scratch[20], sizeof(int64_t) * (size_t)(nc + 1)));
    int64_t *d_cnt = (int64_t *)c->scratch[20].p;
    const unsigned g = (unsigned)((nc + 255) / 256);
    const int km = kt_begin(c, KT_STATS);
    iso_count_kernel<<<g, 256, 0, c->stream>>>(B, d_cnt);
    FWT_TRY(scan_exclusive_i64(c, d_cnt, nc, d_cnt + nc, c->scratch[12]));
    kt_end(c, km);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    int64_t total = 0;
    FWT_CUDA(cudaMemcpyAsync(&total, d_cnt + nc, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    *ntris = total;
    if (!host_tris || total == 0) return 0;
    if (total > max_tris) return fail(FWT_E_RANGE, "isosurface: " + std::to_string(total) +
                                                       " triangles exceed the caller's buffer");
    FWT_TRY(buf_reserve(c, c->scratch[21], sizeof(float) * 12 * (size_t)total));
    float *d_tri = (float *)c->scratch[21].p;
    const int km2 = kt_begin(c, KT_STATS);
    iso_emit_kernel<<<g, 256, 0, c->stream>>>(B, d_cnt, d_tri);
    kt_end(c, km2);
    c->launches += 1;
    FWT_CUDA(cudaGetLastError());
    FWT_CUDA(cudaMemcpyAsync(host_tris, d_tri, sizeof(float) * 12 * (size_t)total, cudaMemcpyDeviceToHost, c->stream));
    FWT_CUDA(cudaStreamSynchronize(c->stream));
    return 0;
}

}  // namespace fwt
