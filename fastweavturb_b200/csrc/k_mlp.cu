// k_mlp.cu -- the learned surrogate: a multilayer perceptron n_in -> width x depth (GELU) ->
// n_out whose matrix products run on the tensor cores (gemm_bf16_tc: BF16 operands, FP32
// accumulation) and whose bias, activation, loss and Adam steps are FP32 elementwise kernels.
// FP32 master weights; BF16 copies (and transposes, for the backward products) are refreshed
// after every update.  No reference counterpart: the surrogate maps generator parameters to
// the statistics the generator produces (the reference only plots those statistics).
//
// Shapes (B = batch padded to a multiple of 64, Kl = layer input width padded to 64):
//   forward   Z_l[B x N_l]  = H_{l-1}[B x K_l] . W_l[N_l x K_l]^T + b_l,  H_l = gelu(Z_l)
//   backward  dW_l[N_l x K_l] = dZ_l^T[N_l x B] . (H_{l-1}^T[K_l x B])^T
//             dH_{l-1}[B x K_l] = dZ_l[B x Np_l] . (W_l^T[K_l x Np_l])^T,  dZ = dH * gelu'(Z)
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fwt.h"
#include "fwt_internal.h"

namespace fwt {

int gemm_bf16_tc(const void *A, const void *B, float *C, int M, int N, int K, int ldc, int *d_err, cudaStream_t st);

static inline int pad64(int x) { return (x + 63) / 64 * 64; }

struct MlpLayer {
    int K = 0, Kp = 0, N = 0, Np = 0;   // input/output widths and their 64-padded sizes
    float *W = nullptr, *b = nullptr;   // FP32 master (N x K), (N)
    float *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;
    float *gW = nullptr, *gb = nullptr;
    __nv_bfloat16 *Wh = nullptr;        // N x Kp
    __nv_bfloat16 *Wt = nullptr;        // Kp x Np (transpose)
    float *Z = nullptr;                 // B x N pre-activation
    __nv_bfloat16 *H = nullptr;         // B x Np activation (input of the next layer)
    __nv_bfloat16 *Ht = nullptr;        // Np x B
    float *dZf = nullptr;               // B x N
    __nv_bfloat16 *dZ = nullptr;        // B x Np
    __nv_bfloat16 *dZt = nullptr;       // N x B
};

}  // namespace fwt

struct fwt_mlp {
    int dev = 0;
    int n_in = 0, width = 0, depth = 0, n_out = 0, bmax = 0;
    std::vector<fwt::MlpLayer> L;
    __nv_bfloat16 *X0 = nullptr, *X0t = nullptr;   // B x 64, 64 x B
    float *C = nullptr;                            // GEMM output scratch (max B x 256, 256 x 256)
    float *T = nullptr, *wout = nullptr;           // targets B x n_out, output weights n_out
    float *Xin = nullptr, *Gx = nullptr;           // inputs and input gradient, B x n_in
    double *loss = nullptr;
    int *err = nullptr;
    int64_t step = 0;
    cudaStream_t st = nullptr;
    std::vector<void *> allocs;
};

namespace fwt {

template <typename T>
static int mlp_alloc(fwt_mlp *m, T **p, size_t n)
{
    void *q = nullptr;
    if (cudaMalloc(&q, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) {
        cudaGetLastError();
        return fail(FWT_E_NOMEM, "mlp: device allocation failed");
    }
    cudaMemset(q, 0, sizeof(T) * std::max<size_t>(n, 1));
    m->allocs.push_back(q);
    *p = (T *)q;
    return 0;
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// X (B x n_in, FP32) -> X0 (Bp x 64 BF16, zero padded) and its transpose
__global__ void mlp_pack_input(const float *__restrict__ X, int B, int Bp, int n_in, __nv_bfloat16 *__restrict__ X0,
                               __nv_bfloat16 *__restrict__ X0t)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bp * 64) return;
    const int r = i / 64, c = i % 64;
    const float v = (r < B && c < n_in) ? X[(size_t)r * n_in + c] : 0.0f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    X0[i] = h;
    X0t[(size_t)c * Bp + r] = h;
}

// Z = C + b; hidden layers also H = gelu(Z) (BF16, zero padded to Np) and H^T
__global__ void mlp_bias_act(const float *__restrict__ C, const float *__restrict__ b, int B, int Bp, int N, int Np,
                             int act, float *__restrict__ Z, __nv_bfloat16 *__restrict__ H,
                             __nv_bfloat16 *__restrict__ Ht)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bp * Np) return;
    const int r = i / Np, c = i % Np;
    float z = 0.0f;
    if (r < B && c < N) {
        z = C[(size_t)r * N + c] + b[c];
        Z[(size_t)r * N + c] = z;
    }
    if (act) {
        const float h = (r < B && c < N) ? gelu(z) : 0.0f;
        const __nv_bfloat16 hb = __float2bfloat16_rn(h);
        H[(size_t)r * Np + c] = hb;
        Ht[(size_t)c * Bp + r] = hb;
    }
}

// loss = sum_b sum_j w_j (y - t)^2 / (B n_out); dZ of the output layer
__global__ void mlp_loss_grad(const float *__restrict__ Y, const float *__restrict__ T, const float *__restrict__ w,
                              int B, int Bp, int N, int Np, double *__restrict__ loss, float *__restrict__ dZf,
                              __nv_bfloat16 *__restrict__ dZ, __nv_bfloat16 *__restrict__ dZt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < Bp * Np) {
        const int r = i / Np, c = i % Np;
        float g = 0.0f;
        if (r < B && c < N) {
            const float d = Y[(size_t)r * N + c] - T[(size_t)r * N + c];
            const float wc = w ? w[c] : 1.0f;
            l = (double)wc * d * d / ((double)B * N);
            g = 2.0f * wc * d / ((float)B * (float)N);
            dZf[(size_t)r * N + c] = g;
        }
        const __nv_bfloat16 gb = __float2bfloat16_rn(g);
        dZ[(size_t)r * Np + c] = gb;
        if (c < N) dZt[(size_t)c * Bp + r] = gb;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

// dZ = dH * gelu'(Z) for a hidden layer (dH = C, B x ldc)
__global__ void mlp_act_back(const float *__restrict__ C, int ldc, const float *__restrict__ Z, int B, int Bp, int N,
                             int Np, float *__restrict__ dZf, __nv_bfloat16 *__restrict__ dZ,
                             __nv_bfloat16 *__restrict__ dZt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Bp * Np) return;
    const int r = i / Np, c = i % Np;
    float g = 0.0f;
    if (r < B && c < N) {
        g = C[(size_t)r * ldc + c] * gelu_d(Z[(size_t)r * N + c]);
        dZf[(size_t)r * N + c] = g;
    }
    const __nv_bfloat16 gb = __float2bfloat16_rn(g);
    dZ[(size_t)r * Np + c] = gb;
    if (c < N) dZt[(size_t)c * Bp + r] = gb;
}

// db = column sums of dZ (FP32), one thread per column
__global__ void mlp_bias_grad(const float *__restrict__ dZf, int B, int N, float *__restrict__ gb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    double s = 0.0;
    for (int r = 0; r < B; ++r) s += dZf[(size_t)r * N + c];
    gb[c] = (float)s;
}

// copy the GEMM's dW (N x Kp) into the K-wide gradient
__global__ void mlp_take_grad(const float *__restrict__ C, int N, int K, int Kp, float *__restrict__ g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * K) return;
    g[i] = C[(size_t)(i / K) * Kp + i % K];
}

__global__ void mlp_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1,
                         float *__restrict__ m2, int n, float lr, float b1, float b2, float c1, float c2, float eps)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi, v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    p[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// BF16 copies of W: Wh (N x Kp, zero padded) and Wt (Kp x Np)
__global__ void mlp_refresh(const float *__restrict__ W, int N, int K, int Kp, int Np, __nv_bfloat16 *__restrict__ Wh,
                            __nv_bfloat16 *__restrict__ Wt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Np * Kp) return;
    const int n = i / Kp, k = i % Kp;
    const __nv_bfloat16 v = __float2bfloat16_rn((n < N && k < K) ? W[(size_t)n * K + k] : 0.0f);
    if (n < N) Wh[(size_t)n * Kp + k] = v;
    Wt[(size_t)k * Np + n] = v;
}

static inline unsigned nblk(int64_t n) { return (unsigned)((n + 255) / 256); }

static int mlp_refresh_all(fwt_mlp *m)
{
    for (auto &l : m->L)
        mlp_refresh<<<nblk((int64_t)l.Np * l.Kp), 256, 0, m->st>>>(l.W, l.N, l.K, l.Kp, l.Np, l.Wh, l.Wt);
    FWT_CUDA(cudaGetLastError());
    return 0;
}

static int mlp_forward(fwt_mlp *m, const float *dX, int B)
{
    const int Bp = pad64(B);
    mlp_pack_input<<<nblk((int64_t)Bp * 64), 256, 0, m->st>>>(dX, B, Bp, m->n_in, m->X0, m->X0t);
    const __nv_bfloat16 *Hin = m->X0;
    for (size_t li = 0; li < m->L.size(); ++li) {
        MlpLayer &l = m->L[li];
        FWT_TRY(gemm_bf16_tc(Hin, l.Wh, m->C, Bp, l.N, l.Kp, l.N, m->err, m->st));
        const int act = li + 1 < m->L.size() ? 1 : 0;
        mlp_bias_act<<<nblk((int64_t)Bp * l.Np), 256, 0, m->st>>>(m->C, l.b, B, Bp, l.N, l.Np, act, l.Z, l.H, l.Ht);
        Hin = l.H;
    }
    FWT_CUDA(cudaGetLastError());
    return 0;
}

// gradients of the weighted MSE w.r.t. every parameter (into l.gW, l.gb) and, if dXout, the
// inputs (B x n_in, device)
static int mlp_backward(fwt_mlp *m, int B, float *dXout)
{
    const int Bp = pad64(B);
    FWT_CUDA(cudaMemsetAsync(m->loss, 0, sizeof(double), m->st));
    MlpLayer &o = m->L.back();
    mlp_loss_grad<<<nblk((int64_t)Bp * o.Np), 256, 0, m->st>>>(o.Z, m->T, m->wout, B, Bp, o.N, o.Np, m->loss, o.dZf,
                                                                 o.dZ, o.dZt);
    for (int li = (int)m->L.size() - 1; li >= 0; --li) {
        MlpLayer &l = m->L[li];
        const __nv_bfloat16 *Hprev_t = li > 0 ? m->L[li - 1].Ht : m->X0t;
        // dW = dZ^T . Hprev   (M = N_l, N = Kp, K = Bp)
        FWT_TRY(gemm_bf16_tc(l.dZt, Hprev_t, m->C, l.N, l.Kp, Bp, l.Kp, m->err, m->st));
        mlp_take_grad<<<nblk((int64_t)l.N * l.K), 256, 0, m->st>>>(m->C, l.N, l.K, l.Kp, l.gW);
        mlp_bias_grad<<<nblk(l.N), 256, 0, m->st>>>(l.dZf, B, l.N, l.gb);
        if (li == 0 && !dXout) break;
        // dH_prev = dZ . W  (M = Bp, N = Kp, K = Np)
        FWT_TRY(gemm_bf16_tc(l.dZ, l.Wt, m->C, Bp, l.Kp, l.Np, l.Kp, m->err, m->st));
        if (li == 0) {
            // input gradient: the first n_in columns
            FWT_CUDA(cudaMemcpy2DAsync(dXout, sizeof(float) * m->n_in, m->C, sizeof(float) * l.Kp,
                                       sizeof(float) * m->n_in, B, cudaMemcpyDeviceToDevice, m->st));
            break;
        }
        MlpLayer &p = m->L[li - 1];
        mlp_act_back<<<nblk((int64_t)Bp * p.Np), 256, 0, m->st>>>(m->C, l.Kp, p.Z, B, Bp, p.N, p.Np, p.dZf, p.dZ,
                                                                    p.dZt);
    }
    FWT_CUDA(cudaGetLastError());
    return 0;
}

static int mlp_check_err(fwt_mlp *m)
{
    int herr = 0;
    FWT_CUDA(cudaMemcpyAsync(&herr, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->st));
    FWT_CUDA(cudaStreamSynchronize(m->st));
    if (herr) return fail(FWT_E_TIMEOUT, "mlp: tensor-core GEMM wait ran out");
    return 0;
}

}  // namespace fwt

using namespace fwt;

extern "C" {

int fwt_gemm_bf16(const void *dA, const void *dB, float *dC, int M, int N, int K, int ldc, void *stream)
{
    if (!dA || !dB || !dC || ldc < N) return fail(FWT_E_ARG, "gemm: null operand or ldc < N");
    int *d_err = nullptr;
    if (cudaMalloc(&d_err, sizeof(int)) != cudaSuccess) return fail(FWT_E_NOMEM, "gemm: error flag allocation");
    cudaStream_t st = (cudaStream_t)stream;
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    int rc = gemm_bf16_tc(dA, dB, dC, M, N, K, ldc, d_err, st);
    int herr = 0;
    if (rc == 0) {
        cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = fail(FWT_E_CUDA, "gemm: kernel failed");
        else if (herr) rc = fail(FWT_E_TIMEOUT, "gemm: tensor-core wait ran out");
    }
    cudaFree(d_err);
    return rc;
}

int fwt_mlp_create(int device, int n_in, int width, int depth, int n_out, int batch_max, uint64_t seed, fwt_mlp **out)
{
    if (!out || n_in < 1 || n_in > 64 || width < 16 || width > 256 || width % 16 || depth < 1 || n_out < 1 ||
        n_out > 256 || batch_max < 1)
        return fail(FWT_E_ARG, "mlp: n_in 1..64, width 16..256 (multiple of 16), depth >= 1, n_out 1..256");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return fail(FWT_E_CUDA, "mlp: no such device");
    fwt_mlp *m = new fwt_mlp();
    m->dev = device;
    m->n_in = n_in;
    m->width = width;
    m->depth = depth;
    m->n_out = n_out;
    m->bmax = pad64(batch_max);
    const int Bp = m->bmax;
    int rc = 0;
    auto try_ = [&](int r) {
        if (rc == 0 && r != 0) rc = r;
    };
    if (cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) != cudaSuccess) rc = fail(FWT_E_CUDA, "mlp: stream");
    // widths: n_in -> width (depth times) -> n_out
    std::vector<int> w = {n_in};
    for (int i = 0; i < depth; ++i) w.push_back(width);
    w.push_back(n_out);
    uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto urand = [&]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    for (size_t i = 0; i + 1 < w.size() && rc == 0; ++i) {
        MlpLayer l;
        l.K = w[i];
        l.Kp = pad64(l.K);
        l.N = w[i + 1];
        l.Np = pad64(l.N);
        try_(mlp_alloc(m, &l.W, (size_t)l.N * l.K));
        try_(mlp_alloc(m, &l.b, l.N));
        try_(mlp_alloc(m, &l.mW, (size_t)l.N * l.K));
        try_(mlp_alloc(m, &l.vW, (size_t)l.N * l.K));
        try_(mlp_alloc(m, &l.mb, l.N));
        try_(mlp_alloc(m, &l.vb, l.N));
        try_(mlp_alloc(m, &l.gW, (size_t)l.N * l.K));
        try_(mlp_alloc(m, &l.gb, l.N));
        try_(mlp_alloc(m, &l.Wh, (size_t)l.N * l.Kp));
        try_(mlp_alloc(m, &l.Wt, (size_t)l.Kp * l.Np));
        try_(mlp_alloc(m, &l.Z, (size_t)Bp * l.N));
        try_(mlp_alloc(m, &l.H, (size_t)Bp * l.Np));
        try_(mlp_alloc(m, &l.Ht, (size_t)l.Np * Bp));
        try_(mlp_alloc(m, &l.dZf, (size_t)Bp * l.N));
        try_(mlp_alloc(m, &l.dZ, (size_t)Bp * l.Np));
        try_(mlp_alloc(m, &l.dZt, (size_t)l.N * Bp));
        if (rc) break;
        // uniform +-sqrt(6 / (fan_in + fan_out)), zero biases
        std::vector<float> hw((size_t)l.N * l.K);
        const double a = std::sqrt(6.0 / (l.K + l.N));
        for (auto &v : hw) v = (float)((2.0 * urand() - 1.0) * a);
        if (cudaMemcpy(l.W, hw.data(), sizeof(float) * hw.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(FWT_E_CUDA, "mlp: weight upload");
        m->L.push_back(l);
    }
    try_(mlp_alloc(m, &m->X0, (size_t)Bp * 64));
    try_(mlp_alloc(m, &m->X0t, (size_t)64 * Bp));
    try_(mlp_alloc(m, &m->C, (size_t)std::max(Bp, 256) * 256));
    try_(mlp_alloc(m, &m->T, (size_t)Bp * n_out));
    try_(mlp_alloc(m, &m->Xin, (size_t)Bp * n_in));
    try_(mlp_alloc(m, &m->Gx, (size_t)Bp * n_in));
    try_(mlp_alloc(m, &m->wout, n_out));
    try_(mlp_alloc(m, &m->loss, 1));
    try_(mlp_alloc(m, &m->err, 1));
    if (rc == 0) {
        std::vector<float> ones(n_out, 1.0f);
        cudaMemcpy(m->wout, ones.data(), sizeof(float) * n_out, cudaMemcpyHostToDevice);
        rc = mlp_refresh_all(m);
    }
    if (rc == 0 && cudaStreamSynchronize(m->st) != cudaSuccess) rc = fail(FWT_E_CUDA, "mlp: set-up failed");
    if (rc) {
        fwt_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return 0;
}

int fwt_mlp_destroy(fwt_mlp *m)
{
    if (!m) return 0;
    cudaSetDevice(m->dev);
    if (m->st) cudaStreamSynchronize(m->st);
    for (void *p : m->allocs) cudaFree(p);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return 0;
}

int fwt_mlp_nparams(fwt_mlp *m, int64_t *n)
{
    if (!m || !n) return fail(FWT_E_ARG, "mlp: null argument");
    int64_t t = 0;
    for (auto &l : m->L) t += (int64_t)l.N * l.K + l.N;
    *n = t;
    return 0;
}

// parameters flattened layer by layer: W_l (N x K, row-major) then b_l
int fwt_mlp_get_params(fwt_mlp *m, float *host)
{
    if (!m || !host) return fail(FWT_E_ARG, "mlp: null argument");
    cudaSetDevice(m->dev);
    for (auto &l : m->L) {
        FWT_CUDA(cudaMemcpyAsync(host, l.W, sizeof(float) * l.N * l.K, cudaMemcpyDeviceToHost, m->st));
        host += (size_t)l.N * l.K;
        FWT_CUDA(cudaMemcpyAsync(host, l.b, sizeof(float) * l.N, cudaMemcpyDeviceToHost, m->st));
        host += l.N;
    }
    FWT_CUDA(cudaStreamSynchronize(m->st));
    return 0;
}

int fwt_mlp_set_params(fwt_mlp *m, const float *host)
{
    if (!m || !host) return fail(FWT_E_ARG, "mlp: null argument");
    cudaSetDevice(m->dev);
    for (auto &l : m->L) {
        FWT_CUDA(cudaMemcpyAsync(l.W, host, sizeof(float) * l.N * l.K, cudaMemcpyHostToDevice, m->st));
        host += (size_t)l.N * l.K;
        FWT_CUDA(cudaMemcpyAsync(l.b, host, sizeof(float) * l.N, cudaMemcpyHostToDevice, m->st));
        host += l.N;
    }
    FWT_TRY(mlp_refresh_all(m));
    FWT_CUDA(cudaStreamSynchronize(m->st));
    return 0;
}

// y (batch x n_out, host) = mlp(x (batch x n_in, host))
int fwt_mlp_forward(fwt_mlp *m, const float *x, int batch, float *y)
{
    if (!m || !x || !y || batch < 1 || batch > m->bmax) return fail(FWT_E_ARG, "mlp: batch outside 1..batch_max");
    cudaSetDevice(m->dev);
    float *dX = m->Xin;
    FWT_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), m->st));
    FWT_CUDA(cudaMemcpyAsync(dX, x, sizeof(float) * batch * m->n_in, cudaMemcpyHostToDevice, m->st));
    FWT_TRY(mlp_forward(m, dX, batch));
    FWT_CUDA(cudaMemcpyAsync(y, m->L.back().Z, sizeof(float) * batch * m->n_out, cudaMemcpyDeviceToHost, m->st));
    return mlp_check_err(m);
}

// loss and its gradients: grad_params (nparams, layout of fwt_mlp_get_params) and grad_x
// (batch x n_in); either may be NULL.  w_out: n_out output weights or NULL (all 1).
int fwt_mlp_loss_grad(fwt_mlp *m, const float *x, const float *t, const float *w_out, int batch, double *loss,
                      float *grad_params, float *grad_x)
{
    if (!m || !x || !t || batch < 1 || batch > m->bmax) return fail(FWT_E_ARG, "mlp: batch outside 1..batch_max");
    cudaSetDevice(m->dev);
    float *dX = m->Xin, *dGx = m->Gx;
    FWT_CUDA(cudaMemsetAsync(m->err, 0, sizeof(int), m->st));
    FWT_CUDA(cudaMemcpyAsync(dX, x, sizeof(float) * batch * m->n_in, cudaMemcpyHostToDevice, m->st));
    FWT_CUDA(cudaMemcpyAsync(m->T, t, sizeof(float) * batch * m->n_out, cudaMemcpyHostToDevice, m->st));
    std::vector<float> ones(m->n_out, 1.0f);
    FWT_CUDA(cudaMemcpyAsync(m->wout, w_out ? w_out : ones.data(), sizeof(float) * m->n_out, cudaMemcpyHostToDevice,
                             m->st));
    int rc = mlp_forward(m, dX, batch);
    if (rc == 0) rc = mlp_backward(m, batch, grad_x ? dGx : nullptr);
    if (rc == 0 && loss) rc = cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st) ? -2 : 0;
    if (rc == 0 && grad_x)
        rc = cudaMemcpyAsync(grad_x, dGx, sizeof(float) * batch * m->n_in, cudaMemcpyDeviceToHost, m->st) ? -2 : 0;
    if (rc == 0 && grad_params) {
        float *h = grad_params;
        for (auto &l : m->L) {
            cudaMemcpyAsync(h, l.gW, sizeof(float) * l.N * l.K, cudaMemcpyDeviceToHost, m->st);
            h += (size_t)l.N * l.K;
            cudaMemcpyAsync(h, l.gb, sizeof(float) * l.N, cudaMemcpyDeviceToHost, m->st);
            h += l.N;
        }
    }
    if (rc) return rc < -1 ? fail(FWT_E_CUDA, "mlp: copy failed") : rc;
    return mlp_check_err(m);
}

// one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the weighted MSE of a batch
int fwt_mlp_train_step(fwt_mlp *m, const float *x, const float *t, const float *w_out, int batch, float lr,
                       double *loss)
{
    FWT_TRY(fwt_mlp_loss_grad(m, x, t, w_out, batch, loss, nullptr, nullptr));
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - (float)std::pow(0.9, (double)m->step), c2 = 1.0f - (float)std::pow(0.999, (double)m->step);
    for (auto &l : m->L) {
        mlp_adam<<<nblk((int64_t)l.N * l.K), 256, 0, m->st>>>(l.W, l.gW, l.mW, l.vW, l.N * l.K, lr, b1, b2, c1, c2,
                                                               1e-8f);
        mlp_adam<<<nblk(l.N), 256, 0, m->st>>>(l.b, l.gb, l.mb, l.vb, l.N, lr, b1, b2, c1, c2, 1e-8f);
    }
    FWT_TRY(mlp_refresh_all(m));
    FWT_CUDA(cudaStreamSynchronize(m->st));
    return 0;
}

}  // extern "C"
