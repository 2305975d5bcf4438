// The learned scheduler's network: a 3-layer perceptron (in -> 64 -> 64 ->
// out, ReLU), BF16 weights with FP32 accumulation, trained on the GPU with
// hand-written forward, backward and Adam kernels.  No reference counterpart
// (the reference has no scheduler beyond its page queues).
//
// The dense layers run on the tensor cores: k_gemm stages 64x16 tiles of
// both operands in shared memory as bf16 (rounding FP32 activations and the
// FP32 master weights on the way) and issues mma.sync.m16n8k16 bf16 ->
// f32; optional transposes of either operand are resolved while staging.
// The layers are tiny (64-wide), so one generic GEMM serves forward and
// backward.  Everything else (bias, ReLU, sigmoid cross-entropy gradient,
// column sums, Adam) is element-wise.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "common.h"
#include "engine.h"

namespace scaph {

namespace {

constexpr int kH = 64;  // hidden width

// C[M x N] = op(A)[M x K] * op(B)[K x N] (+ C if accumulate), FP32 in/out,
// bf16 tensor-core math.  op(A)(m,k) = TA ? A[k*lda + m] : A[m*lda + k];
// op(B)(k,n) = TB ? B[n*ldb + k] : B[k*ldb + n].  64x64 tile per CTA of 4 warps.
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb,
                                              float *C, int ldc, int accumulate)
{
    __shared__ __nv_bfloat16 As[64][16 + 8];  // [m][k]
    __shared__ __nv_bfloat16 Bs[64][16 + 8];  // [n][k]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;

    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int e = tid; e < 64 * 16; e += 128) {
            const int r = e / 16, c = e % 16;
            const int m = m0 + r, k = k0 + c;
            float a = 0.f;
            if (m < M && k < K) a = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[r][c] = __float2bfloat16_rn(a);
            const int n = n0 + r;
            float b = 0.f;
            if (n < N && k < K) b = TB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n];
            Bs[r][c] = __float2bfloat16_rn(b);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int r = wm + i * 16;
            const uint32_t a0 = *reinterpret_cast<const uint32_t *>(&As[r + gid][tig * 2]);
            const uint32_t a1 = *reinterpret_cast<const uint32_t *>(&As[r + gid + 8][tig * 2]);
            const uint32_t a2 = *reinterpret_cast<const uint32_t *>(&As[r + gid][tig * 2 + 8]);
            const uint32_t a3 = *reinterpret_cast<const uint32_t *>(&As[r + gid + 8][tig * 2 + 8]);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = wn + j * 8;
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&Bs[c + gid][tig * 2]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&Bs[c + gid][tig * 2 + 8]);
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                    : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int m = m0 + wm + i * 16 + gid + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
                if (m < M && n < N) {
                    float v = acc[i][j][r];
                    if (accumulate) v += C[(size_t)m * ldc + n];
                    C[(size_t)m * ldc + n] = v;
                }
            }
}

template <bool TA, bool TB>
cudaError_t gemm(int M, int N, int K, const float *A, int lda, const float *B, int ldb, float *C, int ldc,
                 cudaStream_t st, int accumulate = 0)
{
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_gemm<TA, TB><<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, accumulate);
    return cudaGetLastError();
}

__global__ void k_bias_relu(float *X, const float *b, int n, int cols, int relu)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * cols) return;
    float v = X[i] + b[i % cols];
    X[i] = relu ? fmaxf(v, 0.f) : v;
}

// dY = W * (sigmoid(Y) - T), loss terms = W * BCE-with-logits(Y, T)
__global__ void k_bce(const float *Y, const float *T, const float *W, float *dY, float *loss_terms, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float y = Y[i], t = T[i], w = W[i];
    const float s = 1.f / (1.f + expf(-y));
    dY[i] = w * (s - t);
    loss_terms[i] = w * (fmaxf(y, 0.f) - y * t + log1pf(expf(-fabsf(y))));
}

__global__ void k_relu_back(float *dH, const float *H, size_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && H[i] <= 0.f) dH[i] = 0.f;
}

// db[c] = sum over rows of dY[:, c]
__global__ void k_colsum(const float *dY, int n, int cols, float *db)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < n; r++) s += dY[(size_t)r * cols + c];
    db[c] = s;
}

__global__ void k_sum(const float *x, size_t n, float *out)
{
    __shared__ float sh[256];
    float s = 0.f;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// Adam (Kingma & Ba) on the FP32 master weights.
__global__ void k_adam(float *w, const float *g, float *m, float *v, size_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline unsigned grid_of(size_t n) { return (unsigned)((n + 255) / 256); }

// One row through the network in a single CTA (scheduler inference, one
// feature row per level): operands rounded to bf16, FP32 accumulation.
__global__ void __launch_bounds__(256) k_forward1(const float *w, int in, int out, size_t ow1, size_t ob1,
                                                  size_t ow2, size_t ob2, size_t ow3, size_t ob3, const float *x,
                                                  float *y)
{
    extern __shared__ float sx[];  // in floats
    __shared__ float h1[kH], h2[kH];
    auto bf = [](float v) { return __bfloat162float(__float2bfloat16_rn(v)); };
    for (int i = threadIdx.x; i < in; i += blockDim.x) sx[i] = bf(x[i]);
    __syncthreads();
    if (threadIdx.x < kH) {
        float a = w[ob1 + threadIdx.x];
        for (int i = 0; i < in; i++) a += sx[i] * bf(w[ow1 + (size_t)i * kH + threadIdx.x]);
        h1[threadIdx.x] = bf(fmaxf(a, 0.f));
    }
    __syncthreads();
    if (threadIdx.x < kH) {
        float a = w[ob2 + threadIdx.x];
        for (int i = 0; i < kH; i++) a += h1[i] * bf(w[ow2 + i * kH + threadIdx.x]);
        h2[threadIdx.x] = bf(fmaxf(a, 0.f));
    }
    __syncthreads();
    for (int o = threadIdx.x; o < out; o += blockDim.x) {
        float a = w[ob3 + o];
        for (int j = 0; j < kH; j++) a += h2[j] * bf(w[ow3 + (size_t)j * out + o]);
        y[o] = a;
    }
}

}  // namespace

}  // namespace scaph

using namespace scaph;

struct scaph_mlp {
    int in = 0, out = 0, device = 0;
    size_t nparams = 0;
    // parameter block: W1 [in x 64], b1 [64], W2 [64 x 64], b2 [64], W3 [64 x out], b3 [out]
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    size_t off_w1, off_b1, off_w2, off_b2, off_w3, off_b3;
    int step = 0;
    cudaStream_t st = nullptr;
    // activations (capacity in rows)
    int cap = 0;
    float *X = nullptr, *H1 = nullptr, *H2 = nullptr, *Y = nullptr, *T = nullptr, *Wt = nullptr, *dY = nullptr,
          *dH2 = nullptr, *dH1 = nullptr, *lt = nullptr, *loss = nullptr;

    float *W1() { return w + off_w1; }
    float *B1() { return w + off_b1; }
    float *W2() { return w + off_w2; }
    float *B2() { return w + off_b2; }
    float *W3() { return w + off_w3; }
    float *B3() { return w + off_b3; }

    int ensure(int n)
    {
        if (n <= cap) return SCAPH_OK;
        for (float *p : {X, H1, H2, Y, T, Wt, dY, dH2, dH1, lt}) cudaFree(p);
        cap = std::max(n, 64);
        SCAPH_CUDA(cudaMalloc(&X, sizeof(float) * cap * in));
        SCAPH_CUDA(cudaMalloc(&H1, sizeof(float) * cap * kH));
        SCAPH_CUDA(cudaMalloc(&H2, sizeof(float) * cap * kH));
        SCAPH_CUDA(cudaMalloc(&Y, sizeof(float) * cap * out));
        SCAPH_CUDA(cudaMalloc(&T, sizeof(float) * cap * out));
        SCAPH_CUDA(cudaMalloc(&Wt, sizeof(float) * cap * out));
        SCAPH_CUDA(cudaMalloc(&dY, sizeof(float) * cap * out));
        SCAPH_CUDA(cudaMalloc(&dH2, sizeof(float) * cap * kH));
        SCAPH_CUDA(cudaMalloc(&dH1, sizeof(float) * cap * kH));
        SCAPH_CUDA(cudaMalloc(&lt, sizeof(float) * cap * out));
        return SCAPH_OK;
    }

    // forward on the n rows already in X
    int forward(int n)
    {
        SCAPH_CUDA((gemm<false, false>(n, kH, in, X, in, W1(), kH, H1, kH, st)));
        k_bias_relu<<<grid_of((size_t)n * kH), 256, 0, st>>>(H1, B1(), n, kH, 1);
        SCAPH_CUDA((gemm<false, false>(n, kH, kH, H1, kH, W2(), kH, H2, kH, st)));
        k_bias_relu<<<grid_of((size_t)n * kH), 256, 0, st>>>(H2, B2(), n, kH, 1);
        SCAPH_CUDA((gemm<false, false>(n, out, kH, H2, kH, W3(), out, Y, out, st)));
        k_bias_relu<<<grid_of((size_t)n * out), 256, 0, st>>>(Y, B3(), n, out, 0);
        return SCAPH_OK;
    }

    // loss and gradients (into g) for the n rows in X / T / Wt
    int backward(int n)
    {
        const size_t no = (size_t)n * out;
        k_bce<<<grid_of(no), 256, 0, st>>>(Y, T, Wt, dY, lt, no);
        k_sum<<<1, 256, 0, st>>>(lt, no, loss);
        SCAPH_CUDA((gemm<true, false>(kH, out, n, H2, kH, dY, out, g + off_w3, out, st)));
        k_colsum<<<grid_of(out), 256, 0, st>>>(dY, n, out, g + off_b3);
        SCAPH_CUDA((gemm<false, true>(n, kH, out, dY, out, W3(), out, dH2, kH, st)));
        k_relu_back<<<grid_of((size_t)n * kH), 256, 0, st>>>(dH2, H2, (size_t)n * kH);
        SCAPH_CUDA((gemm<true, false>(kH, kH, n, H1, kH, dH2, kH, g + off_w2, kH, st)));
        k_colsum<<<grid_of(kH), 256, 0, st>>>(dH2, n, kH, g + off_b2);
        SCAPH_CUDA((gemm<false, true>(n, kH, kH, dH2, kH, W2(), kH, dH1, kH, st)));
        k_relu_back<<<grid_of((size_t)n * kH), 256, 0, st>>>(dH1, H1, (size_t)n * kH);
        SCAPH_CUDA((gemm<true, false>(in, kH, n, X, in, dH1, kH, g + off_w1, kH, st)));
        k_colsum<<<grid_of(kH), 256, 0, st>>>(dH1, n, kH, g + off_b1);
        return cudaGetLastError() == cudaSuccess ? SCAPH_OK : set_error(SCAPH_ECUDA, "mlp backward launch");
    }

    int upload(const float *hX, const float *hT, const float *hW, int n)
    {
        int rc = ensure(n);
        if (rc) return rc;
        SCAPH_CUDA(cudaMemcpyAsync(X, hX, sizeof(float) * n * in, cudaMemcpyHostToDevice, st));
        if (hT) SCAPH_CUDA(cudaMemcpyAsync(T, hT, sizeof(float) * n * out, cudaMemcpyHostToDevice, st));
        if (hW) SCAPH_CUDA(cudaMemcpyAsync(Wt, hW, sizeof(float) * n * out, cudaMemcpyHostToDevice, st));
        return SCAPH_OK;
    }
};

namespace scaph {

int mlp_forward_device(scaph_mlp *m, const float *hX, int n, float *hY)
{
    int rc = m->upload(hX, nullptr, nullptr, n);
    if (rc) return rc;
    if ((rc = m->forward(n))) return rc;
    SCAPH_CUDA(cudaMemcpyAsync(hY, m->Y, sizeof(float) * n * m->out, cudaMemcpyDeviceToHost, m->st));
    SCAPH_CUDA(cudaStreamSynchronize(m->st));
    return SCAPH_OK;
}

int mlp_forward1(scaph_mlp *m, const float *hX, float *hY, cudaStream_t st)
{
    int rc = m->ensure(1);
    if (rc) return rc;
    SCAPH_CUDA(cudaMemcpyAsync(m->X, hX, sizeof(float) * m->in, cudaMemcpyHostToDevice, st));
    k_forward1<<<1, 256, sizeof(float) * m->in, st>>>(m->w, m->in, m->out, m->off_w1, m->off_b1, m->off_w2,
                                                       m->off_b2, m->off_w3, m->off_b3, m->X, m->Y);
    SCAPH_CUDA(cudaGetLastError());
    SCAPH_CUDA(cudaMemcpyAsync(hY, m->Y, sizeof(float) * m->out, cudaMemcpyDeviceToHost, st));
    SCAPH_CUDA(cudaStreamSynchronize(st));
    return SCAPH_OK;
}

// Round to the nearest bfloat16, ties to even (NaN stays NaN).
static inline float bf16_round_host(float x)
{
    uint32_t u;
    memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) == 0x7F800000u && (u & 0x007FFFFFu)) return x;
    u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
    float r;
    memcpy(&r, &u, 4);
    return r;
}

int mlp_host_snapshot(const scaph_mlp *m, MlpHost &h)
{
    h.in = m->in;
    h.out = m->out;
    h.w.resize(m->nparams);
    SCAPH_CUDA(cudaMemcpy(h.w.data(), m->w, sizeof(float) * m->nparams, cudaMemcpyDeviceToHost));
    // the device rounds every weight to bf16 where it reads it; biases stay
    // in fp32
    const size_t off[3] = {m->off_w1, m->off_w2, m->off_w3};
    const size_t len[3] = {(size_t)m->in * kH, (size_t)kH * kH, (size_t)kH * m->out};
    for (int l = 0; l < 3; l++)
        for (size_t i = 0; i < len[l]; i++) h.w[off[l] + i] = bf16_round_host(h.w[off[l] + i]);
    h.off_w1 = m->off_w1;
    h.off_b1 = m->off_b1;
    h.off_w2 = m->off_w2;
    h.off_b2 = m->off_b2;
    h.off_w3 = m->off_w3;
    h.off_b3 = m->off_b3;
    return SCAPH_OK;
}

int mlp_device_view(const scaph_mlp *m, MlpDev *v)
{
    v->w = m->w;
    v->in = m->in;
    v->out = m->out;
    v->off_w1 = m->off_w1;
    v->off_b1 = m->off_b1;
    v->off_w2 = m->off_w2;
    v->off_b2 = m->off_b2;
    v->off_w3 = m->off_w3;
    v->off_b3 = m->off_b3;
    return SCAPH_OK;
}

int mlp_dims(const scaph_mlp *m, int *in, int *out)
{
    *in = m->in;
    *out = m->out;
    return SCAPH_OK;
}

}  // namespace scaph

extern "C" {

int scaph_mlp_create(int in_dim, int out_dim, uint64_t seed, int device, scaph_mlp **out)
{
    clear_error();
    if (!out || in_dim < 1 || out_dim < 1 || in_dim > 8192 || out_dim > 8192)
        return set_error(SCAPH_EINVAL, "bad mlp dimensions");
    std::unique_ptr<scaph_mlp> m(new scaph_mlp());
    m->in = in_dim;
    m->out = out_dim;
    m->device = device;
    SCAPH_CUDA(cudaSetDevice(device));
    SCAPH_CUDA(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    size_t o = 0;
    m->off_w1 = o; o += (size_t)in_dim * kH;
    m->off_b1 = o; o += kH;
    m->off_w2 = o; o += (size_t)kH * kH;
    m->off_b2 = o; o += kH;
    m->off_w3 = o; o += (size_t)kH * out_dim;
    m->off_b3 = o; o += out_dim;
    m->nparams = o;
    SCAPH_CUDA(cudaMalloc(&m->w, o * 4));
    SCAPH_CUDA(cudaMalloc(&m->g, o * 4));
    SCAPH_CUDA(cudaMalloc(&m->m, o * 4));
    SCAPH_CUDA(cudaMalloc(&m->v, o * 4));
    SCAPH_CUDA(cudaMemset(m->m, 0, o * 4));
    SCAPH_CUDA(cudaMemset(m->v, 0, o * 4));
    SCAPH_CUDA(cudaMalloc(&m->loss, 4));
    // He-uniform weights, zero biases, from a counter-based hash of the seed
    std::vector<float> h(o, 0.f);
    auto fill = [&](size_t off, size_t n, int fan_in) {
        const double lim = std::sqrt(6.0 / fan_in);
        for (size_t i = 0; i < n; i++) h[off + i] = (float)((2.0 * unit_double(mix64(seed * 0x9E37ull + off + i)) - 1.0) * lim);
    };
    fill(m->off_w1, (size_t)in_dim * kH, in_dim);
    fill(m->off_w2, (size_t)kH * kH, kH);
    fill(m->off_w3, (size_t)kH * out_dim, kH);
    for (float &x : h) x = __bfloat162float(__float2bfloat16_rn(x));
    SCAPH_CUDA(cudaMemcpy(m->w, h.data(), o * 4, cudaMemcpyHostToDevice));
    *out = m.release();
    return SCAPH_OK;
}

void scaph_mlp_destroy(scaph_mlp *m)
{
    if (!m) return;
    for (float *p : {m->w, m->g, m->m, m->v, m->X, m->H1, m->H2, m->Y, m->T, m->Wt, m->dY, m->dH2, m->dH1, m->lt,
                     m->loss})
        cudaFree(p);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
}

size_t scaph_mlp_num_params(const scaph_mlp *m) { return m ? m->nparams : 0; }

int scaph_mlp_get_params(const scaph_mlp *m, float *out, size_t n)
{
    if (!m || !out || n < m->nparams) return set_error(SCAPH_EINVAL, "bad argument");
    SCAPH_CUDA(cudaMemcpy(out, m->w, m->nparams * 4, cudaMemcpyDeviceToHost));
    return SCAPH_OK;
}

int scaph_mlp_set_params(scaph_mlp *m, const float *in, size_t n)
{
    if (!m || !in || n < m->nparams) return set_error(SCAPH_EINVAL, "bad argument");
    std::vector<float> h(in, in + m->nparams);
    for (float &x : h) x = __bfloat162float(__float2bfloat16_rn(x));
    SCAPH_CUDA(cudaMemcpy(m->w, h.data(), m->nparams * 4, cudaMemcpyHostToDevice));
    return SCAPH_OK;
}

int scaph_mlp_forward(scaph_mlp *m, const float *X, int n, float *Y)
{
    clear_error();
    if (!m || !X || !Y || n < 1) return set_error(SCAPH_EINVAL, "bad argument");
    SCAPH_CUDA(cudaSetDevice(m->device));
    return mlp_forward_device(m, X, n, Y);
}

// Weighted sigmoid cross-entropy of the n rows (T targets in [0,1], W
// per-output weights) and its gradient w.r.t. every parameter (grad may be
// NULL).
int scaph_mlp_loss_grad(scaph_mlp *m, const float *X, const float *T, const float *W, int n, float *loss,
                        float *grad)
{
    clear_error();
    if (!m || !X || !T || !W || n < 1) return set_error(SCAPH_EINVAL, "bad argument");
    SCAPH_CUDA(cudaSetDevice(m->device));
    int rc = m->upload(X, T, W, n);
    if (rc || (rc = m->forward(n)) || (rc = m->backward(n))) return rc;
    if (loss) SCAPH_CUDA(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
    if (grad) SCAPH_CUDA(cudaMemcpyAsync(grad, m->g, m->nparams * 4, cudaMemcpyDeviceToHost, m->st));
    SCAPH_CUDA(cudaStreamSynchronize(m->st));
    return SCAPH_OK;
}

// One Adam step on the n rows given (beta1 0.9, beta2 0.999, eps 1e-8) on
// the FP32 master weights; every use rounds them to bf16.
int scaph_mlp_adam_step(scaph_mlp *m, const float *X, const float *T, const float *W, int n, float lr, float *loss)
{
    clear_error();
    if (!m || !X || !T || !W || n < 1) return set_error(SCAPH_EINVAL, "bad argument");
    SCAPH_CUDA(cudaSetDevice(m->device));
    int rc = m->upload(X, T, W, n);
    if (rc || (rc = m->forward(n)) || (rc = m->backward(n))) return rc;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    k_adam<<<grid_of(m->nparams), 256, 0, m->st>>>(m->w, m->g, m->m, m->v, m->nparams, lr, b1, b2, 1e-8f, c1, c2);
    SCAPH_CUDA(cudaGetLastError());
    if (loss) SCAPH_CUDA(cudaMemcpyAsync(loss, m->loss, 4, cudaMemcpyDeviceToHost, m->st));
    SCAPH_CUDA(cudaStreamSynchronize(m->st));
    return SCAPH_OK;
}

// Device time (CUDA events on the network's stream, mean over `reps`) of:
// out_us[0] a forward pass over n rows, out_us[1] one training step on n
// rows (forward, loss, backward, Adam), out_us[2] the single-row inference
// kernel (the network part of the graph-mode learned decision).  Inputs are
// zero rows already on the device, so no host copy is timed; the parameters
// and Adam state are restored afterwards.
int scaph_mlp_time(scaph_mlp *m, int n, int reps, float *out_us)
{
    clear_error();
    if (!m || n < 1 || reps < 1 || !out_us) return set_error(SCAPH_EINVAL, "bad argument");
    SCAPH_CUDA(cudaSetDevice(m->device));
    int rc = m->ensure(n);
    if (rc) return rc;
    SCAPH_CUDA(cudaMemsetAsync(m->X, 0, sizeof(float) * n * m->in, m->st));
    SCAPH_CUDA(cudaMemsetAsync(m->T, 0, sizeof(float) * n * m->out, m->st));
    SCAPH_CUDA(cudaMemsetAsync(m->Wt, 0, sizeof(float) * n * m->out, m->st));
    float *save = nullptr;
    SCAPH_CUDA(cudaMalloc(&save, sizeof(float) * 3 * m->nparams));
    SCAPH_CUDA(cudaMemcpyAsync(save, m->w, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice, m->st));
    SCAPH_CUDA(cudaMemcpyAsync(save + m->nparams, m->m, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice, m->st));
    SCAPH_CUDA(cudaMemcpyAsync(save + 2 * m->nparams, m->v, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice,
                               m->st));
    cudaEvent_t e[2];
    SCAPH_CUDA(cudaEventCreate(&e[0]));
    SCAPH_CUDA(cudaEventCreate(&e[1]));
    auto timed = [&](auto &&body, float *us) -> int {
        int r = body();  // warm
        if (r) return r;
        SCAPH_CUDA(cudaEventRecord(e[0], m->st));
        for (int i = 0; i < reps && !r; i++) r = body();
        SCAPH_CUDA(cudaEventRecord(e[1], m->st));
        SCAPH_CUDA(cudaEventSynchronize(e[1]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e[0], e[1]);
        *us = ms * 1e3f / (float)reps;
        return r;
    };
    rc = timed([&]() { return m->forward(n); }, &out_us[0]);
    if (!rc)
        rc = timed([&]() -> int {
            int r = m->forward(n);
            if (r || (r = m->backward(n))) return r;
            k_adam<<<grid_of(m->nparams), 256, 0, m->st>>>(m->w, m->g, m->m, m->v, m->nparams, 1e-3f, 0.9f, 0.999f,
                                                           1e-8f, 0.5f, 0.5f);
            return cudaGetLastError() == cudaSuccess ? SCAPH_OK : set_error(SCAPH_ECUDA, "adam launch");
        }, &out_us[1]);
    if (!rc)
        rc = timed([&]() -> int {
            k_forward1<<<1, 256, sizeof(float) * m->in, m->st>>>(m->w, m->in, m->out, m->off_w1, m->off_b1,
                                                                  m->off_w2, m->off_b2, m->off_w3, m->off_b3, m->X,
                                                                  m->Y);
            return cudaGetLastError() == cudaSuccess ? SCAPH_OK : set_error(SCAPH_ECUDA, "forward1 launch");
        }, &out_us[2]);
    cudaMemcpyAsync(m->w, save, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice, m->st);
    cudaMemcpyAsync(m->m, save + m->nparams, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice, m->st);
    cudaMemcpyAsync(m->v, save + 2 * m->nparams, sizeof(float) * m->nparams, cudaMemcpyDeviceToDevice, m->st);
    cudaStreamSynchronize(m->st);
    cudaFree(save);
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    return rc;
}

// Minibatch training: `epochs` passes over the n rows in a seeded order.
int scaph_mlp_train(scaph_mlp *m, const float *X, const float *T, const float *W, int n, int epochs, int batch,
                    float lr, uint64_t seed, float *final_loss)
{
    clear_error();
    if (!m || !X || !T || !W || n < 1 || epochs < 1 || batch < 1) return set_error(SCAPH_EINVAL, "bad argument");
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::vector<float> bx((size_t)batch * m->in), bt((size_t)batch * m->out), bw((size_t)batch * m->out);
    float loss = 0.f;
    for (int ep = 0; ep < epochs; ep++) {
        for (int i = n - 1; i > 0; i--) {
            const int j = (int)(mix64(seed + (uint64_t)ep * 1000003ull + (uint64_t)i) % (uint64_t)(i + 1));
            std::swap(order[i], order[j]);
        }
        for (int b0 = 0; b0 < n; b0 += batch) {
            const int nb = std::min(batch, n - b0);
            for (int r = 0; r < nb; r++) {
                const int s = order[b0 + r];
                memcpy(&bx[(size_t)r * m->in], X + (size_t)s * m->in, sizeof(float) * m->in);
                memcpy(&bt[(size_t)r * m->out], T + (size_t)s * m->out, sizeof(float) * m->out);
                memcpy(&bw[(size_t)r * m->out], W + (size_t)s * m->out, sizeof(float) * m->out);
            }
            int rc = scaph_mlp_adam_step(m, bx.data(), bt.data(), bw.data(), nb, lr, &loss);
            if (rc) return rc;
        }
    }
    if (final_loss) *final_loss = loss;
    return SCAPH_OK;
}

// Checkpoint: dims, step, the FP32 master weights and the FP32 Adam moments.
int scaph_mlp_save(const scaph_mlp *m, const char *path)
{
    if (!m || !path) return set_error(SCAPH_EINVAL, "bad argument");
    std::vector<float> w(m->nparams), mm(m->nparams), vv(m->nparams);
    SCAPH_CUDA(cudaMemcpy(w.data(), m->w, m->nparams * 4, cudaMemcpyDeviceToHost));
    SCAPH_CUDA(cudaMemcpy(mm.data(), m->m, m->nparams * 4, cudaMemcpyDeviceToHost));
    SCAPH_CUDA(cudaMemcpy(vv.data(), m->v, m->nparams * 4, cudaMemcpyDeviceToHost));
    FILE *f = fopen(path, "wb");
    if (!f) return set_error(SCAPH_EIO, "cannot create %s", path);
    const int32_t hdr[4] = {0x53434D4C, m->in, m->out, m->step};
    bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1 && fwrite(w.data(), 4, m->nparams, f) == m->nparams &&
              fwrite(mm.data(), 4, m->nparams, f) == m->nparams && fwrite(vv.data(), 4, m->nparams, f) == m->nparams;
    ok = (fclose(f) == 0) && ok;
    return ok ? SCAPH_OK : set_error(SCAPH_EIO, "short write to %s", path);
}

int scaph_mlp_load(scaph_mlp *m, const char *path)
{
    if (!m || !path) return set_error(SCAPH_EINVAL, "bad argument");
    FILE *f = fopen(path, "rb");
    if (!f) return set_error(SCAPH_EIO, "cannot open %s", path);
    int32_t hdr[4];
    std::vector<float> w(m->nparams), mm(m->nparams), vv(m->nparams);
    bool ok = fread(hdr, sizeof(hdr), 1, f) == 1 && hdr[0] == 0x53434D4C && hdr[1] == m->in && hdr[2] == m->out &&
              fread(w.data(), 4, m->nparams, f) == m->nparams && fread(mm.data(), 4, m->nparams, f) == m->nparams &&
              fread(vv.data(), 4, m->nparams, f) == m->nparams;
    fclose(f);
    if (!ok) return set_error(SCAPH_EFORMAT, "%s is not a checkpoint of this network", path);
    m->step = hdr[3];
    SCAPH_CUDA(cudaMemcpy(m->w, w.data(), m->nparams * 4, cudaMemcpyHostToDevice));
    SCAPH_CUDA(cudaMemcpy(m->m, mm.data(), m->nparams * 4, cudaMemcpyHostToDevice));
    SCAPH_CUDA(cudaMemcpy(m->v, vv.data(), m->nparams * 4, cudaMemcpyHostToDevice));
    return SCAPH_OK;
}

}  // extern "C"
