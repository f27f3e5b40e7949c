// Small multilayer perceptron for the learned variant picker: forward,
// backward and Adam training kernels with bf16 weights and activations and
// fp32 accumulation.
//
// Shape: in -> H -> H -> H -> out (3 hidden layers of width H, GELU after
// each hidden layer, exact erf form).  All dimensions are multiples of 16.
// GEMMs use warp-level tensor-core tiles (wmma 16x16x16, bf16 in, fp32
// accumulate); at this model size (H = 256) the network is bound by launch
// latency, not by tensor throughput.
//
//   forward:  pre_l = act_{l-1} W_l^T + b_l (fp32), act_l = bf16(gelu(pre_l))
//   loss:     masked mean squared error of the output against targets
//   backward: d_pre = d_act * gelu'(pre) (rounded to bf16 for the GEMMs),
//             dW_l = d_pre^T act_{l-1}, db_l = column sums, d_act_{l-1} = d_pre W_l
//   update:   Adam on fp32 master weights, refreshed bf16 copies.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <cmath>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/bine_b200.h"

namespace {

using bf16 = __nv_bfloat16;
using namespace nvcuda;

thread_local std::string g_mlp_err;

int mfail(int code, const std::string& m) {
    g_mlp_err = m;
    return code;
}

#define MLP_TRY(expr)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess) return mfail(BINE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// C[M x N] (fp32, row-major, ldc) = A[M x K] * B[K x N]; A and B bf16 in the
// given layouts.  Block: 4 warps, 64 x 64 tile; warp: 32 x 32 (2 x 2 tiles).
template <typename ALayout, typename BLayout>
__global__ void __launch_bounds__(128) k_gemm(const bf16* __restrict__ A, int lda, const bf16* __restrict__ B,
                                              int ldb, float* __restrict__ C, int ldc, int M, int N, int K) {
    const int warp = threadIdx.x / 32;
    const int wm = blockIdx.y * 64 + (warp / 2) * 32;
    const int wn = blockIdx.x * 64 + (warp % 2) * 32;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) wmma::fill_fragment(acc[i][j], 0.0f);
    for (int k = 0; k < K; k += 16) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, ALayout> a[2];
        wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, BLayout> b[2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int r = wm + i * 16;
            if (r < M) {
                const bf16* p = std::is_same<ALayout, wmma::row_major>::value ? A + (size_t)r * lda + k
                                                                              : A + (size_t)k * lda + r;
                wmma::load_matrix_sync(a[i], p, lda);
            }
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const int c = wn + j * 16;
            if (c < N) {
                const bf16* p = std::is_same<BLayout, wmma::row_major>::value ? B + (size_t)k * ldb + c
                                                                              : B + (size_t)c * ldb + k;
                wmma::load_matrix_sync(b[j], p, ldb);
            }
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
#pragma unroll
            for (int j = 0; j < 2; j++)
                if (wm + i * 16 < M && wn + j * 16 < N) wmma::mma_sync(acc[i][j], a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++)
            if (wm + i * 16 < M && wn + j * 16 < N)
                wmma::store_matrix_sync(C + (size_t)(wm + i * 16) * ldc + wn + j * 16, acc[i][j], ldc,
                                        wmma::mem_row_major);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// pre += bias; act = bf16(gelu(pre)) (hidden) or out = pre (last layer).
__global__ void k_bias_act(float* pre, const float* bias, bf16* act, int M, int N, int hidden) {
    const long long n = (long long)M * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float v = pre[i] + bias[i % N];
        pre[i] = v;
        if (hidden) act[i] = __float2bfloat16(gelu(v));
    }
}

// Masked MSE: d = mask * (y - t); loss += d^2; grad = bf16(2 d / count).
__global__ void k_loss(const float* y, const float* t, const float* mask, bf16* grad, float* loss, int M, int N,
                       float inv_count) {
    __shared__ float red[256];
    float acc = 0.f;
    const long long n = (long long)M * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = mask[i] * (y[i] - t[i]);
        acc += d * d;
        grad[i] = __float2bfloat16(2.0f * d * inv_count);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] * inv_count);
}

// d_pre = bf16(d_act * gelu'(pre)).
__global__ void k_gelu_back(const float* dact, const float* pre, bf16* dpre, int M, int N) {
    const long long n = (long long)M * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dpre[i] = __float2bfloat16(dact[i] * gelu_grad(pre[i]));
}

// db[j] = sum_i d_pre[i][j] (fp32 accumulation of the bf16 gradients).
__global__ void k_colsum(const bf16* g, float* db, int M, int N) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    float s = 0.f;
    for (int i = 0; i < M; i++) s += __bfloat162float(g[(size_t)i * N + j]);
    db[j] = s;
}

__global__ void k_to_bf16(const float* x, bf16* y, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, bf16* wb, long long n, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

unsigned grid1(long long n) { return (unsigned)std::max(1LL, std::min((n + 255) / 256, 148LL * 8)); }

}  // namespace

struct bine_mlp_s {
    int din, h, dout, max_batch;
    int nlayer = 4;
    int in_dim[4], out_dim[4];
    // fp32 master weights and biases (one arena), gradients, Adam moments.
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    bf16* wb = nullptr;  // bf16 weights (same offsets as w, biases unused)
    size_t woff[4], boff[4], nparams = 0;
    long long step = 0;
    // Activations for max_batch rows.
    bf16* x = nullptr;           // input, bf16
    float* pre[4] = {nullptr};   // pre-activations / outputs (fp32)
    bf16* act[3] = {nullptr};    // hidden activations (bf16)
    float* dact = nullptr;       // backprop scratch (fp32)
    bf16* dpre = nullptr;        // bf16 gradient of the current layer
    float* loss = nullptr;
    float* t = nullptr;          // targets
    float* mask = nullptr;
    ~bine_mlp_s() {
        cudaFree(w);
        cudaFree(g);
        cudaFree(m);
        cudaFree(v);
        cudaFree(wb);
        cudaFree(x);
        for (float* p : pre) cudaFree(p);
        for (bf16* p : act) cudaFree(p);
        cudaFree(dact);
        cudaFree(dpre);
        cudaFree(loss);
        cudaFree(t);
        cudaFree(mask);
    }
};

namespace {

template <typename AL, typename BL>
void gemm(const bf16* A, int lda, const bf16* B, int ldb, float* C, int ldc, int M, int N, int K, cudaStream_t s) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_gemm<AL, BL><<<grid, 128, 0, s>>>(A, lda, B, ldb, C, ldc, M, N, K);
}

// Forward pass of `n` rows already in mlp->x.
void forward(bine_mlp_t mlp, int n, cudaStream_t s) {
    const bf16* in = mlp->x;
    for (int l = 0; l < mlp->nlayer; l++) {
        const int K = mlp->in_dim[l], N = mlp->out_dim[l];
        gemm<wmma::row_major, wmma::col_major>(in, K, mlp->wb + mlp->woff[l], K, mlp->pre[l], N, n, N, K, s);
        const bool hidden = l + 1 < mlp->nlayer;
        k_bias_act<<<grid1((long long)n * N), 256, 0, s>>>(mlp->pre[l], mlp->w + mlp->boff[l], hidden ? mlp->act[l] : nullptr,
                                                         n, N, hidden ? 1 : 0);
        if (hidden) in = mlp->act[l];
    }
}

// Backward pass from the output gradient in mlp->dpre (bf16, n x dout):
// fills mlp->g with the gradients of every weight and bias.
void backward(bine_mlp_t mlp, int n, cudaStream_t s) {
    for (int l = mlp->nlayer - 1; l >= 0; l--) {
        const int K = mlp->in_dim[l], N = mlp->out_dim[l];
        const bf16* a_in = l == 0 ? mlp->x : mlp->act[l - 1];
        // dW = d_pre^T (N x n) * a_in (n x K): fp32 into the gradient arena.
        gemm<wmma::col_major, wmma::row_major>(mlp->dpre, N, a_in, K, mlp->g + mlp->woff[l], K, N, K, n, s);
        k_colsum<<<(N + 127) / 128, 128, 0, s>>>(mlp->dpre, mlp->g + mlp->boff[l], n, N);
        if (l > 0) {
            // d_act_{l-1} = d_pre (n x N) * W (N x K).
            gemm<wmma::row_major, wmma::row_major>(mlp->dpre, N, mlp->wb + mlp->woff[l], K, mlp->dact, K, n, K, N, s);
            k_gelu_back<<<grid1((long long)n * K), 256, 0, s>>>(mlp->dact, mlp->pre[l - 1], mlp->dpre, n, K);
        }
    }
}

int load_batch(bine_mlp_t mlp, const float* d_x, int n, cudaStream_t s) {
    if (!mlp || !d_x || n <= 0 || n > mlp->max_batch || n % 16) return mfail(BINE_ERR_ARG, "batch must be a multiple of 16 within max_batch");
    k_to_bf16<<<grid1((long long)n * mlp->din), 256, 0, s>>>(d_x, mlp->x, (long long)n * mlp->din);
    return BINE_SUCCESS;
}

int loss_and_grad(bine_mlp_t mlp, const float* d_t, const float* d_mask, int n, cudaStream_t s) {
    MLP_TRY(cudaMemsetAsync(mlp->loss, 0, sizeof(float), s));
    MLP_TRY(cudaMemcpyAsync(mlp->t, d_t, sizeof(float) * (size_t)n * mlp->dout, cudaMemcpyDeviceToDevice, s));
    MLP_TRY(cudaMemcpyAsync(mlp->mask, d_mask, sizeof(float) * (size_t)n * mlp->dout, cudaMemcpyDeviceToDevice, s));
    // Mean over the valid (mask != 0) entries: the caller's mask count.
    std::vector<float> hm((size_t)n * mlp->dout);
    MLP_TRY(cudaMemcpyAsync(hm.data(), d_mask, sizeof(float) * hm.size(), cudaMemcpyDeviceToHost, s));
    MLP_TRY(cudaStreamSynchronize(s));
    double cnt = 0;
    for (float q : hm) cnt += q != 0.f;
    const float inv = cnt > 0 ? (float)(1.0 / cnt) : 0.f;
    k_loss<<<grid1((long long)n * mlp->dout), 256, 0, s>>>(mlp->pre[mlp->nlayer - 1], mlp->t, mlp->mask, mlp->dpre,
                                                           mlp->loss, n, mlp->dout, inv);
    return BINE_SUCCESS;
}

}  // namespace

extern "C" {

const char* bine_mlp_last_error(void) { return g_mlp_err.c_str(); }

int bine_mlp_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed, bine_mlp_t* out) {
    if (!out || in_dim <= 0 || hidden <= 0 || out_dim <= 0 || max_batch <= 0 || in_dim % 16 || hidden % 16 ||
        out_dim % 16 || max_batch % 16)
        return mfail(BINE_ERR_ARG, "dimensions must be positive multiples of 16");
    *out = nullptr;
    auto m = std::unique_ptr<bine_mlp_s>(new bine_mlp_s());
    m->din = in_dim;
    m->h = hidden;
    m->dout = out_dim;
    m->max_batch = max_batch;
    const int dims[5] = {in_dim, hidden, hidden, hidden, out_dim};
    size_t off = 0;
    for (int l = 0; l < 4; l++) {
        m->in_dim[l] = dims[l];
        m->out_dim[l] = dims[l + 1];
        m->woff[l] = off;
        off += (size_t)dims[l] * dims[l + 1];
        off = (off + 15) / 16 * 16;
        m->boff[l] = off;
        off += (size_t)dims[l + 1];
        off = (off + 15) / 16 * 16;
    }
    m->nparams = off;
    // He-style initialisation from a seeded generator; biases zero.
    std::vector<float> hw(off, 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < 4; l++) {
        std::normal_distribution<float> nd(0.f, std::sqrt(2.0f / dims[l]) * (l == 3 ? 0.5f : 1.0f));
        for (size_t i = 0; i < (size_t)dims[l] * dims[l + 1]; i++) hw[m->woff[l] + i] = nd(rng);
    }
    MLP_TRY(cudaMalloc(&m->w, off * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->g, off * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->m, off * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->v, off * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->wb, off * sizeof(bf16)));
    MLP_TRY(cudaMemcpy(m->w, hw.data(), off * sizeof(float), cudaMemcpyHostToDevice));
    MLP_TRY(cudaMemset(m->g, 0, off * sizeof(float)));
    MLP_TRY(cudaMemset(m->m, 0, off * sizeof(float)));
    MLP_TRY(cudaMemset(m->v, 0, off * sizeof(float)));
    k_to_bf16<<<grid1(off), 256>>>(m->w, m->wb, (long long)off);
    MLP_TRY(cudaMalloc(&m->x, (size_t)max_batch * in_dim * sizeof(bf16)));
    for (int l = 0; l < 4; l++) MLP_TRY(cudaMalloc(&m->pre[l], (size_t)max_batch * dims[l + 1] * sizeof(float)));
    for (int l = 0; l < 3; l++) MLP_TRY(cudaMalloc(&m->act[l], (size_t)max_batch * hidden * sizeof(bf16)));
    const int wmax = std::max(std::max(in_dim, hidden), out_dim);
    MLP_TRY(cudaMalloc(&m->dact, (size_t)max_batch * wmax * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->dpre, (size_t)max_batch * wmax * sizeof(bf16)));
    MLP_TRY(cudaMalloc(&m->loss, sizeof(float)));
    MLP_TRY(cudaMalloc(&m->t, (size_t)max_batch * out_dim * sizeof(float)));
    MLP_TRY(cudaMalloc(&m->mask, (size_t)max_batch * out_dim * sizeof(float)));
    MLP_TRY(cudaDeviceSynchronize());
    *out = m.release();
    return BINE_SUCCESS;
}

int bine_mlp_destroy(bine_mlp_t mlp) {
    delete mlp;
    return BINE_SUCCESS;
}

int bine_mlp_num_params(bine_mlp_t mlp, size_t* n) {
    if (!mlp || !n) return mfail(BINE_ERR_ARG, "null argument");
    *n = mlp->nparams;
    return BINE_SUCCESS;
}

int bine_mlp_get_params(bine_mlp_t mlp, float* host) {
    if (!mlp || !host) return mfail(BINE_ERR_ARG, "null argument");
    MLP_TRY(cudaMemcpy(host, mlp->w, mlp->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    return BINE_SUCCESS;
}

int bine_mlp_set_params(bine_mlp_t mlp, const float* host) {
    if (!mlp || !host) return mfail(BINE_ERR_ARG, "null argument");
    MLP_TRY(cudaMemcpy(mlp->w, host, mlp->nparams * sizeof(float), cudaMemcpyHostToDevice));
    k_to_bf16<<<grid1(mlp->nparams), 256>>>(mlp->w, mlp->wb, (long long)mlp->nparams);
    MLP_TRY(cudaDeviceSynchronize());
    return BINE_SUCCESS;
}

int bine_mlp_forward(bine_mlp_t mlp, const float* d_x, int n, float* d_y, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    int rc = load_batch(mlp, d_x, n, s);
    if (rc) return rc;
    forward(mlp, n, s);
    MLP_TRY(cudaMemcpyAsync(d_y, mlp->pre[mlp->nlayer - 1], sizeof(float) * (size_t)n * mlp->dout,
                            cudaMemcpyDeviceToDevice, s));
    MLP_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int bine_mlp_gradients(bine_mlp_t mlp, const float* d_x, const float* d_t, const float* d_mask, int n, float* host_grads,
                       float* loss) {
    cudaStream_t s = 0;
    int rc = load_batch(mlp, d_x, n, s);
    if (rc) return rc;
    forward(mlp, n, s);
    rc = loss_and_grad(mlp, d_t, d_mask, n, s);
    if (rc) return rc;
    backward(mlp, n, s);
    MLP_TRY(cudaStreamSynchronize(s));
    if (host_grads) MLP_TRY(cudaMemcpy(host_grads, mlp->g, mlp->nparams * sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) MLP_TRY(cudaMemcpy(loss, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost));
    MLP_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

int bine_mlp_train_step(bine_mlp_t mlp, const float* d_x, const float* d_t, const float* d_mask, int n, float lr,
                        void* stream, float* loss) {
    cudaStream_t s = (cudaStream_t)stream;
    int rc = load_batch(mlp, d_x, n, s);
    if (rc) return rc;
    forward(mlp, n, s);
    rc = loss_and_grad(mlp, d_t, d_mask, n, s);
    if (rc) return rc;
    backward(mlp, n, s);
    mlp->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)mlp->step), c2 = 1.f - std::pow(b2, (float)mlp->step);
    k_adam<<<grid1(mlp->nparams), 256, 0, s>>>(mlp->w, mlp->g, mlp->m, mlp->v, mlp->wb, (long long)mlp->nparams, lr, b1,
                                               b2, 1e-8f, c1, c2);
    if (loss) {
        MLP_TRY(cudaMemcpyAsync(loss, mlp->loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        MLP_TRY(cudaStreamSynchronize(s));
    }
    MLP_TRY(cudaGetLastError());
    return BINE_SUCCESS;
}

}  // extern "C"
