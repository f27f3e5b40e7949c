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
#include <cooperative_groups.h>
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

// ------------------------------------------------- fused ensemble inference
// The picker evaluates a handful of models on one 16-row batch per pick:
// at that size the per-layer GEMM, bias and GELU launches cost far more
// than the arithmetic.  One launch does it all: CTA (m, t) runs model m on
// rows [16t, 16t + 16) through every layer, with the activations in shared
// memory (bf16, as the layered path rounds them), warp-level bf16 tensor-core
// tiles (mma m16n8k16, fp32 accumulation) whose B operands stream straight
// from the model's bf16 weights in L2, and bias + GELU fused into the tile
// epilogue.  The models of one row tile form a thread-block cluster; once
// every model's output tile is in its CTA's shared memory, CTA 0 of the
// cluster reads them through distributed shared memory and writes their
// mean, summed in model order (deterministic).
constexpr int kEnsMaxModels = 8;  // portable cluster size
constexpr int kEnsH = 256;        // hidden width the fused kernel is built for
constexpr int kEnsMaxOut = 256;
constexpr int kEnsThreads = 1024;  // 32 warps: one 8-column tile each (widths up to 256)

struct EnsModel {
    const bf16* wb;   // bf16 weights (layer l at woff[l], [out][in] row-major)
    const float* w;   // fp32 arena (biases at boff[l])
};
struct EnsArgs {
    EnsModel m[kEnsMaxModels];
    long long woff[4], boff[4];
    int nmodels, din, dout;
    const float* x;  // [n][din]
    float* y;        // [n][dout], the mean over the models
};

__device__ __forceinline__ void mma_bf16_16816(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One layer for 16 rows: out[16][N] = act[16][K] W^T + bias, then GELU into
// the next activation buffer (hidden) or fp32 into `outf` (last layer).
// Warp w owns the n-tile w (8 columns; N <= 8 * warps).  Its weight
// fragments for the whole K (at most 16 k-steps, two 32-bit registers each)
// and its two bias values are loaded in one round (ens_fetch), and the
// kernel issues the next layer's round as soon as this layer's mma chain
// has consumed the fragments, so that the L2 latency of layer l + 1 runs
// under layer l's epilogue and block barrier.
//
// Which columns of a 32-column block feed which k slots of the mma is free,
// as long as A and B agree: lane (g, t) gives k-step 2j the columns
// 32j + 8t + {0,1} (slots 2t, 2t+1) and 32j + 8t + {2,3} (slots 2t+8,
// 2t+9), and k-step 2j+1 the columns 32j + 8t + {4..7}.  Each lane then
// reads 16 contiguous bytes of its weight row per two k-steps (one
// fully-used 32-byte sector pair per row and instruction, a quarter of the
// load instructions of the mma's natural column order) and 16 contiguous
// bytes of each activation row.  A trailing single k-step (K not a
// multiple of 32) takes columns 4t + {0,1} and 4t + {2,3} of its 16.
struct EnsFrag {
    uint32_t b[16][2];
    float b0, b1;
};

__device__ __forceinline__ void ens_fetch(EnsFrag& f, int K, const bf16* __restrict__ W, const float* __restrict__ bias,
                                          int N) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    if (warp * 8 >= N) return;
    const int npair = K / 32;
    const bf16* wr = W + (size_t)(warp * 8 + g) * K;
#pragma unroll
    for (int j = 0; j < 8; j++) {  // unrolled: the fragment indices stay static (registers)
        if (j < npair) {
            const uint4 v = __ldg(reinterpret_cast<const uint4*>(wr + 32 * j + 8 * t));
            f.b[2 * j][0] = v.x;
            f.b[2 * j][1] = v.y;
            f.b[2 * j + 1][0] = v.z;
            f.b[2 * j + 1][1] = v.w;
        } else if (j == npair && (K % 32)) {
            const uint2 v = __ldg(reinterpret_cast<const uint2*>(wr + 32 * j + 4 * t));
            f.b[2 * j][0] = v.x;
            f.b[2 * j][1] = v.y;
        }
    }
    const int c = warp * 8 + 2 * t;
    f.b0 = __ldg(bias + c);
    f.b1 = __ldg(bias + c + 1);
}

// The mma chain of one layer from fragments already in registers.
__device__ __forceinline__ void ens_mma(float* acc, const bf16* __restrict__ act, int lda, int K, const EnsFrag& f) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int npair = K / 32;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        if (j < npair) {
            const uint4 r0 = *reinterpret_cast<const uint4*>(act + g * lda + 32 * j + 8 * t);
            const uint4 r1 = *reinterpret_cast<const uint4*>(act + (g + 8) * lda + 32 * j + 8 * t);
            const uint32_t a0[4] = {r0.x, r1.x, r0.y, r1.y};
            const uint32_t a1[4] = {r0.z, r1.z, r0.w, r1.w};
            mma_bf16_16816(acc, a0, f.b[2 * j]);
            mma_bf16_16816(acc, a1, f.b[2 * j + 1]);
        } else if (j == npair && (K % 32)) {
            const uint2 r0 = *reinterpret_cast<const uint2*>(act + g * lda + 32 * j + 4 * t);
            const uint2 r1 = *reinterpret_cast<const uint2*>(act + (g + 8) * lda + 32 * j + 4 * t);
            const uint32_t a[4] = {r0.x, r1.x, r0.y, r1.y};
            mma_bf16_16816(acc, a, f.b[2 * j]);
        }
    }
}

// Bias and GELU into the next activation buffer, or fp32 output.
__device__ __forceinline__ void ens_epilogue(const float* acc, float b0, float b1, bf16* next, int ldn, float* outf,
                                             int ldo) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int c = warp * 8 + 2 * t;
    const float v[4] = {acc[0] + b0, acc[1] + b1, acc[2] + b0, acc[3] + b1};
    if (next) {
        *(__nv_bfloat162*)(next + g * ldn + c) = __floats2bfloat162_rn(gelu(v[0]), gelu(v[1]));
        *(__nv_bfloat162*)(next + (g + 8) * ldn + c) = __floats2bfloat162_rn(gelu(v[2]), gelu(v[3]));
    } else {
        outf[g * ldo + c] = v[0];
        outf[g * ldo + c + 1] = v[1];
        outf[(g + 8) * ldo + c] = v[2];
        outf[(g + 8) * ldo + c + 1] = v[3];
    }
}

__global__ void __launch_bounds__(kEnsThreads) k_mlp_ensemble(EnsArgs a) {
    namespace cg = cooperative_groups;
    // Padded rows (144 words, 16 mod 32): the 16-byte activation loads of a
    // quarter warp (rows g, g + 1; t = 0..3) fall on all 32 banks once.
    constexpr int kLd = kEnsH + 32;
    __shared__ __align__(16) bf16 s_act[2][16 * kLd];
    __shared__ __align__(16) float s_out[16 * kEnsMaxOut];
    cg::cluster_group cluster = cg::this_cluster();
    const int model = (int)cluster.block_rank();
    const int row0 = blockIdx.y * 16;
    const EnsModel M = a.m[model];
    const int dims[5] = {a.din, kEnsH, kEnsH, kEnsH, a.dout};
    const int warp = threadIdx.x >> 5;
    EnsFrag f;
    ens_fetch(f, dims[0], M.wb + a.woff[0], M.w + a.boff[0], dims[1]);
    for (int i = threadIdx.x; i < 16 * a.din; i += kEnsThreads) {
        const int r = i / a.din, k = i % a.din;
        s_act[0][r * kLd + k] = __float2bfloat16(a.x[(size_t)(row0 + r) * a.din + k]);
    }
    __syncthreads();
#pragma unroll 1
    for (int l = 0; l < 4; l++) {
        const bf16* in = s_act[l & 1];
        bf16* nxt = l < 3 ? s_act[(l + 1) & 1] : nullptr;
        if (warp * 8 < dims[l + 1]) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            ens_mma(acc, in, kLd, dims[l], f);
            const float b0 = f.b0, b1 = f.b1;
            if (l < 3) ens_fetch(f, dims[l + 1], M.wb + a.woff[l + 1], M.w + a.boff[l + 1], dims[l + 2]);
            ens_epilogue(acc, b0, b1, nxt, kLd, s_out, a.dout);
        } else if (l < 3) {
            ens_fetch(f, dims[l + 1], M.wb + a.woff[l + 1], M.w + a.boff[l + 1], dims[l + 2]);
        }
        __syncthreads();
    }
    cluster.sync();
    if (model == 0) {
        const float inv = 1.0f / (float)a.nmodels;
        for (int i = threadIdx.x; i < 16 * a.dout; i += kEnsThreads) {
            float sum = 0.f;
            for (int m = 0; m < a.nmodels; m++) sum += cluster.map_shared_rank(s_out, m)[i];
            a.y[(size_t)(row0 + i / a.dout) * a.dout + i % a.dout] = sum * inv;
        }
    }
    cluster.sync();  // keep every CTA's shared memory alive until CTA 0 has read it
}

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

struct bine_mlp_ensemble_s {
    std::vector<bine_mlp_t> models;
};

int bine_mlp_ensemble_create(const bine_mlp_t* models, int nmodels, bine_mlp_ensemble_t* out) {
    if (!out || !models || nmodels < 1 || nmodels > kEnsMaxModels)
        return mfail(BINE_ERR_ARG, "an ensemble holds 1 to 8 models");
    *out = nullptr;
    const bine_mlp_t m0 = models[0];
    if (!m0) return mfail(BINE_ERR_ARG, "null model");
    if (m0->h != kEnsH || m0->din > kEnsH || m0->dout > kEnsMaxOut)
        return mfail(BINE_ERR_ARG, "the fused forward takes hidden width 256, input and output widths up to 256");
    for (int i = 1; i < nmodels; i++)
        if (!models[i] || models[i]->din != m0->din || models[i]->h != m0->h || models[i]->dout != m0->dout)
            return mfail(BINE_ERR_ARG, "the models of an ensemble must have the same shape");
    auto e = new bine_mlp_ensemble_s();
    e->models.assign(models, models + nmodels);
    *out = e;
    return BINE_SUCCESS;
}

int bine_mlp_ensemble_destroy(bine_mlp_ensemble_t e) {
    delete e;
    return BINE_SUCCESS;
}

int bine_mlp_ensemble_forward(bine_mlp_ensemble_t e, const float* d_x, int n, float* d_y, void* stream) {
    if (!e || !d_x || !d_y || n <= 0 || n % 16) return mfail(BINE_ERR_ARG, "batch must be a positive multiple of 16");
    if (n / 16 > 65535) return mfail(BINE_ERR_ARG, "batch too large for one launch");
    EnsArgs a{};
    const bine_mlp_t m0 = e->models[0];
    for (int l = 0; l < 4; l++) {
        a.woff[l] = (long long)m0->woff[l];
        a.boff[l] = (long long)m0->boff[l];
    }
    a.nmodels = (int)e->models.size();
    for (int i = 0; i < a.nmodels; i++) a.m[i] = EnsModel{e->models[i]->wb, e->models[i]->w};
    a.din = m0->din;
    a.dout = m0->dout;
    a.x = d_x;
    a.y = d_y;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)a.nmodels, (unsigned)(n / 16), 1);
    cfg.blockDim = dim3(kEnsThreads, 1, 1);
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)a.nmodels;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MLP_TRY(cudaLaunchKernelEx(&cfg, k_mlp_ensemble, a));
    return BINE_SUCCESS;
}

}  // extern "C"
