// Surrogate network of the data-assimilation forecast: a multilayer
// perceptron in -> H -> H -> 1 with GELU, weights held in BF16 for compute
// (an FP32 master copy is what Adam updates), activations and every
// accumulation in FP32.  Forward, backward (MSE loss) and Adam are kernels of
// this file; there is no counterpart in the reference, whose forecast always
// runs the full simulator (data_assimilation/DataAssimilation.py:353-370).
//
// Parameter order (flat, FP32 master): W1[H][in], b1[H], W2[H][H], b2[H], W3[H], b3[1].
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dtb.h"

namespace {

thread_local std::string g_mlp_err;

int mlp_fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_mlp_err = buf;
    return code;
}

#define MCK(call)                                                                                         \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return mlp_fail(DTB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));    \
    } while (0)

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// ------------------------------------------------------------ kernels

__device__ __forceinline__ float load_f(const float* p) { return *p; }
__device__ __forceinline__ float load_f(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// C[M][N] (+)= A[M][K] * B[K][N] with arbitrary strides (transposes by stride),
// 64x64 output tile per CTA, 16-deep K chunks staged in shared memory, each of
// the 256 threads accumulating a 4x4 block in FP32.  gridDim.z splits K; with
// more than one split the partial tiles are added atomically (C pre-zeroed).
constexpr int TM = 64, TN = 64, TK = 16;

template <typename TA, typename TB>
__global__ void __launch_bounds__(256) k_gemm(int M, int N, int64_t K, const TA* __restrict__ A, int64_t a_m,
                                              int64_t a_k, const TB* __restrict__ B, int64_t b_k, int64_t b_n,
                                              float* __restrict__ C, int64_t c_m, int64_t k_per_split)
{
    __shared__ float As[TK][TM + 4];
    __shared__ float Bs[TK][TN + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
    const int64_t k_begin = (int64_t)blockIdx.z * k_per_split;
    const int64_t k_end = k_begin + k_per_split < K ? k_begin + k_per_split : K;
    float acc[4][4] = {};
    for (int64_t k0 = k_begin; k0 < k_end; k0 += TK) {
        for (int i = threadIdx.x; i < TK * TM; i += 256) {
            const int kk = i / TM, mm = i % TM;
            const int64_t k = k0 + kk;
            const int m = m0 + mm;
            As[kk][mm] = (k < k_end && m < M) ? load_f(A + m * a_m + k * a_k) : 0.0f;
        }
        for (int i = threadIdx.x; i < TK * TN; i += 256) {
            const int kk = i / TN, nn = i % TN;
            const int64_t k = k0 + kk;
            const int n = n0 + nn;
            Bs[kk][nn] = (k < k_end && n < N) ? load_f(B + k * b_k + n * b_n) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            if (gridDim.z > 1) atomicAdd(C + m * c_m + n, acc[i][j]);
            else C[m * c_m + n] = acc[i][j];
        }
    }
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x)
{
    // d/dx [x Phi(x)] = Phi(x) + x phi(x)
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Z += bias (per column); H = GELU(Z) when act, else H = Z.
__global__ void k_bias_act(int64_t rows, int cols, float* Z, const float* __restrict__ bias, float* H, int act)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const float z = Z[i] + bias[i % cols];
    Z[i] = z;
    H[i] = act ? gelu(z) : z;
}

__global__ void k_gelu_bwd(int64_t n, const float* __restrict__ dH, const float* __restrict__ Z, float* dZ)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dZ[i] = dH[i] * gelu_grad(Z[i]);
}

// loss = mean((y - t)^2); dy = 2 (y - t) / B
__global__ void k_mse(int64_t n, const float* __restrict__ y, const float* __restrict__ t, float* dy, float* loss)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (i < n) {
        const float d = y[i] - t[i];
        dy[i] = 2.0f * d / (float)n;
        l = d * d / (float)n;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, l);
}

// column sums of dZ[rows][cols] into db[cols] (pre-zeroed)
__global__ void k_colsum(int64_t rows, int cols, const float* __restrict__ dZ, float* db)
{
    const int c = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r0 = blockIdx.y * 256 + (threadIdx.x >> 5);
    float s = 0.0f;
    if (c < cols)
        for (int64_t r = r0; r < rows && r < (int64_t)blockIdx.y * 256 + 256; r += 8) s += dZ[r * cols + c];
    __shared__ float sh[8][33];
    sh[threadIdx.x >> 5][threadIdx.x & 31] = s;
    __syncthreads();
    if (threadIdx.x < 32 && c < cols) {
        float t = 0.0f;
        for (int w = 0; w < 8; ++w) t += sh[w][threadIdx.x];
        atomicAdd(db + c, t);
    }
}

// Adam on the FP32 master weights; refresh the BF16 compute copy.
__global__ void k_adam(int64_t n, float* w, const float* __restrict__ g, float* m, float* v, __nv_bfloat16* wb,
                       float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
}

__global__ void k_to_bf16(int64_t n, const float* __restrict__ w, __nv_bfloat16* wb)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

}  // namespace

// ------------------------------------------------------------ handle
struct dtb_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    int in = 0, H = 0;
    int64_t n_params = 0;
    int64_t o_W1, o_b1, o_W2, o_b2, o_W3, o_b3;
    float* w = nullptr;            // FP32 master [n_params]
    __nv_bfloat16* wb = nullptr;   // BF16 compute copy
    float* g = nullptr;            // gradients
    float* m = nullptr;            // Adam moments
    float* v = nullptr;
    float* loss = nullptr;         // device scalar
    int64_t cap = 0;               // batch capacity of the activation buffers
    float *Z1 = nullptr, *H1 = nullptr, *Z2 = nullptr, *H2 = nullptr, *Y = nullptr;
    float *dY = nullptr, *dH2 = nullptr, *dZ2 = nullptr, *dH1 = nullptr, *dZ1 = nullptr;
    int64_t t = 0;                 // Adam step
};

namespace {

template <typename TA, typename TB>
int gemm(dtb_mlp* p, int M, int N, int64_t K, const TA* A, int64_t a_m, int64_t a_k, const TB* B, int64_t b_k,
         int64_t b_n, float* C, int64_t c_m, bool split)
{
    int splits = 1;
    if (split) {
        const int64_t tiles = (int64_t)cdiv(M, TM) * cdiv(N, TN);
        splits = (int)std::min<int64_t>(std::max<int64_t>(1, (2 * 148 + tiles - 1) / tiles), std::max<int64_t>(1, K / 256));
        MCK(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * (size_t)c_m, p->stream));
    }
    const int64_t kps = ((K + splits - 1) / splits + TK - 1) / TK * TK;
    dim3 grid(cdiv(N, TN), cdiv(M, TM), splits);
    k_gemm<TA, TB><<<grid, 256, 0, p->stream>>>(M, N, K, A, a_m, a_k, B, b_k, b_n, C, c_m, kps);
    MCK(cudaGetLastError());
    return DTB_OK;
}

int ensure_cap(dtb_mlp* p, int64_t B)
{
    if (B <= p->cap) return DTB_OK;
    float** bufs[] = {&p->Z1, &p->H1, &p->Z2, &p->H2, &p->dH2, &p->dZ2, &p->dH1, &p->dZ1};
    for (float** b : bufs) { if (*b) cudaFree(*b); *b = nullptr; }
    if (p->Y) cudaFree(p->Y);
    if (p->dY) cudaFree(p->dY);
    p->Y = p->dY = nullptr;
    p->cap = 0;
    for (float** b : bufs) MCK(cudaMalloc(b, sizeof(float) * (size_t)B * p->H));
    MCK(cudaMalloc(&p->Y, sizeof(float) * (size_t)B));
    MCK(cudaMalloc(&p->dY, sizeof(float) * (size_t)B));
    p->cap = B;
    return DTB_OK;
}

int forward(dtb_mlp* p, const float* x, int64_t B, float* y)
{
    const int in = p->in, H = p->H;
    const __nv_bfloat16* wb = p->wb;
    // Z1 = X W1^T + b1, H1 = GELU(Z1)
    if (int rc = gemm(p, (int)B, H, in, x, in, 1, wb + p->o_W1, 1, in, p->Z1, H, false)) return rc;
    k_bias_act<<<cdiv(B * H, 256), 256, 0, p->stream>>>(B, H, p->Z1, p->w + p->o_b1, p->H1, 1);
    // Z2 = H1 W2^T + b2, H2 = GELU(Z2)
    if (int rc = gemm(p, (int)B, H, H, p->H1, H, 1, wb + p->o_W2, 1, H, p->Z2, H, false)) return rc;
    k_bias_act<<<cdiv(B * H, 256), 256, 0, p->stream>>>(B, H, p->Z2, p->w + p->o_b2, p->H2, 1);
    // y = H2 W3^T + b3
    if (int rc = gemm(p, (int)B, 1, H, p->H2, H, 1, wb + p->o_W3, 1, H, y, 1, false)) return rc;
    k_bias_act<<<cdiv(B, 256), 256, 0, p->stream>>>(B, 1, y, p->w + p->o_b3, y, 0);
    MCK(cudaGetLastError());
    return DTB_OK;
}

// gradients of mean((y - target)^2) into p->g; loss into p->loss
int backward(dtb_mlp* p, const float* x, const float* target, int64_t B)
{
    const int in = p->in, H = p->H;
    const __nv_bfloat16* wb = p->wb;
    MCK(cudaMemsetAsync(p->g, 0, sizeof(float) * (size_t)p->n_params, p->stream));
    MCK(cudaMemsetAsync(p->loss, 0, sizeof(float), p->stream));
    k_mse<<<cdiv(B, 256), 256, 0, p->stream>>>(B, p->Y, target, p->dY, p->loss);
    // layer 3: dW3 = dY^T H2, db3 = sum dY, dH2 = dY W3
    if (int rc = gemm(p, 1, H, B, p->dY, 1, 1, p->H2, H, 1, p->g + p->o_W3, H, true)) return rc;
    k_colsum<<<dim3(1, cdiv(B, 256)), 256, 0, p->stream>>>(B, 1, p->dY, p->g + p->o_b3);
    if (int rc = gemm(p, (int)B, H, 1, p->dY, 1, 1, wb + p->o_W3, H, 1, p->dH2, H, false)) return rc;
    k_gelu_bwd<<<cdiv(B * H, 256), 256, 0, p->stream>>>(B * H, p->dH2, p->Z2, p->dZ2);
    // layer 2: dW2 = dZ2^T H1, db2 = colsum dZ2, dH1 = dZ2 W2
    if (int rc = gemm(p, H, H, B, p->dZ2, 1, H, p->H1, H, 1, p->g + p->o_W2, H, true)) return rc;
    k_colsum<<<dim3(cdiv(H, 32), cdiv(B, 256)), 256, 0, p->stream>>>(B, H, p->dZ2, p->g + p->o_b2);
    if (int rc = gemm(p, (int)B, H, H, p->dZ2, H, 1, wb + p->o_W2, H, 1, p->dH1, H, false)) return rc;
    k_gelu_bwd<<<cdiv(B * H, 256), 256, 0, p->stream>>>(B * H, p->dH1, p->Z1, p->dZ1);
    // layer 1: dW1 = dZ1^T X, db1 = colsum dZ1
    if (int rc = gemm(p, H, in, B, p->dZ1, 1, H, x, in, 1, p->g + p->o_W1, in, true)) return rc;
    k_colsum<<<dim3(cdiv(H, 32), cdiv(B, 256)), 256, 0, p->stream>>>(B, H, p->dZ1, p->g + p->o_b1);
    MCK(cudaGetLastError());
    return DTB_OK;
}

}  // namespace

extern "C" {

int dtb_mlp_create(int in_dim, int hidden, uint64_t seed, int device, dtb_mlp** out)
{
    if (!out || in_dim < 1 || hidden < 1 || in_dim > 4096 || hidden > 4096) return mlp_fail(DTB_ERR_ARG, "bad sizes");
    *out = nullptr;
    int prev = -1;
    cudaGetDevice(&prev);
    MCK(cudaSetDevice(device));
    dtb_mlp* p = new dtb_mlp();
    p->device = device;
    p->in = in_dim;
    p->H = hidden;
    int64_t o = 0;
    p->o_W1 = o; o += (int64_t)hidden * in_dim;
    p->o_b1 = o; o += hidden;
    p->o_W2 = o; o += (int64_t)hidden * hidden;
    p->o_b2 = o; o += hidden;
    p->o_W3 = o; o += hidden;
    p->o_b3 = o; o += 1;
    p->n_params = o;
    // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (seeded, host side)
    std::vector<float> w((size_t)o, 0.0f);
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((st >> 40) & 0xFFFFFF) / 16777216.0f;
    };
    const float a1 = 1.0f / std::sqrt((float)in_dim), a2 = 1.0f / std::sqrt((float)hidden);
    for (int64_t i = 0; i < (int64_t)hidden * in_dim; ++i) w[(size_t)(p->o_W1 + i)] = (2.0f * uni() - 1.0f) * a1;
    for (int64_t i = 0; i < (int64_t)hidden * hidden; ++i) w[(size_t)(p->o_W2 + i)] = (2.0f * uni() - 1.0f) * a2;
    for (int64_t i = 0; i < hidden; ++i) w[(size_t)(p->o_W3 + i)] = (2.0f * uni() - 1.0f) * a2;
    cudaError_t e = cudaMalloc(&p->w, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) e = cudaMalloc(&p->wb, sizeof(__nv_bfloat16) * (size_t)o);
    if (e == cudaSuccess) e = cudaMalloc(&p->g, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) e = cudaMalloc(&p->m, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) e = cudaMalloc(&p->v, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) e = cudaMalloc(&p->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(p->w, w.data(), sizeof(float) * (size_t)o, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(p->m, 0, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) e = cudaMemset(p->v, 0, sizeof(float) * (size_t)o);
    if (e == cudaSuccess) {
        k_to_bf16<<<cdiv(o, 256), 256>>>(o, p->w, p->wb);
        e = cudaDeviceSynchronize();
    }
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) {
        dtb_mlp_destroy(p);
        return mlp_fail(DTB_ERR_NOMEM, "MLP allocation: %s", cudaGetErrorString(e));
    }
    *out = p;
    return DTB_OK;
}

int dtb_mlp_destroy(dtb_mlp* p)
{
    if (!p) return DTB_OK;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    void* bufs[] = {p->w, p->wb, p->g, p->m, p->v, p->loss, p->Z1, p->H1, p->Z2, p->H2, p->Y,
                    p->dY, p->dH2, p->dZ2, p->dH1, p->dZ1};
    for (void* b : bufs) if (b) cudaFree(b);
    if (prev >= 0) cudaSetDevice(prev);
    delete p;
    return DTB_OK;
}

int dtb_mlp_set_stream(dtb_mlp* p, void* stream)
{
    if (!p) return mlp_fail(DTB_ERR_ARG, "null handle");
    p->stream = (cudaStream_t)stream;
    return DTB_OK;
}

int dtb_mlp_n_params(const dtb_mlp* p, int64_t* n)
{
    if (!p || !n) return mlp_fail(DTB_ERR_ARG, "null argument");
    *n = p->n_params;
    return DTB_OK;
}

int dtb_mlp_get_params(dtb_mlp* p, float* dst, int where)
{
    if (!p || !dst) return mlp_fail(DTB_ERR_ARG, "null argument");
    MCK(cudaMemcpyAsync(dst, p->w, sizeof(float) * (size_t)p->n_params,
                        where == DTB_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, p->stream));
    MCK(cudaStreamSynchronize(p->stream));
    return DTB_OK;
}

int dtb_mlp_set_params(dtb_mlp* p, const float* src, int where)
{
    if (!p || !src) return mlp_fail(DTB_ERR_ARG, "null argument");
    MCK(cudaMemcpyAsync(p->w, src, sizeof(float) * (size_t)p->n_params,
                        where == DTB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, p->stream));
    k_to_bf16<<<cdiv(p->n_params, 256), 256, 0, p->stream>>>(p->n_params, p->w, p->wb);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(p->stream));
    return DTB_OK;
}

int dtb_mlp_forward(dtb_mlp* p, const float* x, int64_t B, float* y)
{
    if (!p || !x || !y || B < 1) return mlp_fail(DTB_ERR_ARG, "bad argument");
    if (int rc = ensure_cap(p, B)) return rc;
    return forward(p, x, B, y);
}

int dtb_mlp_gradient(dtb_mlp* p, const float* x, const float* target, int64_t B, float* grad, float* loss)
{
    if (!p || !x || !target || B < 1) return mlp_fail(DTB_ERR_ARG, "bad argument");
    if (int rc = ensure_cap(p, B)) return rc;
    if (int rc = forward(p, x, B, p->Y)) return rc;
    if (int rc = backward(p, x, target, B)) return rc;
    if (grad) MCK(cudaMemcpyAsync(grad, p->g, sizeof(float) * (size_t)p->n_params, cudaMemcpyDeviceToDevice, p->stream));
    if (loss) MCK(cudaMemcpyAsync(loss, p->loss, sizeof(float), cudaMemcpyDeviceToDevice, p->stream));
    return DTB_OK;
}

int dtb_mlp_train_step(dtb_mlp* p, const float* x, const float* target, int64_t B, float lr, float* loss)
{
    if (int rc = dtb_mlp_gradient(p, x, target, B, nullptr, loss)) return rc;
    p->t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)p->t), c2 = 1.0f - std::pow(b2, (float)p->t);
    k_adam<<<cdiv(p->n_params, 256), 256, 0, p->stream>>>(p->n_params, p->w, p->g, p->m, p->v, p->wb, lr, b1, b2,
                                                          1e-8f, c1, c2);
    MCK(cudaGetLastError());
    return DTB_OK;
}

int dtb_mlp_last_error(char* buf, size_t len)
{
    if (!buf || !len) return DTB_ERR_ARG;
    std::snprintf(buf, len, "%s", g_mlp_err.c_str());
    return DTB_OK;
}

}  // extern "C"
