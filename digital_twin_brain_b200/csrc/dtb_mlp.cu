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
#include <type_traits>
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

// ------------------------------------------------------------ tensor-core GEMM (tcgen05)
// C[M][N] = A[M][K] * B[K][N] on the 5th-generation tensor cores: tcgen05.mma of
// kind::f16 with BF16 operands from shared memory and the FP32 accumulator in
// tensor memory (TMEM), issued by one thread; the accumulator is read back with
// tcgen05.ld by the four warps (warp w owns TMEM lanes 32w..32w+31 = tile rows).
//
// Operand precision: an operand already in BF16 (the weights) enters as one
// term; an FP32 operand (activations, gradients) is split into three BF16 terms
// hi + mid + lo (each the rounding of what the previous ones leave), and the
// products of term pairs (i, j) with i + j < 3 are accumulated: BF16 x BF16
// products are exact in FP32, so the result keeps FP32 accuracy (to a few units
// of 2^-24 relative per product) while every multiply runs on the tensor cores.
//
// Tile: 128 rows (the M = 128 instruction shape, cta_group::1) x n_tile columns
// (16..128, a multiple of 16), K in chunks of 32 (two K = 16 instructions).
// Shared-memory operand layout: K-major, no swizzle, 8x16-byte core matrices,
// core (r, c) of a 128x32 tile at (r * 4 + c) * 128 bytes: leading (K) byte
// offset 128, stride (8-row) byte offset 512.  gridDim.z splits K; partial tiles
// are then added to C atomically (C pre-zeroed).
constexpr int kMmaM = 128;
constexpr int kMmaKc = 32;                        // K per staged chunk
constexpr int kMmaThreads = 128;
constexpr int kMmaTile = kMmaM * kMmaKc * 2;      // bytes of one BF16 term tile (8 KB)
constexpr int kMmaTmemCols = 128;

struct MmaArgs {
    int M, N;
    int64_t K;
    const void* A; int64_t a_m, a_k; int a_bf16;  // A(m, k) = A[m * a_m + k * a_k]
    const void* B; int64_t b_k, b_n; int b_bf16;  // B(k, n) = B[k * b_k + n * b_n]
    float* C; int64_t c_m;                        // C(m, n) = C[m * c_m + n]
    int64_t k_per_split;
    const float* bias;                            // epilogue (nullable): Z = acc + bias[n]
    float* H;                                     // (nullable) H = GELU(Z), same layout as C
    int n_tile;
    unsigned* err;                                // set when a completion wait gave up
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05): start >> 4, leading byte offset >> 4 at
// bit 16, stride byte offset >> 4 at bit 32, descriptor version 1 at bit 46, no swizzle.
__device__ __forceinline__ uint64_t mma_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bit 4), A and B BF16 (bits 7, 10),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__device__ __forceinline__ uint32_t mma_idesc(int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kMmaM >> 4) << 24);
}

__device__ __forceinline__ bool mma_wait(uint32_t mbar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

template <typename T>
__device__ __forceinline__ float ld_elem(const T* p, int64_t i) { return load_f(p + i); }

// Split x into nt BF16 terms (nt = 1: plain rounding).
__device__ __forceinline__ void split_bf16(float x, int nt, __nv_bfloat16* t)
{
    float r = x;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (i < nt) {
            t[i] = __float2bfloat16_rn(r);
            r = r - __bfloat162float(t[i]);
        }
    }
}

// One 128 x 32 operand tile (rows = M or N of the instruction, K-major) into nt term tiles:
// thread t stages row t.  get(row, k) returns the FP32 value (0 outside the matrix).
template <typename Get>
__device__ __forceinline__ void stage_rows(unsigned char* tiles, int nt, Get get)
{
    const int r = threadIdx.x;
#pragma unroll
    for (int c = 0; c < kMmaKc / 8; ++c) {          // four core matrices along K
        __align__(16) __nv_bfloat16 t[3][8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            __nv_bfloat16 s3[3];
            split_bf16(get(r, c * 8 + e), nt, s3);
#pragma unroll
            for (int i = 0; i < 3; ++i) t[i][e] = s3[i];
        }
        const int off = ((r >> 3) * (kMmaKc / 8) + c) * 128 + (r & 7) * 16;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nt) *reinterpret_cast<uint4*>(tiles + i * kMmaTile + off) = *reinterpret_cast<const uint4*>(t[i]);
    }
}

// Eight consecutive elements of a row as FP32 (16-byte aligned source).
__device__ __forceinline__ void load8(const float* p, float* x)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(p)), b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}
__device__ __forceinline__ void load8(const __nv_bfloat16* p, float* x)
{
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    const __nv_bfloat16* h = reinterpret_cast<const __nv_bfloat16*>(&a);
#pragma unroll
    for (int e = 0; e < 8; ++e) x[e] = __bfloat162float(h[e]);
}

// stage_rows for a K-contiguous operand whose chunk lies inside the matrix: thread t loads
// row t's 32 elements with 16-byte loads (row = nullptr: a row past the matrix, zeros).
template <typename T>
__device__ __forceinline__ void stage_rows_contig(unsigned char* tiles, int nt, const T* row)
{
    const int r = threadIdx.x;
    float x[kMmaKc];
#pragma unroll
    for (int c = 0; c < kMmaKc / 8; ++c) {
        if (row) load8(row + c * 8, x + c * 8);
        else {
#pragma unroll
            for (int e = 0; e < 8; ++e) x[c * 8 + e] = 0.0f;
        }
    }
#pragma unroll
    for (int c = 0; c < kMmaKc / 8; ++c) {
        __align__(16) __nv_bfloat16 t[3][8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            __nv_bfloat16 s3[3];
            split_bf16(x[c * 8 + e], nt, s3);
#pragma unroll
            for (int i = 0; i < 3; ++i) t[i][e] = s3[i];
        }
        const int off = ((r >> 3) * (kMmaKc / 8) + c) * 128 + (r & 7) * 16;
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (i < nt) *reinterpret_cast<uint4*>(tiles + i * kMmaTile + off) = *reinterpret_cast<const uint4*>(t[i]);
    }
}

template <typename T>
__device__ __forceinline__ bool aligned16(const T* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename TA, typename TB>
__global__ void __launch_bounds__(kMmaThreads) k_mma_gemm(MmaArgs g)
{
    extern __shared__ __align__(1024) unsigned char mma_smem[];   // A term tiles, then B term tiles
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kMmaM, n0 = blockIdx.x * g.n_tile;
    const int64_t k_begin = (int64_t)blockIdx.z * g.k_per_split;
    const int64_t k_end = k_begin + g.k_per_split < g.K ? k_begin + g.k_per_split : g.K;
    const int nA = g.a_bf16 ? 1 : 3, nB = g.b_bf16 ? 1 : 3;
    unsigned char* sA = mma_smem;
    unsigned char* sB = mma_smem + nA * kMmaTile;
    const TA* A = static_cast<const TA*>(g.A);
    const TB* B = static_cast<const TB*>(g.B);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&tmem_base)), "r"((uint32_t)kMmaTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&mbar)) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    const uint32_t idesc = mma_idesc(g.n_tile);
    const uint32_t mb = smem_addr(&mbar);

    int chunks = 0;
    bool ok = true;
    for (int64_t k0 = k_begin; k0 < k_end; k0 += kMmaKc, ++chunks) {
        if (chunks > 0 && ok) ok = mma_wait(mb, (uint32_t)((chunks - 1) & 1), 1u << 22);   // tiles free again
        // K-contiguous rows with a whole chunk in range: 16-byte loads; otherwise element by element
        const bool full = k0 + kMmaKc <= k_end;
        if (full && g.a_k == 1 && aligned16(A) && (g.a_m * (int64_t)sizeof(TA)) % 16 == 0) {
            const int64_t m = m0 + threadIdx.x;
            stage_rows_contig(sA, nA, m < g.M ? A + m * g.a_m + k0 : static_cast<const TA*>(nullptr));
        } else {
            stage_rows(sA, nA, [&](int r, int k) -> float {
                const int64_t m = m0 + r, kk = k0 + k;
                return (m < g.M && kk < k_end) ? ld_elem(A, m * g.a_m + kk * g.a_k) : 0.0f;
            });
        }
        if (full && g.b_k == 1 && aligned16(B) && (g.b_n * (int64_t)sizeof(TB)) % 16 == 0) {
            const int64_t n = n0 + threadIdx.x;
            stage_rows_contig(sB, nB, (threadIdx.x < g.n_tile && n < g.N) ? B + n * g.b_n + k0
                                                                          : static_cast<const TB*>(nullptr));
        } else {
            stage_rows(sB, nB, [&](int r, int k) -> float {
                const int64_t n = n0 + r, kk = k0 + k;
                return (r < g.n_tile && n < g.N && kk < k_end) ? ld_elem(B, kk * g.b_k + n * g.b_n) : 0.0f;
            });
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic stores -> tensor-core reads
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            int issued = 0;
#pragma unroll
            for (int s = 0; s < kMmaKc / 16; ++s)
                for (int i = 0; i < nA; ++i)
                    for (int j = 0; j < nB; ++j) {
                        if (i + j >= 3) continue;
                        const uint64_t ad = mma_desc(smem_addr(sA + i * kMmaTile + s * 256));
                        const uint64_t bd = mma_desc(smem_addr(sB + j * kMmaTile + s * 256));
                        const uint32_t acc = (chunks > 0 || issued > 0) ? 1u : 0u;
                        asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                     :: "r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc) : "memory");
                        ++issued;
                    }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(mb) : "memory");
        }
    }
    if (chunks > 0) {
        if (ok) ok = mma_wait(mb, (uint32_t)((chunks - 1) & 1), 1u << 24);
        if (!ok) {   // give up: flag it, and make sure the MMAs are done before TMEM is freed
            if (threadIdx.x == 0 && g.err) atomicOr(g.err, 1u);
            mma_wait(mb, (uint32_t)((chunks - 1) & 1), 1u << 26);
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // epilogue: warp w reads rows 32w + lane, 16 columns at a time
        const int64_t m = m0 + warp * 32 + lane;
        for (int c = 0; c < g.n_tile; c += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(taddr) : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (ok && m < g.M) {
                // four columns per access where the row allows it (16-byte aligned, in range)
                const bool vec = (g.c_m & 3) == 0 && (reinterpret_cast<uintptr_t>(g.C) & 15) == 0 &&
                                 (reinterpret_cast<uintptr_t>(g.bias) & 15) == 0 &&
                                 (reinterpret_cast<uintptr_t>(g.H) & 15) == 0;
#pragma unroll
                for (int e = 0; e < 16; e += 4) {
                    const int64_t n = n0 + c + e;
                    if (vec && c + e + 4 <= g.n_tile && n + 4 <= g.N) {
                        float4 z = make_float4(__uint_as_float(v[e]), __uint_as_float(v[e + 1]),
                                               __uint_as_float(v[e + 2]), __uint_as_float(v[e + 3]));
                        float4* cp = reinterpret_cast<float4*>(g.C + m * g.c_m + n);
                        if (gridDim.z > 1) { atomicAdd(cp, z); continue; }
                        if (g.bias) {
                            const float4 b = *reinterpret_cast<const float4*>(g.bias + n);
                            z.x += b.x; z.y += b.y; z.z += b.z; z.w += b.w;
                        }
                        *cp = z;
                        if (g.H)
                            *reinterpret_cast<float4*>(g.H + m * g.c_m + n) =
                                make_float4(gelu(z.x), gelu(z.y), gelu(z.z), gelu(z.w));
                        continue;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int64_t nq = n + q;
                        if (c + e + q >= g.n_tile || nq >= g.N) continue;
                        float z = __uint_as_float(v[e + q]);
                        if (gridDim.z > 1) { atomicAdd(g.C + m * g.c_m + nq, z); continue; }
                        if (g.bias) z += g.bias[nq];
                        g.C[m * g.c_m + nq] = z;
                        if (g.H) g.H[m * g.c_m + nq] = gelu(z);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"((uint32_t)kMmaTmemCols)
                     : "memory");
    }
}
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
    unsigned* err = nullptr;       // device flag: a tensor-core GEMM gave up waiting for its MMAs
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

// The hidden layers' GEMMs on the tensor cores (k_mma_gemm): C = A B (+ bias, GELU when H).
template <typename TA, typename TB>
int mma_gemm(dtb_mlp* p, int M, int N, int64_t K, const TA* A, int64_t a_m, int64_t a_k, const TB* B, int64_t b_k,
             int64_t b_n, float* C, int64_t c_m, bool split, const float* bias = nullptr, float* H = nullptr)
{
    MmaArgs g;
    g.M = M; g.N = N; g.K = K;
    g.A = A; g.a_m = a_m; g.a_k = a_k; g.a_bf16 = std::is_same<TA, __nv_bfloat16>::value ? 1 : 0;
    g.B = B; g.b_k = b_k; g.b_n = b_n; g.b_bf16 = std::is_same<TB, __nv_bfloat16>::value ? 1 : 0;
    g.C = C; g.c_m = c_m;
    g.bias = bias; g.H = H;
    g.err = p->err;
    // 128-column tiles, or 64 when that leaves fewer than two CTAs per SM (more CTAs in flight)
    g.n_tile = N >= 128 ? 128 : ((N + 15) / 16) * 16;
    if (g.n_tile == 128 && (int64_t)cdiv(N, 128) * cdiv(M, kMmaM) < 2 * 148) g.n_tile = 64;
    const int64_t tiles = (int64_t)cdiv(N, g.n_tile) * cdiv(M, kMmaM);
    int64_t splits = 1;
    if (split) {
        splits = std::min<int64_t>(std::max<int64_t>(1, (2 * 148 + tiles - 1) / tiles), std::max<int64_t>(1, K / 256));
        MCK(cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * (size_t)c_m, p->stream));
    }
    g.k_per_split = ((K + splits - 1) / splits + kMmaKc - 1) / kMmaKc * kMmaKc;
    splits = (K + g.k_per_split - 1) / g.k_per_split;      // no empty split
    dim3 grid(cdiv(N, g.n_tile), cdiv(M, kMmaM), (unsigned)splits);
    const int smem = ((g.a_bf16 ? 1 : 3) + (g.b_bf16 ? 1 : 3)) * kMmaTile;
    static bool attr = false;
    if (!attr) {
        MCK(cudaFuncSetAttribute(k_mma_gemm<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 6 * kMmaTile));
        attr = true;
    }
    k_mma_gemm<TA, TB><<<grid, kMmaThreads, smem, p->stream>>>(g);
    MCK(cudaGetLastError());
    return DTB_OK;
}

int check_err(dtb_mlp* p)
{
    unsigned e = 0;
    MCK(cudaMemcpy(&e, p->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(p->err, 0, sizeof(unsigned));
        return mlp_fail(DTB_ERR_CUDA, "a tensor-core GEMM did not complete in time");
    }
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
    // Z1 = X W1^T + b1, H1 = GELU(Z1) (tensor cores, bias and GELU in the epilogue)
    if (int rc = mma_gemm(p, (int)B, H, in, x, in, 1, wb + p->o_W1, 1, in, p->Z1, H, false, p->w + p->o_b1, p->H1))
        return rc;
    // Z2 = H1 W2^T + b2, H2 = GELU(Z2)
    if (int rc = mma_gemm(p, (int)B, H, H, p->H1, H, 1, wb + p->o_W2, 1, H, p->Z2, H, false, p->w + p->o_b2, p->H2))
        return rc;
    // y = H2 W3^T + b3 (one output column: a dot product per row)
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
    // layer 2: dW2 = dZ2^T H1, db2 = colsum dZ2, dH1 = dZ2 W2 (tensor cores)
    if (int rc = mma_gemm(p, H, H, B, p->dZ2, 1, H, p->H1, H, 1, p->g + p->o_W2, H, true)) return rc;
    k_colsum<<<dim3(cdiv(H, 32), cdiv(B, 256)), 256, 0, p->stream>>>(B, H, p->dZ2, p->g + p->o_b2);
    if (int rc = mma_gemm(p, (int)B, H, H, p->dZ2, H, 1, wb + p->o_W2, H, 1, p->dH1, H, false)) return rc;
    k_gelu_bwd<<<cdiv(B * H, 256), 256, 0, p->stream>>>(B * H, p->dH1, p->Z1, p->dZ1);
    // layer 1: dW1 = dZ1^T X, db1 = colsum dZ1 (tensor cores)
    if (int rc = mma_gemm(p, H, in, B, p->dZ1, 1, H, x, in, 1, p->g + p->o_W1, in, true)) return rc;
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
    if (e == cudaSuccess) e = cudaMalloc(&p->err, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(p->err, 0, sizeof(unsigned));
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
    void* bufs[] = {p->w, p->wb, p->g, p->m, p->v, p->loss, p->err, p->Z1, p->H1, p->Z2, p->H2, p->Y,
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
    return check_err(p);
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
