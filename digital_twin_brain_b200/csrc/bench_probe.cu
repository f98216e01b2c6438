// Measurement helper of bench.py, built as its own library (libdtb_bench_probe.so)
// and not part of libdtb.so: the rate at which this GPU performs float2 atomic
// additions (the push scatter's per-synapse operation) into J-sized targets.
// Nothing in the simulator calls it.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

namespace {

// n_ops target indices in [0, n): each drawn inside a window of `window` targets
// that moves with the operation index (a region's intra-region synapses), or
// anywhere when window >= n.
__global__ void k_probe_fill(uint32_t* idx, int64_t n_ops, uint32_t n, uint32_t window, uint32_t seed)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_ops) return;
    uint32_t x = (uint32_t)i * 2654435761u ^ seed;
    x ^= x >> 13; x *= 0x5bd1e995u; x ^= x >> 15;
    const uint32_t w = window < n ? window : n;
    const uint32_t start = (uint32_t)(((uint64_t)(i / 100) * 100u) % n);
    idx[i] = (uint32_t)(((uint64_t)start + (x % w)) % n);
}

__global__ void k_probe_red(const uint32_t* __restrict__ idx, int64_t n_ops, float2* J)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_ops; i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(J + __ldcs(idx + i), make_float2(1.0f, 0.5f));
}

}  // namespace

// ms_out = milliseconds for n_ops float2 atomic additions into n_targets targets
// (mean of 10 launches after 2 warm-up launches).  Returns 0, or the CUDA error code.
extern "C" int dtb_bench_atomic_rate(int device, int64_t n_targets, int64_t n_ops, int64_t window, float* ms_out)
{
    if (!ms_out || n_targets < 1 || n_targets > 0x7fffffffLL || n_ops < 1 || window < 1) return -1;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    uint32_t* idx = nullptr;
    float2* J = nullptr;
    cudaEvent_t a = nullptr, z = nullptr;
    cudaError_t e = cudaMalloc(&idx, sizeof(uint32_t) * (size_t)n_ops);
    if (e == cudaSuccess) e = cudaMalloc(&J, sizeof(float2) * (size_t)n_targets);
    if (e == cudaSuccess) e = cudaMemset(J, 0, sizeof(float2) * (size_t)n_targets);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&z);
    if (e == cudaSuccess) {
        const unsigned fill_grid = (unsigned)((n_ops + 255) / 256);
        k_probe_fill<<<fill_grid, 256>>>(idx, n_ops, (uint32_t)n_targets,
                                         (uint32_t)std::min<int64_t>(window, n_targets), 12345u);
        for (int w = 0; w < 2; ++w) k_probe_red<<<sms * 16, 256>>>(idx, n_ops, J);
        cudaEventRecord(a);
        for (int r = 0; r < 10; ++r) k_probe_red<<<sms * 16, 256>>>(idx, n_ops, J);
        cudaEventRecord(z);
        e = cudaEventSynchronize(z);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, z);
        *ms_out = ms / 10.0f;
    }
    if (a) cudaEventDestroy(a);
    if (z) cudaEventDestroy(z);
    cudaFree(idx);
    cudaFree(J);
    cudaSetDevice(prev);
    return e == cudaSuccess ? 0 : (int)e;
}
