// dtb_step_preallocated: one time step of a caller-owned network, with all
// scratch memory in one static device array of this file (no allocation).
//
// Callers that cannot allocate device memory (a host framework that owns a
// fixed pool or budget, a real-time loop in which cudaMalloc / cudaFree are
// forbidden) keep every network array themselves; the step's scratch (spike
// bitmask, subblock accumulators, control block) lives in g_scratch below,
// held by every GPU that loads libdtb.so until the process exits.  Calls
// share it: each call re-initialises the parts it reads, and calls whose GPU
// work overlaps race on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "dtb.h"

// This file carries its own copy of the step kernels (same source), in a
// namespace of its own so that it links beside dtb_api.cu's copy.
#define dtb dtb_prealloc_impl
#include "dtb_kernels.cuh"
#undef dtb

using namespace dtb_prealloc_impl;

static_assert(sizeof(dtb_param_class) == sizeof(ParamClass), "dtb_param_class must match the kernels' class layout");

namespace {

constexpr int64_t kMaxNeurons = DTB_PREALLOC_MAX_NEURONS;
constexpr int kMaxSub = DTB_PREALLOC_MAX_SUBBLOCKS;
constexpr int64_t kMaxWords = ((kMaxNeurons + 127) / 128) * 4;

// Byte offsets inside the scratch array (each 256-byte aligned).
constexpr size_t kOffCtl = 0;
constexpr size_t kOffSpk = 256;
constexpr size_t kOffNact = kOffSpk + sizeof(uint32_t) * kMaxSub;
constexpr size_t kOffVsum = kOffNact + sizeof(uint32_t) * kMaxSub;
constexpr size_t kOffUnmapped = kOffVsum + sizeof(double) * kMaxSub;
constexpr size_t kOffStats = kOffUnmapped + 256;                       // spare stats rows
constexpr size_t kOffBits = kOffStats + 2 * sizeof(float) * kMaxSub + 256;
constexpr size_t kOffABits = kOffBits + sizeof(uint32_t) * kMaxWords;
constexpr size_t kScratchBytes = kOffABits + sizeof(uint32_t) * kMaxWords;   // ~1.04 MB

}  // namespace

// The scratch: fixed size, one per device, for the whole life of the process.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

namespace {

// Status only: the entry point reports its errors by dtb_status code.
int err(int code, const char*, ...) { return code; }

// Device address of g_scratch per device, looked up once with the device current.
std::mutex g_mu;
unsigned char* g_addr[64] = {nullptr};

int scratch_address(int device, unsigned char** out)
{
    if (device < 0 || device >= 64) return err(DTB_ERR_ARG, "device %d out of range", device);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaError_t e = cudaSetDevice(device);
        void* p = nullptr;
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&p, g_scratch);
        if (prev >= 0 && prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess) return err(DTB_ERR_CUDA, "cudaGetSymbolAddress(g_scratch): %s", cudaGetErrorString(e));
        g_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[device];
    return DTB_OK;
}

// Re-initialises the shared scratch for one step: control block and the
// subblock accumulators (the bitmask is rewritten in full by the update).
__global__ void k_prealloc_setup(Ctl* ctl, uint32_t* spk, uint32_t* nact, double* vsum, uint32_t* unmapped,
                                 int n_sub, unsigned long long step, float t, float noise_rate, int isolated)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        ctl->steps_done = step;
        ctl->run_base = step;
        ctl->noise_rate = noise_rate;
        ctl->isolated = isolated;
        ctl->t = t;
        ctl->done = 0u;
        ctl->stats_cap = 1u;
        ctl->use_isyn_override = 0u;
        ctl->err = 0u;
        ctl->events = 0ull;
        *unmapped = 0u;
    }
    if (i < n_sub) { spk[i] = 0u; nact[i] = 0u; vsum[i] = 0.0; }
}

}  // namespace

extern "C" {

int dtb_step_preallocated(const dtb_prealloc_net* net, float t, uint64_t step, float noise_rate, int isolated,
                          float* sum_out, float* mean_out, void* stream)
{
    if (!net) return err(DTB_ERR_ARG, "null network");
    const int64_t N = net->n_neurons;
    if (N <= 0 || N > kMaxNeurons)
        return err(DTB_ERR_LIMIT, "n_neurons %lld outside [1, %lld] (the fixed scratch array holds a bitmask of "
                   "DTB_PREALLOC_MAX_NEURONS neurons)", (long long)N, (long long)kMaxNeurons);
    if (net->n_subblocks < 0 || net->n_subblocks > kMaxSub)
        return err(DTB_ERR_LIMIT, "n_subblocks %d outside [0, %d]", net->n_subblocks, kMaxSub);
    if (!net->V || !net->J || !net->t_last || !net->cls || !net->classes || !net->rowptr || !net->index ||
        !net->weight || (net->n_subblocks > 0 && !net->sub_count))
        return err(DTB_ERR_ARG, "null array in the network description");
    if (!(net->dt > 0.0f)) return err(DTB_ERR_ARG, "dt must be positive");
    unsigned char* base = nullptr;
    const int rc = scratch_address(net->device, &base);
    if (rc != DTB_OK) return rc;

    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != net->device) cudaSetDevice(net->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    DevState s;
    std::memset(&s, 0, sizeof(s));
    s.N = N;
    s.n_words = ((N + 127) / 128) * 4;
    s.V = net->V;
    s.J2 = reinterpret_cast<float2*>(net->J);   // caller layout [N][4]: pairs interleaved per neuron
    s.j_ps = 1;
    s.j_es = 2;
    s.tlast = net->t_last;
    s.isyn_override = nullptr;
    s.cls = net->cls;
    s.pc = reinterpret_cast<const ParamClass*>(net->classes);
    uint32_t* bits = reinterpret_cast<uint32_t*>(base + kOffBits);
    s.bits[0] = bits;           // one step: the update writes and the gather reads one bitmask
    s.bits[1] = bits;
    s.abits = reinterpret_cast<uint32_t*>(base + kOffABits);
    s.prow = net->rowptr;
    s.pcol = net->index;
    s.pw = reinterpret_cast<const float2*>(net->weight);
    s.n_sub = net->n_subblocks;
    s.sub_count = net->sub_count;
    s.sub_spk = reinterpret_cast<uint32_t*>(base + kOffSpk);
    s.sub_nact = reinterpret_cast<uint32_t*>(base + kOffNact);
    s.sub_vsum = reinterpret_cast<double*>(base + kOffVsum);
    s.unmapped_nact = reinterpret_cast<uint32_t*>(base + kOffUnmapped);
    s.ctl = reinterpret_cast<Ctl*>(base + kOffCtl);
    s.seed = net->seed;
    s.stream_id = net->stream_id;
    s.dt = net->dt;
    s.bold.n_regions = 0;
    float* spare = reinterpret_cast<float*>(base + kOffStats);
    s.st_spk = sum_out ? sum_out : spare;
    s.st_mean = mean_out ? mean_out : spare + kMaxSub;
    s.st_nact = reinterpret_cast<uint32_t*>(base + kOffUnmapped) + 1;

    const int setup_threads = 256;
    const unsigned setup_grid = (unsigned)((std::max(1, net->n_subblocks) + setup_threads - 1) / setup_threads);
    k_prealloc_setup<<<setup_grid, setup_threads, 0, st>>>(s.ctl, s.sub_spk, s.sub_nact, s.sub_vsum,
                                                           s.unmapped_nact, net->n_subblocks,
                                                           (unsigned long long)step, t, noise_rate, isolated ? 1 : 0);
    // one tile of 128 neurons per warp (the kernels also take longer runs of tiles)
    const unsigned grid = (unsigned)((N + kWarpNeurons * (kStepThreads / 32) - 1) / (kWarpNeurons * (kStepThreads / 32)));
    k_step<false, true, false><<<grid, kStepThreads, 0, st>>>(s, 1);   // update (models/block.py:133-142)
    k_step<true, false, false><<<grid, kStepThreads, 0, st>>>(s, 1);   // pull gather, bit-identical order
    const cudaError_t e = cudaGetLastError();
    if (prev >= 0 && prev != net->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return err(DTB_ERR_CUDA, "launch failed: %s", cudaGetErrorString(e));
    return DTB_OK;
}

}  // extern "C"
