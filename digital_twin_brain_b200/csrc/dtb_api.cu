// C ABI of libdtb (include/dtb.h): host-side construction of the network
// (parameter classes, pull / push CSR), memory plan, step scheduling (push or
// pull per chunk of steps, CUDA graphs), state access and BOLD.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "dtb.h"
#include "dtb_io.h"
#include "dtb_kernels.cuh"

using namespace dtb;

// ------------------------------------------------------------ errors
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(DTB_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                        __LINE__);                                                                    \
    } while (0)

#define RET(expr)                      \
    do {                               \
        int r_ = (expr);               \
        if (r_ != DTB_OK) return r_;   \
    } while (0)

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

using Row26 = std::array<uint32_t, 26>;
struct RowHash {
    size_t operator()(const Row26& r) const
    {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t v : r) { h ^= v; h *= 1099511628211ull; }
        return (size_t)h;
    }
};

inline uint32_t fbits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Property row (+ decay) -> class parameters (models/block.py:156-169 split).
ParamClass make_class(const float* prop, const float* decay, float dt)
{
    ParamClass p;
    std::memset(&p, 0, sizeof(p));
    p.g = make_float4(prop[10], prop[11], prop[12], prop[13]);
    p.Vu = make_float4(prop[14], prop[15], prop[16], prop[17]);
    p.decay = make_float4(decay[0], decay[1], decay[2], decay[3]);
    p.gL = prop[6];
    p.VL = prop[7];
    volatile float rc = 1.0f / prop[4];  // torch: C.reciprocal() * dt
    p.rCdt = rc * dt;
    p.Vth = prop[8];
    p.Vreset = prop[9];
    p.Tref = prop[5];
    p.Iext = prop[2];
    p.noise = prop[0];
    const float s = prop[3];
    p.sub = (s >= 0.0f && s < 2147483647.0f && std::floor(s) == s) ? (int32_t)s : -1;
    p.C = prop[4];
    p.member = -1;
    return p;
}

// exp(-dt/tau) evaluated as tau.reciprocal() * (-dt) then exp (block.py:71).
void default_decay(const float* prop, float dt, float* out)
{
    for (int c = 0; c < 4; ++c) {
        volatile float r = 1.0f / prop[18 + c];
        volatile float x = r * (-dt);
        out[c] = std::exp(x);
    }
}

}  // namespace

// ------------------------------------------------------------ handle
struct dtb_block {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int64_t N = 0, S = 0;
    int n_sub = 0, n_classes = 0;
    int pc_cap = 0, sub_cap = 0;
    int n_sm = 148;
    ParamClass* d_pc = nullptr;
    uint32_t* d_sub_count = nullptr;
    float dt = 0.1f;
    uint64_t seed = 0;
    uint32_t stream_id = 0;
    DevState ds{};
    std::vector<void*> allocs;
    std::vector<size_t> alloc_bytes;
    int64_t dev_bytes = 0;
    // host mirrors
    std::vector<ParamClass> classes;
    std::vector<std::array<float, 22>> class_prop_base;  // creation-time rows (scale_property base)
    std::vector<std::array<float, 22>> class_prop;       // current rows
    std::vector<std::array<float, 4>> class_decay;
    std::vector<uint32_t> sub_count;
    uint64_t steps = 0;          // host mirror of ctl->steps_done
    uint32_t stats_cap = 0;
    bool has_pull = false, has_push = false;
    int64_t max_out = 0, max_in = 0;
    // scratch
    uint32_t* d_forced[2] = {nullptr, nullptr};
    uint8_t* d_u8 = nullptr;      // [N] upload staging for forced sets
    float* d_export = nullptr;    // [4N]
    float* d_iui_override = nullptr;
    bool override_pending = false;
    bool override_live = false;   // the device's I_syn override flag may be set: the next update runs the general form
    unsigned* d_err = nullptr;
    // pinned host staging
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    RunParams* h_run = nullptr;   // pinned
    // auto mode
    int64_t launches = 0;
    uint64_t samples_from = 0;    // step at which sampling started
    int64_t samples_written = 0;
    double last_frac = -1.0;
    double pull_threshold = 0.05;
    int chunk = 32;
    int scatter_wpw = 32;         // bitmask words per warp in the push scatter
    int scatter_variant = 0;      // 0: registers unbounded, 1: budgeted for 6 resident CTAs per SM
    int step_variant = 3;         // 0: 2 resident CTAs/SM register budget, 1: 3; 2..4: staged, 2..4 CTAs/SM
    // ordered push (bit-exact pull through per-neuron slots)
    bool has_qpos = false;
    int pull_method = 0;          // 0: auto, 1: row gather, 2: ordered push (slots), 3: (masks), 4: streamed gather
    double slot_threshold = 0.1;
    // binned push (DTB_TUNE_PUSH_METHOD)
    int push_method = 1;          // 0: binned when its bins fit, 1: float2 atomics into J, 2: binned
    int bin_shift_req = 0;        // 0: chosen from N
    int bin_cap_per_neuron = 8;   // bin entries per neuron of a bin
    int bin_words = 256;          // bitmask words per scatter round
    int bin_scatter_per_sm = 0;   // resident scatter CTAs per SM (from the occupancy calculator)
    bool bins_pending = false;    // the bins hold events not yet folded into J
    bool bins_failed = false;     // the bins could not be allocated (auto pushes with atomics)
    // graphs: one chunk graph per propagation method (push, pull rows, pull slots, ..., binned push)
    cudaGraphExec_t graph[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    int graph_len[7] = {0, 0, 0, 0, 0, 0, 0};
    bool use_graphs = true;
    // attached BOLD
    int bold_R = 0;
    // gamma-distributed g_ui (per-neuron factors; ds.gnrn points here while active)
    float4* d_gnrn = nullptr;
    uint32_t gamma_calls = 0;
};

struct dtb_bold {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t R = 0;
    int dtype = 0;
    double eps, ts, tf, t0, alpha, E0, V0, dt;
    void* s = nullptr; void* q = nullptr; void* v = nullptr; void* f = nullptr;
    void* tmp_u = nullptr; void* tmp_o = nullptr;  // device staging for host pointers
    void* tmp_w = nullptr; size_t tmp_w_bytes = 0;
};

template <typename T>
static int dalloc(dtb_block* b, T** p, size_t count)
{
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(DTB_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s (held %lld bytes)", bytes,
                    cudaGetErrorString(e), (long long)b->dev_bytes);
    }
    b->allocs.push_back(q);
    b->alloc_bytes.push_back(bytes);
    b->dev_bytes += (int64_t)bytes;
    *p = reinterpret_cast<T*>(q);
    return DTB_OK;
}

// Frees one allocation of the handle (after its stream is idle).
template <typename T>
static void dfree(dtb_block* b, T*& p)
{
    if (!p) return;
    void* q = const_cast<void*>(reinterpret_cast<const void*>(p));
    for (size_t i = 0; i < b->allocs.size(); ++i) {
        if (b->allocs[i] != q) continue;
        cudaFree(q);
        b->dev_bytes -= (int64_t)b->alloc_bytes[i];
        b->allocs[i] = b->allocs.back(); b->allocs.pop_back();
        b->alloc_bytes[i] = b->alloc_bytes.back(); b->alloc_bytes.pop_back();
        break;
    }
    p = nullptr;
}

static int ensure_pinned(dtb_block* b, size_t bytes)
{
    if (b->pinned_bytes >= bytes) return DTB_OK;
    if (b->pinned) cudaFreeHost(b->pinned);
    b->pinned = nullptr;
    b->pinned_bytes = 0;
    CK(cudaMallocHost(&b->pinned, bytes));
    b->pinned_bytes = bytes;
    return DTB_OK;
}

static inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// ctl->events <- the sum of the per-warp event counters (before the host reads it).
static int sum_events(dtb_block* b)
{
    k_sum_events<<<1, kEvParts, 0, b->stream>>>(b->ds.ev_part, b->ds.ctl);
    CK(cudaGetLastError());
    return DTB_OK;
}

static int copy_out(dtb_block* b, void* dst, const void* dsrc, size_t bytes, int where)
{
    if (bytes == 0) return DTB_OK;
    if (where == DTB_DEVICE) {
        CK(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToDevice, b->stream));
    } else {
        CK(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToHost, b->stream));
        CK(cudaStreamSynchronize(b->stream));
    }
    return DTB_OK;
}

// ------------------------------------------------------------ classes
// Deduplicates property rows (+ decay) into the class table.
static int build_classes(dtb_block* b, int64_t N, const float* property, const float* decay,
                         std::vector<uint32_t>& cls)
{
    std::unordered_map<Row26, uint32_t, RowHash> map;
    map.reserve(1024);
    b->classes.clear();
    b->class_prop.clear();
    b->class_decay.clear();
    cls.resize((size_t)N);
    int max_sub = -1;
    for (int64_t i = 0; i < N; ++i) {
        const float* pr = property + i * DTB_NPROP;
        float dc[4];
        if (decay) std::memcpy(dc, decay + i * 4, sizeof(dc));
        else default_decay(pr, b->dt, dc);
        Row26 key;
        for (int c = 0; c < 22; ++c) key[c] = fbits(pr[c]);
        for (int c = 0; c < 4; ++c) key[22 + c] = fbits(dc[c]);
        auto it = map.find(key);
        uint32_t id;
        if (it == map.end()) {
            id = (uint32_t)b->classes.size();
            map.emplace(key, id);
            b->classes.push_back(make_class(pr, dc, b->dt));
            std::array<float, 22> row;
            std::memcpy(row.data(), pr, sizeof(float) * 22);
            b->class_prop.push_back(row);
            std::array<float, 4> d4 = {dc[0], dc[1], dc[2], dc[3]};
            b->class_decay.push_back(d4);
            max_sub = std::max(max_sub, b->classes.back().sub);
        } else {
            id = it->second;
        }
        cls[(size_t)i] = id;
    }
    // models/block.py:146 iterates range(sub_idx.max().int() + 1)
    float mx = -INFINITY;
    for (auto& r : b->class_prop) mx = std::max(mx, r[3]);
    b->n_sub = (N > 0 && mx >= 0.0f) ? (int)mx + 1 : 0;
    b->n_classes = (int)b->classes.size();
    b->sub_count.assign((size_t)b->n_sub, 0u);
    for (int64_t i = 0; i < N; ++i) {
        const int s = b->classes[cls[(size_t)i]].sub;
        if (s >= 0 && s < b->n_sub) b->sub_count[(size_t)s]++;
    }
    (void)max_sub;
    return DTB_OK;
}

// ------------------------------------------------------------ input checks
// A NaN in a property row would turn into NaN membrane potentials (models/block.py
// computes with it unchecked); the library refuses such rows up front.  Infinite
// values stay allowed (V_th = +inf marks neurons that never fire).
static int check_property(int64_t N, const float* property, const char* what)
{
    for (int64_t i = 0; i < N; ++i)
        for (int c = 0; c < DTB_NPROP; ++c)
            if (std::isnan(property[i * DTB_NPROP + c]))
                return fail(DTB_ERR_ARG, "%s: property row %lld column %d is NaN", what, (long long)i, c);
    return DTB_OK;
}

// ------------------------------------------------------------ state setup
static int alloc_state(dtb_block* b)
{
    const int64_t N = b->N;
    DevState& s = b->ds;
    s.N = N;
    s.n_words = ((N + 127) / 128) * 4;
    RET(dalloc(b, &s.V, (size_t)N));
    // split receptor-pair planes, the second starting on a 128-neuron boundary (1 KB)
    const int64_t jps = ((N + kWarpNeurons - 1) / kWarpNeurons) * kWarpNeurons;
    RET(dalloc(b, &s.J2, 2 * (size_t)jps));
    s.j_ps = jps;   // split layout: excitatory pairs, then inhibitory pairs
    s.j_es = 1;
    RET(dalloc(b, &s.tlast, (size_t)N));
    RET(dalloc(b, &s.isyn_override, (size_t)N));
    for (int p = 0; p < 2; ++p) RET(dalloc(b, &s.bits[p], (size_t)s.n_words));
    RET(dalloc(b, &s.abits, (size_t)s.n_words));
    RET(dalloc(b, &s.ctl, 1));
    RET(dalloc(b, &s.ev_part, kEvParts));
    RET(dalloc(b, &s.unmapped_nact, 1));
    RET(dalloc(b, &b->d_err, 4));
    CK(cudaMemsetAsync(s.J2, 0, sizeof(float2) * 2 * (size_t)jps, b->stream));
    CK(cudaMemsetAsync(s.tlast, 0, sizeof(float) * (size_t)N, b->stream));
    for (int p = 0; p < 2; ++p) CK(cudaMemsetAsync(s.bits[p], 0, sizeof(uint32_t) * (size_t)s.n_words, b->stream));
    CK(cudaMemsetAsync(s.abits, 0, sizeof(uint32_t) * (size_t)s.n_words, b->stream));
    CK(cudaMemsetAsync(s.ctl, 0, sizeof(Ctl), b->stream));
    CK(cudaMemsetAsync(s.ev_part, 0, sizeof(unsigned long long) * kEvParts, b->stream));
    CK(cudaMemsetAsync(s.unmapped_nact, 0, sizeof(uint32_t), b->stream));
    s.seed = b->seed;
    s.stream_id = b->stream_id;
    s.dt = b->dt;
    s.stage_wait_limit = 1u << 20;
    s.forced_active = nullptr;
    s.forced_new = nullptr;
    return DTB_OK;
}

// Class table, per-neuron class ids, subblock tables and initial V.
static int upload_class_tables(dtb_block* b)
{
    DevState& s = b->ds;
    if (b->n_classes > b->pc_cap || !b->d_pc) {
        const int cap = std::max(64, b->n_classes);
        RET(dalloc(b, &b->d_pc, (size_t)cap));
        b->pc_cap = cap;
    }
    CK(cudaMemcpyAsync(b->d_pc, b->classes.data(), sizeof(ParamClass) * b->classes.size(), cudaMemcpyHostToDevice,
                       b->stream));
    s.pc = b->d_pc;
    if (b->n_sub > b->sub_cap || !b->d_sub_count) {
        const int cap = std::max(16, b->n_sub);
        RET(dalloc(b, &b->d_sub_count, (size_t)cap));
        RET(dalloc(b, &s.sub_spk, (size_t)cap));
        RET(dalloc(b, &s.sub_nact, (size_t)cap));
        RET(dalloc(b, &s.sub_vsum, (size_t)cap));
        RET(dalloc(b, &s.win_spk, (size_t)cap));
        CK(cudaMemsetAsync(s.win_spk, 0, sizeof(unsigned long long) * cap, b->stream));
        CK(cudaMemsetAsync(s.sub_spk, 0, sizeof(uint32_t) * cap, b->stream));
        CK(cudaMemsetAsync(s.sub_nact, 0, sizeof(uint32_t) * cap, b->stream));
        CK(cudaMemsetAsync(s.sub_vsum, 0, sizeof(double) * cap, b->stream));
        b->sub_cap = cap;
        s.st_spk = nullptr;       // stats rows are n_sub wide: reallocate
        b->stats_cap = 0;
    }
    if (b->n_sub)
        CK(cudaMemcpyAsync(b->d_sub_count, b->sub_count.data(), sizeof(uint32_t) * b->n_sub, cudaMemcpyHostToDevice,
                           b->stream));
    s.sub_count = b->d_sub_count;
    s.n_sub = b->n_sub;
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

// Per-tile class ids: the class of a 128-neuron tile whose neurons all share one (the
// update then reads no per-neuron class id for it), else kMixedTile.
static int upload_tile_classes(dtb_block* b, const std::vector<uint32_t>& cls)
{
    DevState& s = b->ds;
    const int64_t nt = (b->N + kWarpNeurons - 1) / kWarpNeurons;
    if (nt <= 0) return DTB_OK;
    std::vector<uint32_t> tc((size_t)nt);
    for (int64_t t = 0; t < nt; ++t) {
        const int64_t n0 = t * kWarpNeurons, n1 = std::min<int64_t>(b->N, n0 + kWarpNeurons);
        uint32_t c = cls[(size_t)n0];
        for (int64_t n = n0 + 1; n < n1; ++n)
            if (cls[(size_t)n] != c) { c = kMixedTile; break; }
        tc[(size_t)t] = c;
    }
    if (!s.tile_cls) {
        uint32_t* d = nullptr;
        RET(dalloc(b, &d, (size_t)nt));
        s.tile_cls = d;
    }
    CK(cudaMemcpy(const_cast<uint32_t*>(s.tile_cls), tc.data(), sizeof(uint32_t) * (size_t)nt, cudaMemcpyHostToDevice));
    return DTB_OK;
}

// Class table, per-neuron class ids, subblock tables and initial V.
static int upload_classes(dtb_block* b, const std::vector<uint32_t>& cls, bool init_v)
{
    DevState& s = b->ds;
    RET(upload_class_tables(b));
    uint32_t* dcls = nullptr;
    RET(dalloc(b, &dcls, (size_t)b->N));
    CK(cudaMemcpy(dcls, cls.data(), sizeof(uint32_t) * (size_t)b->N, cudaMemcpyHostToDevice));
    s.cls = dcls;
    RET(upload_tile_classes(b, cls));
    if (init_v) {
        // models/block.py:56: V = ones * (V_th + V_reset) / 2
        std::vector<float> v0((size_t)b->N);
        for (int64_t i = 0; i < b->N; ++i) {
            const ParamClass& p = b->classes[cls[(size_t)i]];
            volatile float sum = p.Vth + p.Vreset;
            v0[(size_t)i] = sum / 2.0f;
        }
        CK(cudaMemcpy(s.V, v0.data(), sizeof(float) * (size_t)b->N, cudaMemcpyHostToDevice));
    }
    return DTB_OK;
}

static int ensure_stats(dtb_block* b, uint32_t rows)
{
    if (b->stats_cap >= rows && b->ds.st_spk) return DTB_OK;
    const uint32_t cap = std::max<uint32_t>(rows, 64);
    DevState& s = b->ds;
    RET(dalloc(b, &s.st_spk, (size_t)cap * std::max(1, b->n_sub)));
    RET(dalloc(b, &s.st_mean, (size_t)cap * std::max(1, b->n_sub)));
    RET(dalloc(b, &s.st_nact, (size_t)cap));
    b->stats_cap = cap;
    CK(cudaMemcpyAsync(&s.ctl->stats_cap, &cap, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (auto& g : b->graph) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    return DTB_OK;
}

// Host CSR builders: stable counting sorts keep the given entry order
// inside every row (pull: by post, torch.sparse.mm order; push: by pre,
// cuda/src/configuration.cpp:228 stable_sort_by_key).
// rel_out[e]: position of entry e inside its row; carried[d] = carry[e] for
// the entry e placed at d (the pull-row positions travel into the push CSR).
static int build_csr_host(int64_t N, int64_t S, const uint32_t* key, const uint32_t* other, const uint8_t* kind,
                          const float* w, std::vector<int64_t>& rowptr, std::vector<uint32_t>& col,
                          std::vector<float2>& val, int64_t& max_row, std::vector<uint16_t>* rel_out = nullptr,
                          const std::vector<uint16_t>* carry = nullptr, std::vector<uint16_t>* carried = nullptr)
{
    rowptr.assign((size_t)N + 1, 0);
    for (int64_t e = 0; e < S; ++e) rowptr[(size_t)key[e] + 1]++;
    max_row = 0;
    for (int64_t i = 0; i < N; ++i) {
        max_row = std::max<int64_t>(max_row, rowptr[(size_t)i + 1]);
        rowptr[(size_t)i + 1] += rowptr[(size_t)i];
    }
    col.resize((size_t)S);
    val.resize((size_t)S);
    std::vector<int64_t> cur(rowptr.begin(), rowptr.end() - 1);
    if (rel_out) rel_out->resize((size_t)S);
    if (carried) carried->resize((size_t)S);
    for (int64_t e = 0; e < S; ++e) {
        const int64_t d = cur[(size_t)key[e]]++;
        col[(size_t)d] = other[e] | (kind[e] ? kKindBit : 0u);
        val[(size_t)d] = make_float2(w[2 * e], w[2 * e + 1]);
        if (rel_out) (*rel_out)[(size_t)e] = (uint16_t)(d - rowptr[(size_t)key[e]]);
        if (carried) (*carried)[(size_t)d] = (*carry)[(size_t)e];
    }
    return DTB_OK;
}

static int upload_csr(dtb_block* b, const std::vector<int64_t>& rowptr, const std::vector<uint32_t>& col,
                      const std::vector<float2>& val, const int64_t** drow, const uint32_t** dcol, const float2** dval)
{
    int64_t* r = nullptr; uint32_t* c = nullptr; float2* v = nullptr;
    RET(dalloc(b, &r, rowptr.size()));
    RET(dalloc(b, &c, col.size()));
    RET(dalloc(b, &v, val.size()));
    CK(cudaMemcpy(r, rowptr.data(), sizeof(int64_t) * rowptr.size(), cudaMemcpyHostToDevice));
    if (!col.empty()) {
        CK(cudaMemcpy(c, col.data(), sizeof(uint32_t) * col.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(v, val.data(), sizeof(float2) * val.size(), cudaMemcpyHostToDevice));
    }
    *drow = r; *dcol = c; *dval = v;
    return DTB_OK;
}

static void destroy_block(dtb_block* b)
{
    if (!b) return;
    DeviceGuard g(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& gr : b->graph) if (gr) cudaGraphExecDestroy(gr);
    for (void* p : b->allocs) cudaFree(p);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    if (b->pinned) cudaFreeHost(b->pinned);
    if (b->h_run) cudaFreeHost(b->h_run);
    delete b;
}

static int rebuild_groups(dtb_block* b, const int32_t* sub_to_region);

static int finish_create(dtb_block* b)
{
    RET(rebuild_groups(b, nullptr));
    CK(cudaMallocHost((void**)&b->h_run, sizeof(RunParams)));
    RET(ensure_stats(b, 256));
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

// ------------------------------------------------------------ launches
// Statistics outside the update kernel when the subblock / region count is
// large: groups = BOLD regions with their subblocks, plus lone subblocks.
static int rebuild_groups(dtb_block* b, const int32_t* sub_to_region)
{
    DevState& s = b->ds;
    const int n_sub = b->n_sub;
    const int R = b->bold_R;
    s.stats_ext = (n_sub > 512 || R > 128) ? 1 : 0;
    if (!s.stats_ext) return DTB_OK;
    std::vector<int32_t> ptr, sub, reg;
    if (R > 0 && sub_to_region) {
        std::vector<std::vector<int32_t>> members((size_t)R);
        std::vector<int32_t> lone;
        for (int i = 0; i < n_sub; ++i) {
            const int r = sub_to_region[i];
            if (r >= 0 && r < R) members[(size_t)r].push_back(i); else lone.push_back(i);
        }
        ptr.push_back(0);
        for (int r = 0; r < R; ++r) {
            for (int32_t i : members[(size_t)r]) sub.push_back(i);
            ptr.push_back((int32_t)sub.size());
            reg.push_back(r);
        }
        for (int32_t i : lone) { sub.push_back(i); ptr.push_back((int32_t)sub.size()); reg.push_back(-1); }
    } else {
        for (int i = 0; i <= n_sub; ++i) ptr.push_back(i);
        for (int i = 0; i < n_sub; ++i) { sub.push_back(i); reg.push_back(-1); }
    }
    int32_t *dp = nullptr, *ds = nullptr, *dr = nullptr;
    RET(dalloc(b, &dp, ptr.size()));
    RET(dalloc(b, &ds, std::max<size_t>(1, sub.size())));
    RET(dalloc(b, &dr, std::max<size_t>(1, reg.size())));
    CK(cudaMemcpy(dp, ptr.data(), sizeof(int32_t) * ptr.size(), cudaMemcpyHostToDevice));
    if (!sub.empty()) CK(cudaMemcpy(ds, sub.data(), sizeof(int32_t) * sub.size(), cudaMemcpyHostToDevice));
    if (!reg.empty()) CK(cudaMemcpy(dr, reg.data(), sizeof(int32_t) * reg.size(), cudaMemcpyHostToDevice));
    s.grp_ptr = dp; s.grp_sub = ds; s.grp_region = dr;
    s.n_groups = (int)reg.size();
    return DTB_OK;
}

static int launch_stats(dtb_block* b, const DevState& s)
{
    if (s.stats_ext && s.n_groups > 0) {
        k_stats<<<grid_for(s.n_groups, 256), 256, 0, b->stream>>>(s);
        CK(cudaGetLastError());
        b->launches++;
    }
    if (s.n_samples > 0) {
        k_samples<<<grid_for(s.n_samples, 256), 256, 0, b->stream>>>(s);
        CK(cudaGetLastError());
        b->launches++;
    }
    return DTB_OK;
}

// Persistent step kernels: as many CTAs as are resident at once, each warp
// streaming a contiguous run of tiles.
// Dynamic shared memory of the step kernels: the mask gather's per-warp entry lists.
static constexpr int step_dyn_smem(int g)
{
    return g == kGatherMasks ? (kStepThreads / 32) * kMaskList * 10
                             : (g == kGatherStream ? (kStepThreads / 32) * kStreamWarpBytes : 0);
}

template <int G, bool U, bool F, int M>
static int step_blocks_per_sm()
{
    static int v = 0;
    if (!v) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_step<G, U, F, M>, kStepThreads, step_dyn_smem(G));
        if (v < 1) v = 1;
    }
    return v;
}

static void step_grid(const dtb_block* b, int per_sm, unsigned& grid, int& tiles_per_warp)
{
    const int64_t ntiles = (b->N + kWarpNeurons - 1) / kWarpNeurons;
    const int warps = kStepThreads / 32;
    const int64_t max_blocks = (int64_t)std::max(1, b->n_sm) * per_sm;
    int64_t blocks = std::min<int64_t>((ntiles + warps - 1) / warps, max_blocks);
    if (blocks < 1) blocks = 1;
    const int64_t tpw = (ntiles + blocks * warps - 1) / (blocks * warps);
    tiles_per_warp = (int)std::max<int64_t>(1, tpw);
    grid = (unsigned)((ntiles + (int64_t)tiles_per_warp * warps - 1) / ((int64_t)tiles_per_warp * warps));
}

template <int G, bool U, bool F, int M>
static void launch_step_m(dtb_block* b, const DevState& s)
{
    unsigned grid;
    int tpw;
    step_grid(b, step_blocks_per_sm<G, U, F, M>(), grid, tpw);
    k_step<G, U, F, M><<<grid, kStepThreads, step_dyn_smem(G), b->stream>>>(s, tpw);
}

// Update with staged (bulk-copied, one tile ahead) state loads: split J planes
// whose second plane starts on 16 bytes (even plane stride).  M = resident
// CTAs per SM its registers are budgeted for.
template <bool U, bool F, int M>
static void launch_step_staged(dtb_block* b, const DevState& s)
{
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_step<0, U, F, M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kStagedSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step<0, U, F, M, true>, kStepThreads, kStagedSmem);
        if (per_sm < 1) per_sm = 1;
    }
    unsigned grid;
    int tpw;
    step_grid(b, per_sm, grid, tpw);
    k_step<0, U, F, M, true><<<grid, kStepThreads, kStagedSmem, b->stream>>>(s, tpw);
}

static bool staged_layout(const DevState& s) { return s.j_es == 1 && s.j_ps >= s.N && (s.j_ps % 2) == 0; }

// Update that first folds the binned push events of its chunks (one chunk = one bin of
// 2^bin_shift neurons, its sums in 16 << bin_shift bytes of shared memory): each CTA
// takes an equal run of chunks.
template <bool U, bool F, int M>
static void launch_step_bins(dtb_block* b, const DevState& s)
{
    static int per_sm[kBinMaxShift + 1] = {0};
    const int B = s.bin_shift;
    const size_t smem = (size_t)16 << B;
    if (!per_sm[B]) {
        cudaFuncSetAttribute(k_step<kGatherBins, U, F, M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             16 << kBinMaxShift);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[B], k_step<kGatherBins, U, F, M>, kStepThreads, smem);
        if (per_sm[B] < 1) per_sm[B] = 1;
    }
    const int64_t nchunks = (b->N + ((int64_t)1 << B) - 1) >> B;
    const int64_t maxb = (int64_t)std::max(1, b->n_sm) * per_sm[B];
    const int64_t cpc = std::max<int64_t>(1, (nchunks + maxb - 1) / maxb);
    const unsigned grid = (unsigned)std::max<int64_t>(1, (nchunks + cpc - 1) / cpc);
    k_step<kGatherBins, U, F, M><<<grid, kStepThreads, smem, b->stream>>>(s, (int)cpc);
}

// The update with the bin fold and staged state loads: bins of 1024 neurons (one tile per
// warp of a CTA per chunk), the events added into the tiles' staged J planes.
template <bool F, int M>
static void launch_step_bins_staged(dtb_block* b, const DevState& s)
{
    static int per_sm = 0;
    if (!per_sm) {
        cudaFuncSetAttribute(k_step<kGatherBins, true, F, M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kBinStagedSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step<kGatherBins, true, F, M, true>, kStepThreads,
                                                      kBinStagedSmem);
        if (per_sm < 1) per_sm = 1;
    }
    const int64_t nchunks = (b->N + ((int64_t)1 << kBinMinShift) - 1) >> kBinMinShift;
    const int64_t maxb = (int64_t)std::max(1, b->n_sm) * per_sm;
    const int64_t cpc = std::max<int64_t>(1, (nchunks + maxb - 1) / maxb);
    const unsigned grid = (unsigned)std::max<int64_t>(1, (nchunks + cpc - 1) / cpc);
    k_step<kGatherBins, true, F, M, true><<<grid, kStepThreads, kBinStagedSmem, b->stream>>>(s, (int)cpc);
}

static bool staged_layout(const DevState& s);

template <int G, bool U, bool F>
static void launch_step(dtb_block* b, const DevState& s)
{
    if constexpr (G == kGatherBins) {
        if constexpr (U) {
            // step variants 2..4 stage the state (bins of 1024 neurons, split J planes)
            if (b->step_variant >= 2 && s.bin_shift == kBinMinShift && staged_layout(s)) {
                if (b->step_variant == 2) launch_step_bins_staged<F, 2>(b, s);
                else launch_step_bins_staged<F, 3>(b, s);
                return;
            }
        }
        if (b->step_variant == 1 || b->step_variant >= 3) launch_step_bins<U, F, 3>(b, s);
        else launch_step_bins<U, F, 2>(b, s);
        return;
    }
    if constexpr (G == 0) {
        if (b->step_variant == 2 && staged_layout(s)) { launch_step_staged<U, F, 2>(b, s); return; }
        if (b->step_variant == 3 && staged_layout(s)) { launch_step_staged<U, F, 3>(b, s); return; }
        if (b->step_variant == 4 && staged_layout(s)) { launch_step_staged<U, F, 4>(b, s); return; }
    }
    if (b->step_variant == 1) launch_step_m<G, U, F, 3>(b, s);
    else launch_step_m<G, U, F, 2>(b, s);
}

// models/block.py:104-109 reads column iter + 1 of src after replaying column
// iter, so a raster of T columns serves T - 1 steps (an IndexError after that).
static int check_src_steps(dtb_block* b, int64_t n)
{
    const DevState& s = b->ds;
    if (s.n_src <= 0) return DTB_OK;
    if ((int64_t)(b->steps - s.src_from) + n > s.src_T - 1)
        return fail(DTB_ERR_ARG, "input spike raster exhausted: %lld columns serve %lld steps, %lld taken, %lld asked",
                    (long long)s.src_T, (long long)(s.src_T - 1), (long long)(b->steps - s.src_from), (long long)n);
    return DTB_OK;
}

static int launch_src(dtb_block* b, const DevState& s)
{
    CK(cudaMemsetAsync(s.src_val, 0, sizeof(uint32_t) * (size_t)s.n_words, b->stream));
    k_src_bits<<<grid_for(s.n_src, 256), 256, 0, b->stream>>>(s);
    CK(cudaGetLastError());
    b->launches++;
    return DTB_OK;
}

// gather: 0 none, kGatherRows (fused pull gather), kGatherSlots / kGatherMasks (ordered push)
static int launch_update(dtb_block* b, const DevState& s, int gather, bool forced)
{
    if (s.N <= 0) return DTB_OK;
    if (s.n_src > 0 && s.forced_active == s.src_val) {   // input neurons replay their raster
        RET(launch_src(b, s));
        forced = true;
    }
    // the general form also serves the I_syn override and gamma-distributed g_ui
    if (s.gnrn != nullptr || b->override_live) forced = true;
    b->override_live = false;   // this update consumes the override
    if (forced) {
        if (gather == kGatherBins) launch_step<kGatherBins, true, true>(b, s);
        else if (gather == kGatherRows) launch_step<kGatherRows, true, true>(b, s);
        else if (gather == kGatherSlots) launch_step<kGatherSlots, true, true>(b, s);
        else if (gather == kGatherMasks) launch_step<kGatherMasks, true, true>(b, s);
        else if (gather == kGatherStream) launch_step<kGatherStream, true, true>(b, s);
        else launch_step<0, true, true>(b, s);
    } else {
        if (gather == kGatherBins) launch_step<kGatherBins, true, false>(b, s);
        else if (gather == kGatherRows) launch_step<kGatherRows, true, false>(b, s);
        else if (gather == kGatherSlots) launch_step<kGatherSlots, true, false>(b, s);
        else if (gather == kGatherMasks) launch_step<kGatherMasks, true, false>(b, s);
        else if (gather == kGatherStream) launch_step<kGatherStream, true, false>(b, s);
        else launch_step<0, true, false>(b, s);
    }
    CK(cudaGetLastError());
    b->launches++;
    return launch_stats(b, s);
}

// Folds the propagation of the last step into J (end of a pull run).
static int launch_gather_only(dtb_block* b, const DevState& s, int gather = kGatherRows)
{
    if (s.N <= 0) return DTB_OK;
    if (gather == kGatherSlots) launch_step<kGatherSlots, false, false>(b, s);
    else if (gather == kGatherMasks) launch_step<kGatherMasks, false, false>(b, s);
    else if (gather == kGatherStream) launch_step<kGatherStream, false, false>(b, s);
    else launch_step<kGatherRows, false, false>(b, s);
    CK(cudaGetLastError());
    b->launches++;
    return DTB_OK;
}

// how: kScatterJ (push), kScatterSlots / kScatterMasks (ordered push)
static int launch_scatter(dtb_block* b, const DevState& s, int how = kScatterJ)
{
    const int wpw = b->scatter_wpw;
    const int64_t warps = (s.n_words + wpw - 1) / wpw;
    const unsigned grid = grid_for(warps * 32, kScatterThreads);
    if (grid == 0) return DTB_OK;
    const size_t smem = sizeof(uint32_t) * 32 * (size_t)wpw * (kScatterThreads / 32);   // <= 32 KB
    if (how == kScatterSlots) k_scatter<kScatterSlots><<<grid, kScatterThreads, smem, b->stream>>>(s, wpw);
    else if (how == kScatterMasks) k_scatter<kScatterMasks><<<grid, kScatterThreads, smem, b->stream>>>(s, wpw);
    else if (b->scatter_variant == 1) k_scatter<kScatterJ, 6><<<grid, kScatterThreads, smem, b->stream>>>(s, wpw);
    else k_scatter<kScatterJ><<<grid, kScatterThreads, smem, b->stream>>>(s, wpw);
    CK(cudaGetLastError());
    b->launches++;
    return DTB_OK;
}

static void drop_graphs(dtb_block* b)
{
    for (auto& ge : b->graph) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
}

// ------------------------------------------------------------ binned push
// Bin geometry: 2^B neurons per bin (the update's chunk), B >= 10 (one tile per warp of
// the update CTA), at most kBinMaxShift (the unstaged update's 16 << B bytes of sums in
// shared memory).  The default, 10, is the geometry of the staged update (its chunk's
// eight tiles are the warps' stage buffers); the scatter's window of kBinWin bins then
// spans 1M neurons.
static int bin_shift_for(const dtb_block* b)
{
    if (b->bin_shift_req) return b->bin_shift_req;
    return kBinMinShift;
}

// Bitmask words per scatter round: the round's synapses must stay below 2^31.
static int bin_words_for(const dtb_block* b)
{
    const int64_t lim = ((int64_t)1 << 31) - 1;
    int w = b->bin_words;
    while (w > 1 && (int64_t)w * 32 * std::max<int64_t>(1, b->max_out) > lim) w >>= 1;
    return w;
}

static bool bins_possible(const dtb_block* b)
{
    if (!b->has_push || b->N <= 0) return false;
    const int B = bin_shift_for(b);
    if (B > kBinMaxShift || ((b->N + ((int64_t)1 << B) - 1) >> B) > kBinMaxBins) return false;
    return (int64_t)32 * std::max<int64_t>(1, b->max_out) < ((int64_t)1 << 31);   // one round's synapses
}

static void free_bins(dtb_block* b)
{
    DevState& s = b->ds;
    dfree(b, s.bin_idx);
    dfree(b, s.bin_w);
    dfree(b, s.bin_cnt);
    s.n_bins = 0;
    s.bin_cap = 0;
    b->bins_pending = false;
}

static int ensure_bins(dtb_block* b)
{
    DevState& s = b->ds;
    if (s.bin_cnt) return DTB_OK;
    if (!bins_possible(b)) return fail(DTB_ERR_STATE, "binned push not possible for this network");
    const int B = bin_shift_for(b);
    const int64_t n_bins = (b->N + ((int64_t)1 << B) - 1) >> B;
    int64_t cap = (int64_t)b->bin_cap_per_neuron << B;
    cap = std::min<int64_t>(cap, (int64_t)0xffffffffLL / n_bins) & ~(int64_t)7;   // whole 16-byte units per bin
    const size_t entries = (size_t)n_bins * (size_t)cap;
    uint16_t* bi = nullptr; float2* bw = nullptr; uint32_t* bc = nullptr;
    int rc = dalloc(b, &bi, entries);
    if (rc == DTB_OK) rc = dalloc(b, &bw, entries);
    if (rc == DTB_OK) rc = dalloc(b, &bc, (size_t)n_bins);
    if (rc != DTB_OK) {
        dfree(b, bi); dfree(b, bw); dfree(b, bc);
        b->bins_failed = true;
        return rc;
    }
    CK(cudaMemsetAsync(bc, 0, sizeof(uint32_t) * (size_t)n_bins, b->stream));
    s.bin_idx = bi; s.bin_w = bw; s.bin_cnt = bc;
    s.n_bins = n_bins;
    s.bin_cap = (uint32_t)cap;
    s.bin_shift = B;
    static bool smem_set = false;
    if (!smem_set) {
        CK(cudaFuncSetAttribute(k_bin_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, kBinSmem));
        smem_set = true;
    }
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bin_scatter, kBinThreads, kBinSmem));
    b->bin_scatter_per_sm = std::max(1, per_sm);
    b->bins_pending = false;
    drop_graphs(b);
    return DTB_OK;
}

static bool use_bins(dtb_block* b)
{
    if (b->push_method == 1 || !b->has_push) return false;
    if (b->push_method == 0 && (b->bins_failed || !bins_possible(b))) return false;
    return true;
}

static int launch_bin_scatter(dtb_block* b, const DevState& s)
{
    const int wpr = bin_words_for(b);
    const int64_t rounds = (s.n_words + wpr - 1) / wpr;
    if (rounds <= 0) return DTB_OK;
    const unsigned grid = (unsigned)std::min<int64_t>(rounds, (int64_t)std::max(1, b->n_sm) * b->bin_scatter_per_sm);
    k_bin_scatter<<<grid, kBinThreads, kBinSmem, b->stream>>>(s, wpr);
    CK(cudaGetLastError());
    b->launches++;
    return DTB_OK;
}

// Folds events still waiting in the bins into J (before anything else reads J).
static int flush_bins(dtb_block* b)
{
    if (!b->bins_pending) return DTB_OK;
    b->bins_pending = false;
    launch_step_bins<false, false, 2>(b, b->ds);
    CK(cudaGetLastError());
    b->launches++;
    return DTB_OK;
}

// Drops events still waiting in the bins (J is about to be overwritten).
static int discard_bins(dtb_block* b)
{
    if (!b->bins_pending) return DTB_OK;
    b->bins_pending = false;
    CK(cudaMemsetAsync(b->ds.bin_cnt, 0, sizeof(uint32_t) * (size_t)b->ds.n_bins, b->stream));
    return DTB_OK;
}

// Internal propagation methods: DTB_MODE_PUSH, DTB_MODE_PULL (row gather) and
// the ordered push that DTB_MODE_PULL resolves to while activity is low.
constexpr int kModeSlots = 3;
constexpr int kModeMasks = 4;
constexpr int kModeStream = 5;
constexpr int kModeBinned = 6;

static int ensure_slots(dtb_block* b)
{
    DevState& s = b->ds;
    if (s.slots) return DTB_OK;
    uint32_t* cnt = nullptr; uint4* sl = nullptr;
    RET(dalloc(b, &cnt, (size_t)std::max<int64_t>(b->N, 1)));
    RET(dalloc(b, &sl, (size_t)std::max<int64_t>(b->N, 1) * kSlotCap));
    CK(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (size_t)std::max<int64_t>(b->N, 1), b->stream));
    s.slot_cnt = cnt;
    s.slots = sl;
    drop_graphs(b);
    return DTB_OK;
}

static bool masks_possible(const dtb_block* b) { return b->has_qpos && b->has_push && b->max_in <= 32 * kMaskWords; }

static int ensure_masks(dtb_block* b)
{
    DevState& s = b->ds;
    if (s.pmask) return DTB_OK;
    const size_t words = (size_t)std::max<int64_t>(b->N, 1) * 2 * kMaskWords;
    uint32_t* m = nullptr;
    RET(dalloc(b, &m, words));
    CK(cudaMemsetAsync(m, 0, sizeof(uint32_t) * words, b->stream));
    s.pmask = m;
    drop_graphs(b);
    return DTB_OK;
}

// n steps with one propagation method (no host synchronisation).
static int enqueue_steps(dtb_block* b, int n, int mode)
{
    if (n <= 0) return DTB_OK;
    const DevState& s = b->ds;
    if (mode == DTB_MODE_PUSH) {
        for (int k = 0; k < n; ++k) {
            RET(launch_update(b, s, 0, false));
            RET(launch_scatter(b, s));
        }
    } else if (mode == kModeBinned) {
        for (int k = 0; k < n; ++k) {
            RET(launch_update(b, s, kGatherBins, false));
            RET(launch_bin_scatter(b, s));
        }
    } else if (mode == kModeSlots || mode == kModeMasks) {
        const int g = mode == kModeSlots ? kGatherSlots : kGatherMasks;
        const int how = mode == kModeSlots ? kScatterSlots : kScatterMasks;
        RET(launch_update(b, s, 0, false));
        RET(launch_scatter(b, s, how));
        for (int k = 1; k < n; ++k) {
            RET(launch_update(b, s, g, false));
            RET(launch_scatter(b, s, how));
        }
        RET(launch_gather_only(b, s, g));
    } else {
        const int g = mode == kModeStream ? kGatherStream : kGatherRows;
        RET(launch_update(b, s, 0, false));
        for (int k = 1; k < n; ++k) RET(launch_update(b, s, g, false));
        RET(launch_gather_only(b, s, g));
    }
    return DTB_OK;
}

static int enqueue_chunk_inner(dtb_block* b, int n, int mode);

// The binned push leaves its last step's events in the bins; any other method first
// folds them into J.
static int enqueue_chunk(dtb_block* b, int n, int mode)
{
    if (n <= 0) return DTB_OK;
    if (mode != kModeBinned) RET(flush_bins(b));
    RET(enqueue_chunk_inner(b, n, mode));
    if (mode == kModeBinned) b->bins_pending = true;
    return DTB_OK;
}

static int enqueue_chunk_inner(dtb_block* b, int n, int mode)
{
    // a chunk whose first update takes the I_syn override runs ungraphed (the captured graphs
    // hold the plain form of every step)
    if (!b->use_graphs || n != b->chunk || b->stream == nullptr || b->override_live) return enqueue_steps(b, n, mode);
    cudaGraphExec_t& ge = b->graph[mode];
    if (!ge) {
        cudaGraph_t g = nullptr;
        const int64_t before = b->launches;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_steps(b, n, mode);
        b->graph_len[mode] = (int)(b->launches - before);
        b->launches = before;
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (rc != DTB_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (ce != cudaSuccess) return fail(DTB_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { ge = nullptr; return fail(DTB_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ce)); }
    }
    CK(cudaGraphLaunch(ge, b->stream));
    b->launches += b->graph_len[mode];
    return DTB_OK;
}

static int choose_mode(dtb_block* b, int mode)
{
    if (mode == DTB_MODE_PUSH && !b->has_push) return DTB_MODE_PULL;
    if (mode == DTB_MODE_PULL && !b->has_pull) return DTB_MODE_PUSH;
    if (mode != DTB_MODE_AUTO) return mode;
    if (!b->has_push) return DTB_MODE_PULL;
    if (!b->has_pull) return DTB_MODE_PUSH;
    const double f = b->last_frac < 0.0 ? 0.0 : b->last_frac;
    return f > b->pull_threshold ? DTB_MODE_PULL : DTB_MODE_PUSH;
}

// DTB_MODE_PULL runs as ordered push when the push CSR carries pull-row
// positions and activity is low enough that rows rarely overflow their slots.
static int resolve_method(dtb_block* b, int m)
{
    if (m == DTB_MODE_PUSH) return (use_bins(b) && ensure_bins(b) == DTB_OK) ? kModeBinned : DTB_MODE_PUSH;
    if (m != DTB_MODE_PULL || b->pull_method == 1) return m;
    if (b->pull_method == 4 || !b->has_qpos || !b->has_push) return kModeStream;
    if (b->pull_method == 2) return kModeSlots;
    if (b->pull_method == 3) return kModeMasks;
    const double f = b->last_frac < 0.0 ? 0.0 : b->last_frac;
    return f <= b->slot_threshold ? kModeSlots : kModeStream;   // slots measured faster than masks on B200
}

static int ensure_method(dtb_block* b, int mm)
{
    if (mm == kModeSlots) return ensure_slots(b);
    if (mm == kModeMasks) return ensure_masks(b);
    return DTB_OK;
}

static int set_run_params(dtb_block* b, float noise_rate, int isolated)
{
    b->h_run->run_base = b->steps;
    b->h_run->noise_rate = noise_rate;
    b->h_run->isolated = isolated ? 1 : 0;
    CK(cudaMemcpyAsync(&b->ds.ctl->run_base, b->h_run, sizeof(RunParams), cudaMemcpyHostToDevice, b->stream));
    return DTB_OK;
}

// Copies `rows` stats rows to the caller (row offset `row0` of the outputs).
static int emit_stats(dtb_block* b, int rows, int64_t row0, float* sum_out, float* mean_out, uint32_t* nact_out,
                      int where, std::vector<uint32_t>* nact_host)
{
    const size_t ns = (size_t)b->n_sub;
    const size_t bs = rows * ns * sizeof(float);
    const size_t bn = rows * sizeof(uint32_t);
    if (where == DTB_DEVICE) {
        if (sum_out && bs) CK(cudaMemcpyAsync(sum_out + row0 * ns, b->ds.st_spk, bs, cudaMemcpyDeviceToDevice, b->stream));
        if (mean_out && bs) CK(cudaMemcpyAsync(mean_out + row0 * ns, b->ds.st_mean, bs, cudaMemcpyDeviceToDevice, b->stream));
        if (nact_out) CK(cudaMemcpyAsync(nact_out + row0, b->ds.st_nact, bn, cudaMemcpyDeviceToDevice, b->stream));
    }
    const bool need_host = where == DTB_HOST || nact_host;
    if (need_host) {
        RET(ensure_pinned(b, 2 * bs + bn + 64));   // + the error word
        char* p = reinterpret_cast<char*>(b->pinned);
        if (where == DTB_HOST && bs) {
            if (sum_out) CK(cudaMemcpyAsync(p, b->ds.st_spk, bs, cudaMemcpyDeviceToHost, b->stream));
            if (mean_out) CK(cudaMemcpyAsync(p + bs, b->ds.st_mean, bs, cudaMemcpyDeviceToHost, b->stream));
        }
        CK(cudaMemcpyAsync(p + 2 * bs, b->ds.st_nact, bn, cudaMemcpyDeviceToHost, b->stream));
        uint32_t* herr = reinterpret_cast<uint32_t*>(p + ((2 * bs + bn + 7) & ~(size_t)7));
        CK(cudaMemcpyAsync(herr, &b->ds.ctl->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, b->stream));
        CK(cudaStreamSynchronize(b->stream));
        if (*herr) {   // reported once: the flags are cleared
            CK(cudaMemsetAsync(&b->ds.ctl->err, 0, sizeof(uint32_t), b->stream));
            CK(cudaStreamSynchronize(b->stream));
            if (*herr & kErrGeneralSkipped)
                return fail(DTB_ERR_STATE, "internal: an update ran without the I_syn override or gamma g_ui it needed");
            if (*herr & (kErrStageTimeout | kErrStageDrain))
                return fail(DTB_ERR_CUDA, "a staged state copy did not complete in time%s (the update loaded that "
                            "state from global memory instead)", (*herr & kErrStageDrain) ? " and had not landed at exit" : "");
        }
        if (where == DTB_HOST) {
            if (sum_out && bs) std::memcpy(sum_out + row0 * ns, p, bs);
            if (mean_out && bs) std::memcpy(mean_out + row0 * ns, p + bs, bs);
            if (nact_out) std::memcpy(nact_out + row0, p + 2 * bs, bn);
        }
        if (nact_host) {
            nact_host->resize(rows);
            std::memcpy(nact_host->data(), p + 2 * bs, bn);
        }
    }
    return DTB_OK;
}

template <typename T>
static BoldScalars<T> bold_scalars(const dtb_bold* m)
{
    BoldScalars<T> c;
    const double div_alpha = 1.0 / m->alpha;
    c.eps = (T)m->eps; c.ts = (T)m->ts; c.tf = (T)m->tf; c.t0 = (T)m->t0; c.E0 = (T)m->E0; c.V0 = (T)m->V0;
    c.dt = (T)m->dt; c.base = (T)(1.0 - m->E0); c.exq = (T)(div_alpha - 1.0); c.exv = (T)div_alpha;
    c.k7 = (T)(7.0 * m->E0); c.k2 = (T)(2.0 * m->E0 - 0.2); c.one_em5 = (T)1e-05;
    return c;
}

// ------------------------------------------------------------ C ABI
extern "C" {

int dtb_abi_version(void) { return DTB_ABI_VERSION; }

int dtb_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return DTB_ERR_ARG;
    std::snprintf(buf, len, "%s", g_err.c_str());
    return DTB_OK;
}

static int create_common(dtb_block* b, int device, float dt, uint64_t seed, uint32_t stream_id)
{
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(DTB_ERR_ARG, "device %d out of range (%d devices)", device, ndev);
    if (!(dt > 0.0f)) return fail(DTB_ERR_ARG, "dt must be positive");
    b->device = device;
    b->dt = dt;
    b->seed = seed;
    b->stream_id = stream_id;
    CK(cudaSetDevice(device));
    CK(cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking));
    b->stream = b->own_stream;
    return DTB_OK;
}

// Host sort of push rows longer than the device sort holds (same key).
static int sort_long_push_rows(dtb_block* b, const std::vector<int64_t>& qrow, uint32_t* qcol, float2* qw,
                               uint16_t* qpos)
{
    for (int64_t r = 0; r < b->N; ++r) {
        const int64_t e0 = qrow[(size_t)r], len = qrow[(size_t)r + 1] - e0;
        if (len <= kSortCap) continue;
        std::vector<uint32_t> c((size_t)len), c2((size_t)len);
        std::vector<float2> w((size_t)len), w2((size_t)len);
        std::vector<uint16_t> p(qpos ? (size_t)len : 0), p2(qpos ? (size_t)len : 0);
        CK(cudaMemcpy(c.data(), qcol + e0, 4 * (size_t)len, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.data(), qw + e0, 8 * (size_t)len, cudaMemcpyDeviceToHost));
        if (qpos) CK(cudaMemcpy(p.data(), qpos + e0, 2 * (size_t)len, cudaMemcpyDeviceToHost));
        std::vector<int64_t> ord((size_t)len);
        for (int64_t k = 0; k < len; ++k) ord[(size_t)k] = k;
        auto key = [&](int64_t k) {
            return ((uint64_t)(c[(size_t)k] & kIndexMask) << 32) | (uint64_t)(c[(size_t)k] & kKindBit) |
                   (qpos ? (uint64_t)p[(size_t)k] : 0ull);
        };
        std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t z) { return key(a) < key(z); });
        for (int64_t k = 0; k < len; ++k) {
            c2[(size_t)k] = c[(size_t)ord[(size_t)k]];
            w2[(size_t)k] = w[(size_t)ord[(size_t)k]];
            if (qpos) p2[(size_t)k] = p[(size_t)ord[(size_t)k]];
        }
        CK(cudaMemcpy(qcol + e0, c2.data(), 4 * (size_t)len, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(qw + e0, w2.data(), 8 * (size_t)len, cudaMemcpyHostToDevice));
        if (qpos) CK(cudaMemcpy(qpos + e0, p2.data(), 2 * (size_t)len, cudaMemcpyHostToDevice));
    }
    return DTB_OK;
}

// Push CSR (rows = presynaptic neurons) by transposing the pull CSR on the
// device: rows ordered by (postsynaptic neuron, kind, pull-row position), with
// every entry's pull-row position (qpos, for the ordered push) when in-degrees
// fit 16 bits.  counts: device [N+1] out-degrees, reused as fill cursors.
static int build_push_device(dtb_block* b, uint32_t* counts, bool with_qpos)
{
    const int64_t N = b->N, S = b->S;
    int64_t* qrow = nullptr; uint32_t* qcol = nullptr; float2* qw = nullptr; uint16_t* qpos = nullptr;
    RET(dalloc(b, &qrow, (size_t)N + 1));
    RET(dalloc(b, &qcol, (size_t)S));
    RET(dalloc(b, &qw, (size_t)S));
    if (with_qpos) RET(dalloc(b, &qpos, (size_t)S));
    long long* tiles = nullptr;
    const int64_t ntiles = (N + kScanTile - 1) / kScanTile;
    CK(cudaMalloc(&tiles, sizeof(long long) * (size_t)(ntiles + 1)));
    k_scan_tiles<<<(unsigned)ntiles, kScanThreads, 0, b->stream>>>(counts, N, qrow, tiles);
    k_scan_tile_sums<<<1, kScanThreads, 0, b->stream>>>(tiles, ntiles);
    k_scan_add<<<grid_for(N, 256), 256, 0, b->stream>>>(qrow, N, tiles, ntiles);
    cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (size_t)(N + 1), b->stream);
    k_fill_push<<<grid_for(N * 32, 256), 256, 0, b->stream>>>(N, b->ds.prow, b->ds.pcol, b->ds.pw, qrow, counts,
                                                               qcol, qw, qpos);
    cudaMemsetAsync(b->d_err, 0, 16, b->stream);
    const size_t smem = (sizeof(unsigned long long) + sizeof(float2) + sizeof(uint16_t)) * (size_t)kSortCap * kSortWarps;
    cudaFuncSetAttribute(k_sort_push_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_sort_push_rows<<<grid_for(N, kSortWarps), kSortWarps * 32, smem, b->stream>>>(N, qrow, qcol, qw, qpos, b->d_err);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(tiles);
    unsigned herr[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(herr, b->d_err, 16, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(DTB_ERR_CUDA, "push CSR build: %s", cudaGetErrorString(e));
    std::vector<int64_t> hq((size_t)N + 1);
    CK(cudaMemcpy(hq.data(), qrow, sizeof(int64_t) * hq.size(), cudaMemcpyDeviceToHost));
    if (herr[0]) RET(sort_long_push_rows(b, hq, qcol, qw, qpos));
    int64_t mx = 0;
    for (int64_t i = 0; i < N; ++i) mx = std::max(mx, hq[(size_t)i + 1] - hq[(size_t)i]);
    b->max_out = mx;
    b->ds.qrow = qrow; b->ds.qcol = qcol; b->ds.qw = qw; b->ds.qpos = qpos;
    b->has_push = true;
    b->has_qpos = qpos != nullptr;
    return DTB_OK;
}

int dtb_block_create(const dtb_block_desc* d, dtb_block** out)
{
    if (!d || !out) return fail(DTB_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->n_neurons <= 0 || d->n_neurons > (int64_t)kIndexMask) return fail(DTB_ERR_LIMIT, "n_neurons must be in [1, 2^31-1]");
    if (!d->property) return fail(DTB_ERR_ARG, "property is null");
    if (d->n_synapses < 0) return fail(DTB_ERR_ARG, "n_synapses < 0");
    if (d->n_synapses > 0 && (!d->post || !d->pre || !d->kind || !d->weight)) return fail(DTB_ERR_ARG, "synapse arrays are null");
    const int64_t N = d->n_neurons, S = d->n_synapses;
    RET(check_property(N, d->property, "dtb_block_create"));
    for (int64_t e = 0; e < S; ++e) {
        if (d->post[e] >= (uint64_t)N || d->pre[e] >= (uint64_t)N)
            return fail(DTB_ERR_ARG, "synapse %lld references neuron out of range (post %u, pre %u, N %lld)", (long long)e,
                        d->post[e], d->pre[e], (long long)N);
        if (d->kind[e] != 0 && d->kind[e] != 2) return fail(DTB_ERR_ARG, "synapse %lld: kind must be 0 or 2", (long long)e);
    }
    dtb_block* b = new dtb_block();
    DeviceGuard guard(d->device < 0 ? 0 : d->device);
    int rc = create_common(b, d->device, d->dt, d->seed, d->stream_id);
    if (rc == DTB_OK) {
        b->N = N;
        b->S = S;
        std::vector<uint32_t> cls;
        rc = build_classes(b, N, d->property, d->decay, cls);
        if (rc == DTB_OK) rc = alloc_state(b);
        if (rc == DTB_OK) rc = upload_classes(b, cls, true);
        if (rc == DTB_OK) {
            std::vector<int64_t> rp; std::vector<uint32_t> col; std::vector<float2> val;
            std::vector<uint16_t> rel, qpos;
            rc = build_csr_host(N, S, d->post, d->pre, d->kind, d->weight, rp, col, val, b->max_in,
                                d->build_push ? &rel : nullptr);
            if (rc == DTB_OK) rc = upload_csr(b, rp, col, val, &b->ds.prow, &b->ds.pcol, &b->ds.pw);
            b->has_pull = (rc == DTB_OK);
            if (rc == DTB_OK && d->build_push) {
                const bool pos16 = b->max_in <= 65535;   // pull-row positions fit 16 bits
                rc = build_csr_host(N, S, d->pre, d->post, d->kind, d->weight, rp, col, val, b->max_out, nullptr,
                                    pos16 ? &rel : nullptr, pos16 ? &qpos : nullptr);
                if (rc == DTB_OK) rc = upload_csr(b, rp, col, val, &b->ds.qrow, &b->ds.qcol, &b->ds.qw);
                b->has_push = (rc == DTB_OK);
                if (rc == DTB_OK && pos16) {
                    uint16_t* dq = nullptr;
                    rc = dalloc(b, &dq, (size_t)S);
                    if (rc == DTB_OK && S > 0) {
                        cudaError_t e = cudaMemcpy(dq, qpos.data(), sizeof(uint16_t) * (size_t)S, cudaMemcpyHostToDevice);
                        if (e != cudaSuccess) rc = fail(DTB_ERR_CUDA, "qpos upload: %s", cudaGetErrorString(e));
                    }
                    b->ds.qpos = dq;
                    b->has_qpos = (rc == DTB_OK);
                }
            }
        }
        if (rc == DTB_OK) rc = finish_create(b);
    }
    if (rc != DTB_OK) { destroy_block(b); return rc; }
    *out = b;
    return DTB_OK;
}

int dtb_block_create_synthetic(const dtb_synth_desc* d, dtb_block** out)
{
    if (!d || !out) return fail(DTB_ERR_ARG, "null argument");
    *out = nullptr;
    const int R = d->n_regions;
    if (R <= 0 || !d->region_start || !d->region_n_exc || !d->class_property || (!d->cum && !d->src_count))
        return fail(DTB_ERR_ARG, "bad synthetic description");
    if (d->K < 1 || d->K > 1024) return fail(DTB_ERR_LIMIT, "K must be in [1, 1024]");
    const int64_t N = d->region_start[R];
    if (d->region_start[0] != 0 || N <= 0 || N > (int64_t)kIndexMask) return fail(DTB_ERR_LIMIT, "bad neuron count");
    for (int r = 0; r < R; ++r) {
        if (d->region_start[r + 1] < d->region_start[r]) return fail(DTB_ERR_ARG, "region_start must be non-decreasing");
        if (d->region_n_exc[r] < 0 || d->region_n_exc[r] > d->region_start[r + 1] - d->region_start[r])
            return fail(DTB_ERR_ARG, "region_n_exc out of range");
    }
    const int64_t S = N * (int64_t)d->K;
    // source-region tables: explicit (ensembles) or derived from cum[R][R]
    std::vector<int32_t> src_base(R), src_count(R), region_member(R);
    std::vector<int64_t> cum_off(R), member_start;
    std::vector<uint64_t> member_seed;
    std::vector<float> cum_flat;
    const bool ens = d->src_count != nullptr;
    if (ens) {
        if (!d->src_base || !d->cum_off || !d->cum_flat || d->n_members <= 0 || !d->region_member ||
            !d->member_start || !d->member_seed)
            return fail(DTB_ERR_ARG, "ensemble tables incomplete");
        int64_t flat = 0;
        for (int r = 0; r < R; ++r) {
            src_base[r] = d->src_base[r]; src_count[r] = d->src_count[r]; cum_off[r] = d->cum_off[r];
            region_member[r] = d->region_member[r];
            if (src_count[r] < 1 || src_base[r] < 0 || src_base[r] + src_count[r] > R || cum_off[r] < 0 ||
                region_member[r] < 0 || region_member[r] >= d->n_members)
                return fail(DTB_ERR_ARG, "region %d: bad source table or member", r);
            flat = std::max<int64_t>(flat, cum_off[r] + src_count[r]);
        }
        cum_flat.assign(d->cum_flat, d->cum_flat + flat);
        member_start.assign(d->member_start, d->member_start + d->n_members);
        member_seed.assign(d->member_seed, d->member_seed + d->n_members);
        for (int m = 0; m < d->n_members; ++m)
            if (member_start[m] % kWarpNeurons != 0 || member_start[m] < 0 || member_start[m] > N)
                return fail(DTB_ERR_ARG, "member %d must start on a multiple of %d neurons", m, kWarpNeurons);
        for (int r = 0; r < R; ++r)
            if (d->region_start[r] < member_start[region_member[r]])
                return fail(DTB_ERR_ARG, "region %d starts before its member", r);
    } else {
        for (int r = 0; r < R; ++r) { src_base[r] = 0; src_count[r] = R; cum_off[r] = (int64_t)r * R; region_member[r] = 0; }
        cum_flat.assign(d->cum, d->cum + (size_t)R * R);
        member_start.assign(1, 0);
        member_seed.assign(1, d->gen_seed);
    }
    dtb_block* b = new dtb_block();
    DeviceGuard guard(d->device < 0 ? 0 : d->device);
    int rc = create_common(b, d->device, d->dt, d->seed, d->stream_id);
    std::vector<uint32_t> cls;
    if (rc == DTB_OK) {
        b->N = N;
        b->S = S;
        // classes 2r (excitatory) / 2r+1 (inhibitory); subblock from property column 3
        const int nc = 2 * R;
        b->classes.clear(); b->class_prop.clear(); b->class_decay.clear();
        int max_sub = -1;
        for (int c = 0; c < nc; ++c) {
            const float* pr = d->class_property + (size_t)c * DTB_NPROP;
            float dc[4];
            if (d->class_decay) std::memcpy(dc, d->class_decay + (size_t)c * 4, sizeof(dc));
            else default_decay(pr, b->dt, dc);
            ParamClass p = make_class(pr, dc, b->dt);
            p.member = ens ? region_member[c / 2] : -1;
            max_sub = std::max(max_sub, p.sub);
            b->classes.push_back(p);
            std::array<float, 22> row; std::memcpy(row.data(), pr, sizeof(float) * 22);
            b->class_prop.push_back(row);
            b->class_decay.push_back({dc[0], dc[1], dc[2], dc[3]});
        }
        b->n_classes = nc;
        b->n_sub = max_sub + 1;
        b->sub_count.assign((size_t)std::max(0, b->n_sub), 0u);
        cls.resize((size_t)N);
        for (int r = 0; r < R; ++r) {
            const int64_t s0 = d->region_start[r], s1 = d->region_start[r + 1], ne = d->region_n_exc[r];
            for (int64_t i = s0; i < s1; ++i) cls[(size_t)i] = (uint32_t)(2 * r + ((i - s0) >= ne ? 1 : 0));
            const int se = b->classes[(size_t)(2 * r)].sub, si = b->classes[(size_t)(2 * r + 1)].sub;
            if (se >= 0) b->sub_count[(size_t)se] += (uint32_t)ne;
            if (si >= 0) b->sub_count[(size_t)si] += (uint32_t)(s1 - s0 - ne);
        }
        rc = alloc_state(b);
        if (rc == DTB_OK) rc = upload_classes(b, cls, true);
        if (rc == DTB_OK && ens) {
            int64_t* ms = nullptr;
            rc = dalloc(b, &ms, member_start.size());
            if (rc == DTB_OK) {
                cudaMemcpy(ms, member_start.data(), sizeof(int64_t) * member_start.size(), cudaMemcpyHostToDevice);
                b->ds.member_start = ms;
            }
        }
    }
    // generate the pull CSR on the device
    if (rc == DTB_OK) {
        int64_t* prow = nullptr; uint32_t* pcol = nullptr; float2* pw = nullptr;
        int64_t* rs = nullptr; int64_t* ne = nullptr; float* cum = nullptr; uint32_t* outdeg = nullptr;
        rc = dalloc(b, &prow, (size_t)N + 1);
        if (rc == DTB_OK) rc = dalloc(b, &pcol, (size_t)S);
        if (rc == DTB_OK) rc = dalloc(b, &pw, (size_t)S);
        // temporaries (freed at the end of creation)
        void *t_rs = nullptr, *t_ne = nullptr, *t_cum = nullptr, *t_out = nullptr, *t_tab = nullptr;
        const size_t tab_bytes = sizeof(int32_t) * 3 * R + sizeof(int64_t) * R + sizeof(int64_t) * member_start.size() +
                                 sizeof(uint64_t) * member_seed.size() + 64;
        if (rc == DTB_OK) {
            cudaError_t e = cudaMalloc(&t_rs, sizeof(int64_t) * (R + 1));
            if (e == cudaSuccess) e = cudaMalloc(&t_ne, sizeof(int64_t) * R);
            if (e == cudaSuccess) e = cudaMalloc(&t_cum, sizeof(float) * std::max<size_t>(1, cum_flat.size()));
            if (e == cudaSuccess) e = cudaMalloc(&t_out, sizeof(uint32_t) * (size_t)(N + 1));
            if (e == cudaSuccess) e = cudaMalloc(&t_tab, tab_bytes);
            if (e != cudaSuccess) { cudaGetLastError(); rc = fail(DTB_ERR_NOMEM, "generator temporaries: %s", cudaGetErrorString(e)); }
            rs = (int64_t*)t_rs; ne = (int64_t*)t_ne; cum = (float*)t_cum; outdeg = (uint32_t*)t_out;
        }
        int64_t* d_cum_off = nullptr; int64_t* d_mstart = nullptr; uint64_t* d_mseed = nullptr;
        int32_t* d_sbase = nullptr; int32_t* d_scount = nullptr; int32_t* d_rmem = nullptr;
        if (rc == DTB_OK) {
            char* tp = (char*)t_tab;
            d_cum_off = (int64_t*)tp; tp += sizeof(int64_t) * R;
            d_mstart = (int64_t*)tp; tp += sizeof(int64_t) * member_start.size();
            d_mseed = (uint64_t*)tp; tp += sizeof(uint64_t) * member_seed.size();
            d_sbase = (int32_t*)tp; tp += sizeof(int32_t) * R;
            d_scount = (int32_t*)tp; tp += sizeof(int32_t) * R;
            d_rmem = (int32_t*)tp;
            cudaMemcpy(d_cum_off, cum_off.data(), sizeof(int64_t) * R, cudaMemcpyHostToDevice);
            cudaMemcpy(d_mstart, member_start.data(), sizeof(int64_t) * member_start.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(d_mseed, member_seed.data(), sizeof(uint64_t) * member_seed.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(d_sbase, src_base.data(), sizeof(int32_t) * R, cudaMemcpyHostToDevice);
            cudaMemcpy(d_scount, src_count.data(), sizeof(int32_t) * R, cudaMemcpyHostToDevice);
            cudaMemcpy(d_rmem, region_member.data(), sizeof(int32_t) * R, cudaMemcpyHostToDevice);
        }
        if (rc == DTB_OK) {
            cudaMemcpy(rs, d->region_start, sizeof(int64_t) * (R + 1), cudaMemcpyHostToDevice);
            cudaMemcpy(ne, d->region_n_exc, sizeof(int64_t) * R, cudaMemcpyHostToDevice);
            cudaMemcpy(cum, cum_flat.data(), sizeof(float) * cum_flat.size(), cudaMemcpyHostToDevice);
            cudaMemset(outdeg, 0, sizeof(uint32_t) * (size_t)(N + 1));
            cudaMemset(b->d_err, 0, 16);
            // rowptr = i*K
            std::vector<int64_t> hrow((size_t)N + 1);
            for (int64_t i = 0; i <= N; ++i) hrow[(size_t)i] = i * d->K;
            cudaMemcpy(prow, hrow.data(), sizeof(int64_t) * hrow.size(), cudaMemcpyHostToDevice);
            GenArgs g;
            g.N = N; g.R = R; g.region_start = rs; g.region_n_exc = ne; g.K = d->K;
            g.src_base = d_sbase; g.src_count = d_scount; g.cum_off = d_cum_off; g.cum_flat = cum;
            g.region_member = d_rmem; g.member_start = d_mstart; g.member_seed = d_mseed;
            int Kp = 1; while (Kp < d->K) Kp <<= 1;
            g.Kp = Kp; g.w_scale = d->w_scale; g.pcol = pcol; g.pw = pw;
            g.outdeg = d->build_push ? outdeg : nullptr; g.err = b->d_err;
            const size_t smem = sizeof(unsigned long long) * (size_t)Kp * kGenWarps;
            cudaFuncSetAttribute(k_gen_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_gen_rows<<<grid_for(N, kGenWarps), kGenWarps * 32, smem, b->stream>>>(g);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
            unsigned herr[4] = {0, 0, 0, 0};
            if (e == cudaSuccess) e = cudaMemcpy(herr, b->d_err, 16, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = fail(DTB_ERR_CUDA, "generator: %s", cudaGetErrorString(e));
            else if (herr[0]) rc = fail(DTB_ERR_ARG, "generator: %u rows could not draw K distinct sources", herr[0]);
            b->ds.prow = prow; b->ds.pcol = pcol; b->ds.pw = pw;
            b->has_pull = (rc == DTB_OK);
            b->max_in = d->K;
        }
        // push CSR by transposition on the device
        if (rc == DTB_OK && d->build_push) rc = build_push_device(b, outdeg, d->K <= 65535);
        cudaFree(t_rs); cudaFree(t_ne); cudaFree(t_cum); cudaFree(t_out); cudaFree(t_tab);
    }
    if (rc == DTB_OK) rc = finish_create(b);
    if (rc != DTB_OK) { destroy_block(b); return rc; }
    *out = b;
    return DTB_OK;
}

int dtb_block_create_from_npz(const char* dir, float dt, uint64_t seed, uint32_t stream_id, int device, int build_push,
                              dtb_block** out)
{
    if (!dir || !out) return fail(DTB_ERR_ARG, "null argument");
    *out = nullptr;
    // generation/read_block.py:31-40: block_0.npz, block_1.npz, ... and their bases.
    // Two passes over the files keep host memory at one file's synapses: the first
    // reads the properties and counts the synapses, the second sorts every file's
    // synapses into its own pull rows (a file holds every row of its population)
    // and copies them to the device.
    std::vector<std::string> paths;
    for (int i = 0;; ++i) {
        std::string path = std::string(dir) + "/block_" + std::to_string(i) + ".npz";
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) break;
        std::fclose(f);
        paths.push_back(path);
    }
    if (paths.empty()) return fail(DTB_ERR_IO, "no block_0.npz in %s", dir);
    const size_t F = paths.size();
    std::vector<int64_t> bases(F + 1, 0), syn(F + 1, 0);
    std::vector<float> prop;
    {
        const std::vector<std::string> only = {"property", "output_neuron_idx"};
        for (size_t i = 0; i < F; ++i) {
            std::map<std::string, NpyArray> m;
            std::vector<std::string> names;
            std::string err;
            if (!npz_read(paths[i], m, err, &only, &names)) return fail(DTB_ERR_FORMAT, "%s", err.c_str());
            auto it = m.find("property");
            if (it == m.end() || it->second.shape.size() != 2 || it->second.shape[1] != DTB_NPROP ||
                it->second.descr != "<f4")
                return fail(DTB_ERR_FORMAT, "block_%zu.npz: property must be float32 [N,22]", i);
            for (auto& nm : names)
                if (nm == "src_timestamp" || nm == "src_neuron_idx")
                    return fail(DTB_ERR_FORMAT, "block_%zu.npz: input (src) blocks are not supported", i);
            if (!m.count("output_neuron_idx")) return fail(DTB_ERR_FORMAT, "block_%zu.npz: missing output_neuron_idx", i);
            bases[i + 1] = bases[i] + it->second.shape[0];
            syn[i + 1] = syn[i] + m["output_neuron_idx"].count();
            const size_t at = prop.size();
            prop.resize(at + it->second.data.size() / sizeof(float));
            std::memcpy(prop.data() + at, it->second.data.data(), it->second.data.size());
        }
    }
    const int64_t N = bases.back(), S = syn.back();
    if (N <= 0 || N > (int64_t)kIndexMask) return fail(DTB_ERR_LIMIT, "n_neurons must be in [1, 2^31-1]");
    RET(check_property(N, prop.data(), "dtb_block_create_from_npz"));
    dtb_block* b = new dtb_block();
    DeviceGuard guard(device < 0 ? 0 : device);
    int rc = create_common(b, device, dt, seed, stream_id);
    std::vector<uint32_t> cls;
    if (rc == DTB_OK) {
        b->N = N;
        b->S = S;
        rc = build_classes(b, N, prop.data(), nullptr, cls);
    }
    if (rc == DTB_OK) rc = alloc_state(b);
    if (rc == DTB_OK) rc = upload_classes(b, cls, true);
    int64_t* prow = nullptr; uint32_t* pcol = nullptr; float2* pw = nullptr; uint32_t* counts = nullptr;
    if (rc == DTB_OK) rc = dalloc(b, &prow, (size_t)N + 1);
    if (rc == DTB_OK) rc = dalloc(b, &pcol, (size_t)S);
    if (rc == DTB_OK) rc = dalloc(b, &pw, (size_t)S);
    // Second pass, the files in parallel (worker threads, each with its own file): a worker
    // reads a file, sorts its entries into the file's own rows (stable: file order inside a
    // row) and uploads them to their place; out-degrees are counted on the device afterwards.
    std::vector<int64_t> rp((size_t)N + 1, 0);
    const std::vector<std::string> syn_names = {"output_neuron_idx", "input_block_idx", "input_neuron_idx",
                                                "input_channel_offset", "weight"};
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int workers = (int)std::min<size_t>(F, std::min(8u, hw));
    std::atomic<size_t> next_file{0};
    std::atomic<int> wstatus{rc};
    std::mutex err_mu;
    std::string werr;
    std::vector<int64_t> wmax_in((size_t)workers, 0);
    auto report = [&](int code, const std::string& msg) {
        std::lock_guard<std::mutex> lk(err_mu);
        if (wstatus.load() == DTB_OK) { werr = msg; wstatus.store(code); }
    };
    auto work = [&](int w) {
        if (cudaSetDevice(device) != cudaSuccess) { report(DTB_ERR_CUDA, "cudaSetDevice in a loader thread"); return; }
        char msg[256];
        for (;;) {
            if (wstatus.load() != DTB_OK) return;
            const size_t i = next_file.fetch_add(1);
            if (i >= F) return;
            std::map<std::string, NpyArray> m;
            std::string err;
            if (!npz_read(paths[i], m, err, &syn_names)) { report(DTB_ERR_FORMAT, err); return; }
            for (auto& nm : syn_names)
                if (!m.count(nm)) {
                    std::snprintf(msg, sizeof(msg), "block_%zu.npz: missing %s", i, nm.c_str());
                    report(DTB_ERR_FORMAT, msg);
                    return;
                }
            const NpyArray &on = m["output_neuron_idx"], &ib = m["input_block_idx"], &in = m["input_neuron_idx"],
                           &ic = m["input_channel_offset"], &wt = m["weight"];
            const int64_t E = on.count();
            if (E != syn[i + 1] - syn[i] || ib.count() != E || in.count() != E || ic.count() != E || wt.count() != 2 * E) {
                std::snprintf(msg, sizeof(msg), "block_%zu.npz: inconsistent synapse array lengths", i);
                report(DTB_ERR_FORMAT, msg);
                return;
            }
            if (on.descr != "<u4" || in.descr != "<u4" || ib.descr != "<i2" || ic.descr != "|u1" || wt.descr != "<f4") {
                std::snprintf(msg, sizeof(msg), "block_%zu.npz: unexpected synapse dtypes", i);
                report(DTB_ERR_FORMAT, msg);
                return;
            }
            const uint32_t* onp = reinterpret_cast<const uint32_t*>(on.data.data());
            const int16_t* ibp = reinterpret_cast<const int16_t*>(ib.data.data());
            const uint32_t* inp = reinterpret_cast<const uint32_t*>(in.data.data());
            const uint8_t* icp = reinterpret_cast<const uint8_t*>(ic.data.data());
            const float* wtp = reinterpret_cast<const float*>(wt.data.data());
            // stable counting sort of this file's entries into its rows (file order inside a row)
            const int64_t n_i = bases[i + 1] - bases[i];
            std::vector<int64_t> cur((size_t)n_i + 1, 0);
            for (int64_t e = 0; e < E; ++e) {
                if ((int64_t)onp[e] >= n_i) {
                    std::snprintf(msg, sizeof(msg), "block_%zu.npz: neuron index out of range", i);
                    report(DTB_ERR_FORMAT, msg);
                    return;
                }
                cur[(size_t)onp[e] + 1]++;
            }
            for (int64_t r = 0; r < n_i; ++r) {
                wmax_in[(size_t)w] = std::max<int64_t>(wmax_in[(size_t)w], cur[(size_t)r + 1]);
                cur[(size_t)r + 1] += cur[(size_t)r];
                rp[(size_t)(bases[i] + r + 1)] = syn[i] + cur[(size_t)r + 1];
            }
            std::vector<uint32_t> col((size_t)E);
            std::vector<float2> val((size_t)E);
            for (int64_t e = 0; e < E; ++e) {
                const int64_t sb = (int64_t)i + ibp[e];
                const bool ok = sb >= 0 && sb < (int64_t)F && bases[(size_t)sb] + inp[e] < bases[(size_t)sb + 1] &&
                                (icp[e] == 0 || icp[e] == 2);
                if (!ok) {
                    std::snprintf(msg, sizeof(msg), "block_%zu.npz: synapse %lld: %s", i, (long long)e,
                                  (sb < 0 || sb >= (int64_t)F) ? "input_block_idx out of range"
                                  : (icp[e] != 0 && icp[e] != 2) ? "input_channel_offset must be 0 or 2"
                                                                 : "neuron index out of range");
                    report(DTB_ERR_FORMAT, msg);
                    return;
                }
                const int64_t pr = bases[(size_t)sb] + inp[e];
                const int64_t d = cur[onp[e]]++;
                col[(size_t)d] = (uint32_t)pr | (icp[e] ? kKindBit : 0u);
                val[(size_t)d] = make_float2(wtp[2 * e], wtp[2 * e + 1]);
            }
            if (E > 0) {
                cudaError_t e1 = cudaMemcpy(pcol + syn[i], col.data(), 4 * (size_t)E, cudaMemcpyHostToDevice);
                if (e1 == cudaSuccess) e1 = cudaMemcpy(pw + syn[i], val.data(), 8 * (size_t)E, cudaMemcpyHostToDevice);
                if (e1 != cudaSuccess) { report(DTB_ERR_CUDA, std::string("synapse upload: ") + cudaGetErrorString(e1)); return; }
            }
        }
    };
    if (rc == DTB_OK) {
        std::vector<std::thread> pool;
        for (int w = 1; w < workers; ++w) pool.emplace_back(work, w);
        work(0);
        for (auto& t : pool) t.join();
        cudaSetDevice(device);
        if (wstatus.load() != DTB_OK) rc = fail(wstatus.load(), "%s", werr.c_str());
        for (int64_t v : wmax_in) b->max_in = std::max(b->max_in, v);
    }
    if (rc == DTB_OK) {
        cudaError_t e1 = cudaMemcpy(prow, rp.data(), sizeof(int64_t) * rp.size(), cudaMemcpyHostToDevice);
        if (e1 != cudaSuccess) rc = fail(DTB_ERR_CUDA, "row pointer upload: %s", cudaGetErrorString(e1));
        b->ds.prow = prow; b->ds.pcol = pcol; b->ds.pw = pw;
        b->has_pull = (rc == DTB_OK);
    }
    if (rc == DTB_OK && build_push) {
        rc = dalloc(b, &counts, (size_t)N + 1);
        if (rc == DTB_OK) {
            cudaError_t e1 = cudaMemsetAsync(counts, 0, sizeof(uint32_t) * ((size_t)N + 1), b->stream);
            if (e1 == cudaSuccess && S > 0) {
                k_count_outdeg<<<grid_for(S, 256), 256, 0, b->stream>>>(S, pcol, counts);
                e1 = cudaGetLastError();
            }
            if (e1 != cudaSuccess) rc = fail(DTB_ERR_CUDA, "out-degree count: %s", cudaGetErrorString(e1));
        }
        if (rc == DTB_OK) rc = build_push_device(b, counts, b->max_in <= 65535);
    }
    if (rc == DTB_OK) rc = finish_create(b);
    if (rc != DTB_OK) { destroy_block(b); return rc; }
    *out = b;
    return DTB_OK;
}

int dtb_block_destroy(dtb_block* b)
{
    destroy_block(b);
    return DTB_OK;
}

int dtb_block_set_stream(dtb_block* b, void* stream)
{
    if (!b) return fail(DTB_ERR_ARG, "null handle");
    DeviceGuard g(b->device);
    if (b->stream != (cudaStream_t)stream) {
        for (auto& ge : b->graph) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
    }
    b->stream = (cudaStream_t)stream;
    return DTB_OK;
}

int dtb_block_synchronize(dtb_block* b)
{
    if (!b) return fail(DTB_ERR_ARG, "null handle");
    DeviceGuard g(b->device);
    CK(cudaStreamSynchronize(b->stream));
    uint32_t err = 0;
    CK(cudaMemcpy(&err, &b->ds.ctl->err, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        CK(cudaMemset(&b->ds.ctl->err, 0, sizeof(uint32_t)));
        if (err & kErrGeneralSkipped)
            return fail(DTB_ERR_STATE, "internal: an update ran without the I_syn override or gamma g_ui it needed");
        if (err & (kErrStageTimeout | kErrStageDrain))
            return fail(DTB_ERR_CUDA, "a staged state copy did not complete in time (the update loaded that state "
                        "from global memory instead)");
    }
    return DTB_OK;
}

int dtb_block_get_info(const dtb_block* b, dtb_block_info* info)
{
    if (!b || !info) return fail(DTB_ERR_ARG, "null argument");
    info->n_neurons = b->N;
    info->n_synapses = b->S;
    info->n_subblocks = b->n_sub;
    info->n_classes = b->n_classes;
    info->has_pull = b->has_pull;
    info->has_push = b->has_push;
    info->device_bytes = b->dev_bytes;
    info->max_outdegree = b->max_out;
    info->max_indegree = b->max_in;
    info->kernel_launches = b->launches;
    return DTB_OK;
}

int dtb_block_run(dtb_block* b, int n_steps, float noise_rate, int isolated, int mode, float* sum_out,
                  float* mean_out, uint32_t* nact_out, int where)
{
    if (!b) return fail(DTB_ERR_ARG, "null handle");
    if (n_steps < 0) return fail(DTB_ERR_ARG, "n_steps < 0");
    if (mode < DTB_MODE_AUTO || mode > DTB_MODE_PULL) return fail(DTB_ERR_ARG, "bad mode %d", mode);
    if (where != DTB_HOST && where != DTB_DEVICE) return fail(DTB_ERR_ARG, "bad where");
    if (!b->has_pull && !b->has_push) return fail(DTB_ERR_STATE, "network has no synapse tables");
    RET(check_src_steps(b, n_steps));
    DeviceGuard g(b->device);
    b->override_pending = false;
    int64_t done = 0;
    while (done < n_steps) {
        const int m = choose_mode(b, mode);
        const int mm = resolve_method(b, m);
        RET(ensure_method(b, mm));
        const uint32_t cap = b->stats_cap;
        int n = (int)std::min<int64_t>(n_steps - done, (int64_t)std::min<uint32_t>(cap, (uint32_t)b->chunk));
        RET(set_run_params(b, noise_rate, isolated));
        RET(enqueue_chunk(b, n, mm));
        b->steps += (uint64_t)n;
        std::vector<uint32_t> nact;
        const bool want_nact = (mode == DTB_MODE_AUTO) || (m == DTB_MODE_PULL && b->has_qpos && b->pull_method == 0);
        RET(emit_stats(b, n, done, sum_out, mean_out, nact_out, where, want_nact ? &nact : nullptr));
        if (want_nact && n > 0) {
            double tot = 0.0;
            for (uint32_t v : nact) tot += v;
            b->last_frac = tot / ((double)n * (double)std::max<int64_t>(1, b->N));
        }
        done += n;
    }
    return DTB_OK;
}

int dtb_block_time_kernels(dtb_block* b, int n_steps, float noise_rate, int isolated, int mode, float* out_ms)
{
    if (!b || !out_ms || n_steps <= 0) return fail(DTB_ERR_ARG, "bad argument");
    RET(check_src_steps(b, n_steps));
    DeviceGuard g(b->device);
    const int m = resolve_method(b, choose_mode(b, mode));
    RET(ensure_method(b, m));
    RET(ensure_stats(b, (uint32_t)n_steps));
    RET(set_run_params(b, noise_rate, isolated));
    unsigned long long ev0 = 0, ev1 = 0;
    RET(sum_events(b));
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemcpy(&ev0, &b->ds.ctl->events, 8, cudaMemcpyDeviceToHost));
    const int n_ev = 4 * n_steps + 4;
    std::vector<cudaEvent_t> ev((size_t)n_ev);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    std::vector<int> kind;  // 0 update kernel, 1 propagation kernel, 2 closing fold (not averaged)
    int k = 0;
    auto rec = [&](int i) { return cudaEventRecord(ev[(size_t)i], b->stream); };
    int rc = DTB_OK;
    int done_steps = 0;
    if (m != kModeBinned) rc = flush_bins(b);
    if (rc != DTB_OK) {
        for (auto& x : ev) cudaEventDestroy(x);
        return rc;
    }
    if (m == kModeBinned) {
        for (int st = 0; st < n_steps && rc == DTB_OK && k + 6 <= n_ev; ++st) {
            rec(k); rc = launch_update(b, b->ds, kGatherBins, false); rec(k + 1);
            kind.push_back(0); k += 2;
            if (rc != DTB_OK) break;
            rec(k); rc = launch_bin_scatter(b, b->ds); rec(k + 1); kind.push_back(1); k += 2;
            done_steps++;
        }
        if (done_steps) b->bins_pending = true;
    } else if (m == DTB_MODE_PUSH || m == kModeSlots || m == kModeMasks) {
        const bool ord = m != DTB_MODE_PUSH;
        const int g = m == kModeSlots ? kGatherSlots : kGatherMasks;
        const int how = m == kModeSlots ? kScatterSlots : (m == kModeMasks ? kScatterMasks : kScatterJ);
        for (int st = 0; st < n_steps && rc == DTB_OK && k + 6 <= n_ev; ++st) {
            rec(k); rc = launch_update(b, b->ds, (ord && st > 0) ? g : 0, false); rec(k + 1);
            kind.push_back(0); k += 2;
            if (rc != DTB_OK) break;
            rec(k); rc = launch_scatter(b, b->ds, how); rec(k + 1); kind.push_back(1); k += 2;
            done_steps++;
        }
        if (ord && rc == DTB_OK) {
            rec(k); rc = launch_gather_only(b, b->ds, g); rec(k + 1); kind.push_back(2); k += 2;
        }
    } else {
        const int g = m == kModeStream ? kGatherStream : kGatherRows;
        rec(k); rc = launch_update(b, b->ds, 0, false); rec(k + 1); kind.push_back(0); k += 2;
        for (int st = 1; st < n_steps && rc == DTB_OK && k + 4 <= n_ev; ++st) {
            rec(k); rc = launch_update(b, b->ds, g, false); rec(k + 1); kind.push_back(0); k += 2;
        }
        if (rc == DTB_OK) { rec(k); rc = launch_gather_only(b, b->ds, g); rec(k + 1); kind.push_back(1); k += 2; }
        done_steps = (int)kind.size() - 1;
    }
    b->steps += (uint64_t)done_steps;
    cudaError_t e = cudaStreamSynchronize(b->stream);
    double sum[3] = {0.0, 0.0, 0.0};
    int cnt[3] = {0, 0, 0};
    for (size_t i = 0; i < kind.size() && e == cudaSuccess; ++i) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
        sum[kind[i]] += ms;
        cnt[kind[i]]++;
    }
    float total = 0.0f;
    if (e == cudaSuccess && k >= 2) e = cudaEventElapsedTime(&total, ev[0], ev[(size_t)k - 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (rc != DTB_OK) return rc;
    if (e != cudaSuccess) return fail(DTB_ERR_CUDA, "event timing: %s", cudaGetErrorString(e));
    RET(sum_events(b));
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemcpy(&ev1, &b->ds.ctl->events, 8, cudaMemcpyDeviceToHost));
    out_ms[0] = cnt[0] ? (float)(sum[0] / cnt[0]) : 0.0f;
    out_ms[1] = cnt[1] ? (float)(sum[1] / cnt[1]) : 0.0f;
    out_ms[2] = done_steps ? total / (float)done_steps : 0.0f;
    out_ms[3] = done_steps ? (float)((double)(ev1 - ev0) / done_steps) : 0.0f;
    return DTB_OK;
}


int dtb_block_set_tuning(dtb_block* b, int key, int64_t value)
{
    if (!b) return fail(DTB_ERR_ARG, "null handle");
    switch (key) {
    case DTB_TUNE_SCATTER_WORDS:
        if (value < 1 || value > 32) return fail(DTB_ERR_ARG, "scatter words per warp must be 1..32");
        b->scatter_wpw = (int)value;
        break;
    case DTB_TUNE_SCATTER_VARIANT:
        if (value < 0 || value > 1) return fail(DTB_ERR_ARG, "scatter variant must be 0 or 1");
        b->scatter_variant = (int)value;
        break;
    case DTB_TUNE_J_CACHE:
        if (value < 0 || value > 1) return fail(DTB_ERR_ARG, "J cache policy must be 0 (stream) or 1 (keep)");
        b->ds.j_keep = (int)value;
        break;
    case DTB_TUNE_PULL_METHOD:
        if (value < 0 || value > 4)
            return fail(DTB_ERR_ARG, "pull method must be 0 (auto), 1 (rows), 2 (slots), 3 (masks) or 4 (streamed)");
        if (value >= 2 && !b->has_qpos) return fail(DTB_ERR_STATE, "ordered push needs the push CSR with pull-row positions");
        if (value == 3 && !masks_possible(b))
            return fail(DTB_ERR_STATE, "position masks hold in-degrees up to %d (max in-degree %lld)", 32 * kMaskWords,
                        (long long)b->max_in);
        b->pull_method = (int)value;
        break;
    case DTB_TUNE_CHUNK:
        if (value < 1 || value > 4096) return fail(DTB_ERR_ARG, "chunk must be 1..4096");
        b->chunk = (int)value;
        break;
    case DTB_TUNE_PULL_THRESHOLD_PPM:
        if (value < 0) return fail(DTB_ERR_ARG, "threshold must be >= 0");
        b->pull_threshold = (double)value * 1e-6;
        break;
    case DTB_TUNE_USE_GRAPHS: b->use_graphs = value != 0; break;
    case DTB_TUNE_STEP_VARIANT:
        if (value < 0 || value > 4) return fail(DTB_ERR_ARG, "step variant must be 0..4");
        b->step_variant = (int)value;
        break;
    case DTB_TUNE_SCATTER_REVERSE:
        if (value < 0 || value > 1) return fail(DTB_ERR_ARG, "scatter order must be 0 (forward) or 1 (reverse)");
        b->ds.rev_scatter = (int)value;
        break;
    case DTB_TUNE_STAGE_WAIT_LIMIT:
        if (value < 0 || value > 0x7fffffffLL) return fail(DTB_ERR_ARG, "stage wait limit must be 0..2^31-1");
        b->ds.stage_wait_limit = (uint32_t)value;
        break;
    case DTB_TUNE_PUSH_METHOD:
        if (value < 0 || value > 2) return fail(DTB_ERR_ARG, "push method must be 0 (auto), 1 (atomics) or 2 (binned)");
        if (value == 2 && !bins_possible(b)) return fail(DTB_ERR_STATE, "binned push not possible for this network");
        if (value == 2) { b->bins_failed = false; RET(ensure_bins(b)); }
        b->push_method = (int)value;
        break;
    case DTB_TUNE_BIN_WORDS:
        if (value < 1 || value > kBinMaxWords) return fail(DTB_ERR_ARG, "bin scatter words per round must be 1..%d", kBinMaxWords);
        b->bin_words = (int)value;
        break;
    case DTB_TUNE_BIN_CAPACITY:
    case DTB_TUNE_BIN_SHIFT: {
        if (key == DTB_TUNE_BIN_CAPACITY && (value < 1 || value > 1024))
            return fail(DTB_ERR_ARG, "bin capacity must be 1..1024 entries per neuron");
        if (key == DTB_TUNE_BIN_SHIFT && value != 0 && (value < kBinMinShift || value > kBinMaxShift))
            return fail(DTB_ERR_ARG, "bin shift must be 0 (auto) or %d..%d", kBinMinShift, kBinMaxShift);
        RET(flush_bins(b));   // the events waiting in the old bins go to J first
        CK(cudaStreamSynchronize(b->stream));
        free_bins(b);
        b->bins_failed = false;
        if (key == DTB_TUNE_BIN_CAPACITY) b->bin_cap_per_neuron = (int)value;
        else b->bin_shift_req = (int)value;
        break;
    }
    default: return fail(DTB_ERR_ARG, "unknown tuning key %d", key);
    }
    drop_graphs(b);
    return DTB_OK;
}

int dtb_block_get_tuning(dtb_block* b, int key, int64_t* value)
{
    if (!b || !value) return fail(DTB_ERR_ARG, "null argument");
    switch (key) {
    case DTB_TUNE_SCATTER_WORDS: *value = b->scatter_wpw; break;
    case DTB_TUNE_CHUNK: *value = b->chunk; break;
    case DTB_TUNE_PULL_THRESHOLD_PPM: *value = (int64_t)std::llround(b->pull_threshold * 1e6); break;
    case DTB_TUNE_USE_GRAPHS: *value = b->use_graphs ? 1 : 0; break;
    case DTB_TUNE_STEP_VARIANT: *value = b->step_variant; break;
    case DTB_TUNE_PULL_METHOD: *value = b->pull_method; break;
    case DTB_TUNE_J_CACHE: *value = b->ds.j_keep; break;
    case DTB_TUNE_SCATTER_VARIANT: *value = b->scatter_variant; break;
    case DTB_TUNE_PUSH_METHOD: *value = b->push_method; break;
    case DTB_TUNE_STAGE_WAIT_LIMIT: *value = b->ds.stage_wait_limit; break;
    case DTB_TUNE_SCATTER_REVERSE: *value = b->ds.rev_scatter; break;
    case DTB_TUNE_BIN_WORDS: *value = b->bin_words; break;
    case DTB_TUNE_BIN_CAPACITY: *value = b->bin_cap_per_neuron; break;
    case DTB_TUNE_BIN_SHIFT: *value = b->ds.bin_cnt ? b->ds.bin_shift : bin_shift_for(b); break;
    default: return fail(DTB_ERR_ARG, "unknown tuning key %d", key);
    }
    return DTB_OK;
}

int dtb_block_autotune(dtb_block* b, int n_steps, float noise_rate, float* report)
{
    if (!b || n_steps < 2) return fail(DTB_ERR_ARG, "bad argument");
    float best_ms = 1e30f, push_ms = 0.0f, pull_ms = 0.0f, ev = 0.0f;
    int best_w = b->scatter_wpw;
    const int pm0 = b->push_method;
    if (b->has_push) b->push_method = 1;   // atomic push first
    {   // register budget of the update kernel
        const int mode = b->has_push ? DTB_MODE_PUSH : DTB_MODE_PULL;
        float best_u = 1e30f;
        int best_v = 0;
        for (int v = 0; v < 5; ++v) {
            if (v >= 2 && !staged_layout(b->ds)) continue;
            b->step_variant = v;
            float o[4];
            RET(dtb_block_time_kernels(b, n_steps, noise_rate, 0, mode, o));
            if (o[0] < best_u) { best_u = o[0]; best_v = v; }
        }
        b->step_variant = best_v;
    }
    if (b->has_push) {
        const int cand[6] = {1, 2, 4, 8, 16, 32};
        int best_sv = b->scatter_variant;
        for (int sv = 0; sv < 2; ++sv)
            for (int w : cand) {
                b->scatter_wpw = w;
                b->scatter_variant = sv;
                float o[4];
                RET(dtb_block_time_kernels(b, n_steps, noise_rate, 0, DTB_MODE_PUSH, o));
                if (o[2] < best_ms) { best_ms = o[2]; best_w = w; best_sv = sv; ev = o[3]; }
            }
        b->scatter_wpw = best_w;
        b->scatter_variant = best_sv;
        {   // J lines kept in L2 for the scatter vs streamed, scatter order forward vs reverse
            const int keep0 = b->ds.j_keep, rev0 = b->ds.rev_scatter;
            int bk = keep0, br = rev0;
            for (int keep = 0; keep < 2; ++keep)
                for (int rev = 0; rev < 2; ++rev) {
                    if (keep == keep0 && rev == rev0) continue;
                    b->ds.j_keep = keep;
                    b->ds.rev_scatter = rev;
                    float o[4];
                    RET(dtb_block_time_kernels(b, n_steps, noise_rate, 0, DTB_MODE_PUSH, o));
                    if (o[2] < best_ms) { best_ms = o[2]; ev = o[3]; bk = keep; br = rev; }
                }
            b->ds.j_keep = bk;
            b->ds.rev_scatter = br;
        }
        // binned push: update variant (registers, staging) x scatter round size, kept when faster
        b->push_method = pm0;
        if (pm0 != 1 && bins_possible(b) && ensure_bins(b) == DTB_OK) {
            const int atomic_v = b->step_variant, atomic_words = b->bin_words;
            float best_b = 1e30f, ev_b = 0.0f;
            int bv = 0, bw = atomic_words;
            b->push_method = 2;
            const bool stageable = staged_layout(b->ds) && b->ds.bin_shift == kBinMinShift;
            for (int v = 0; v < 4; ++v)
                for (int w : {64, 128, 256}) {
                    if (v >= 2 && !stageable) continue;
                    b->step_variant = v;
                    b->bin_words = w;
                    float o[4];
                    RET(dtb_block_time_kernels(b, n_steps, noise_rate, 0, DTB_MODE_PUSH, o));
                    if (o[2] < best_b) { best_b = o[2]; bv = v; bw = w; ev_b = o[3]; }
                }
            if (best_b < best_ms) {
                best_ms = best_b; ev = ev_b;
                b->step_variant = bv; b->bin_words = bw;
            } else {
                b->push_method = 1;
                b->step_variant = atomic_v; b->bin_words = atomic_words;
            }
        } else if (pm0 == 0) {
            b->push_method = 1;
        }
        push_ms = best_ms;
    }
    if (b->has_pull) {
        float o[4];
        RET(dtb_block_time_kernels(b, n_steps, noise_rate, 0, DTB_MODE_PULL, o));
        pull_ms = o[2];
        if (!b->has_push) ev = o[3];
    }
    // activity fraction of the tuned steps; push cost grows with it, pull cost hardly does
    const double deg = b->N ? (double)b->S / (double)b->N : 1.0;
    const double f = deg > 0 ? (double)ev / deg / (double)std::max<int64_t>(1, b->N) : 0.0;
    if (b->has_push && b->has_pull && push_ms > 0.0f) b->pull_threshold = f * (double)pull_ms / (double)push_ms;
    drop_graphs(b);
    if (report) {
        report[0] = (float)best_w; report[1] = push_ms; report[2] = pull_ms; report[3] = (float)f;
        report[4] = (float)b->pull_threshold; report[5] = (float)b->step_variant;
    }
    return DTB_OK;
}

int dtb_block_step_forced(dtb_block* b, float noise_rate, int isolated, int mode, const uint8_t* forced_active,
                          const uint8_t* forced_new_active, float* sum_out, float* mean_out, int where)
{
    if (!b) return fail(DTB_ERR_ARG, "null handle");
    DeviceGuard g(b->device);
    b->override_pending = false;
    DevState s = b->ds;
    const uint8_t* src[2] = {forced_active, forced_new_active};
    for (int k = 0; k < 2; ++k) {
        if (!src[k]) continue;
        if (!b->d_forced[k]) RET(dalloc(b, &b->d_forced[k], (size_t)s.n_words));
        if (!b->d_u8) RET(dalloc(b, &b->d_u8, (size_t)b->N));
        if (where == DTB_HOST) CK(cudaMemcpyAsync(b->d_u8, src[k], (size_t)b->N, cudaMemcpyHostToDevice, b->stream));
        else CK(cudaMemcpyAsync(b->d_u8, src[k], (size_t)b->N, cudaMemcpyDeviceToDevice, b->stream));
        k_u8_to_bits<<<grid_for(s.n_words, 256), 256, 0, b->stream>>>(b->d_u8, b->N, b->d_forced[k], s.n_words);
        CK(cudaGetLastError());
    }
    s.forced_active = forced_active ? b->d_forced[0] : b->ds.forced_active;   // input neurons stay forced
    s.forced_mask = forced_active ? nullptr : b->ds.forced_mask;
    s.forced_new = forced_new_active ? b->d_forced[1] : nullptr;
    RET(check_src_steps(b, 1));
    RET(set_run_params(b, noise_rate, isolated));
    const int m = choose_mode(b, mode);
    const int mm = m == DTB_MODE_PUSH ? resolve_method(b, m) : m;
    if (mm == kModeBinned) {
        s.bin_idx = b->ds.bin_idx; s.bin_w = b->ds.bin_w; s.bin_cnt = b->ds.bin_cnt;
        s.n_bins = b->ds.n_bins; s.bin_cap = b->ds.bin_cap; s.bin_shift = b->ds.bin_shift;
        RET(launch_update(b, s, kGatherBins, true));
        RET(launch_bin_scatter(b, s));
        b->bins_pending = true;
    } else {
        RET(flush_bins(b));
        RET(launch_update(b, s, 0, true));
        if (m == DTB_MODE_PUSH) RET(launch_scatter(b, s));
        else RET(launch_gather_only(b, s));
    }
    b->steps += 1;
    RET(emit_stats(b, 1, 0, sum_out, mean_out, nullptr, where, nullptr));
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

int dtb_block_get(dtb_block* b, int field, void* dst, int where)
{
    if (!b || !dst) return fail(DTB_ERR_ARG, "null argument");
    if (where != DTB_HOST && where != DTB_DEVICE) return fail(DTB_ERR_ARG, "bad where");
    DeviceGuard g(b->device);
    const DevState& s = b->ds;
    const int64_t N = b->N;
    auto export_buf = [&](void** p) -> int {
        if (where == DTB_DEVICE) { *p = dst; return DTB_OK; }
        if (!b->d_export) RET(dalloc(b, &b->d_export, (size_t)N * 4));
        *p = b->d_export;
        return DTB_OK;
    };
    switch (field) {
    case DTB_FIELD_V: return copy_out(b, dst, s.V, sizeof(float) * N, where);
    case DTB_FIELD_T_LAST: return copy_out(b, dst, s.tlast, sizeof(float) * N, where);
    case DTB_FIELD_J: {
        RET(flush_bins(b));
        void* p; RET(export_buf(&p));
        k_export_J<<<grid_for(N, 256), 256, 0, b->stream>>>(s, (float*)p);
        CK(cudaGetLastError());
        if (where == DTB_HOST) return copy_out(b, dst, p, sizeof(float) * 4 * N, where);
        return DTB_OK;
    }
    case DTB_FIELD_I_UI:
    case DTB_FIELD_I_SYN: {
        if (b->override_pending) {
            if (field == DTB_FIELD_I_SYN) return copy_out(b, dst, s.isyn_override, sizeof(float) * N, where);
            return copy_out(b, dst, b->d_iui_override, sizeof(float) * 4 * N, where);
        }
        RET(flush_bins(b));
        void* p; RET(export_buf(&p));
        if (field == DTB_FIELD_I_UI) k_export_current<<<grid_for(N, 256), 256, 0, b->stream>>>(s, (float*)p, nullptr);
        else k_export_current<<<grid_for(N, 256), 256, 0, b->stream>>>(s, nullptr, (float*)p);
        CK(cudaGetLastError());
        if (where == DTB_HOST) return copy_out(b, dst, p, sizeof(float) * (field == DTB_FIELD_I_UI ? 4 : 1) * N, where);
        return DTB_OK;
    }
    case DTB_FIELD_ACTIVE:
    case DTB_FIELD_NEW_ACTIVE: {
        const uint32_t* bits = field == DTB_FIELD_ACTIVE ? s.abits : s.bits[(b->steps + 1) & 1];
        void* p; RET(export_buf(&p));
        k_bits_to_u8<<<grid_for(N, 256), 256, 0, b->stream>>>(bits, N, (uint8_t*)p);
        CK(cudaGetLastError());
        if (where == DTB_HOST) return copy_out(b, dst, p, (size_t)N, where);
        return DTB_OK;
    }
    case DTB_FIELD_T: return copy_out(b, dst, &s.ctl->t, sizeof(float), where);
    case DTB_FIELD_STEP: {
        if (where == DTB_HOST) { std::memcpy(dst, &b->steps, sizeof(uint64_t)); return DTB_OK; }
        return copy_out(b, dst, &s.ctl->steps_done, sizeof(uint64_t), where);
    }
    case DTB_FIELD_EVENTS:
        RET(sum_events(b));
        return copy_out(b, dst, &s.ctl->events, sizeof(unsigned long long), where);
    case DTB_FIELD_WINDOW_SPIKES:
        return copy_out(b, dst, s.win_spk, sizeof(unsigned long long) * (size_t)b->n_sub, where);
    case DTB_FIELD_G_FACTOR:
        if (!s.gnrn) return fail(DTB_ERR_STATE, "no gamma-distributed g_ui");
        return copy_out(b, dst, s.gnrn, sizeof(float4) * N, where);
    case DTB_FIELD_SUB_COUNT:
        if (where == DTB_HOST) { if (b->n_sub) std::memcpy(dst, b->sub_count.data(), sizeof(uint32_t) * b->n_sub); return DTB_OK; }
        return copy_out(b, dst, s.sub_count, sizeof(uint32_t) * b->n_sub, where);
    default: return fail(DTB_ERR_ARG, "unknown field %d", field);
    }
}

int dtb_block_get_csr(dtb_block* b, int which, int64_t* rowptr, uint32_t* index, float* weight, int where)
{
    if (!b || (which != 0 && which != 1)) return fail(DTB_ERR_ARG, "bad argument");
    if ((which == 0 && !b->has_pull) || (which == 1 && !b->has_push)) return fail(DTB_ERR_STATE, "CSR not built");
    DeviceGuard g(b->device);
    const int64_t* r = which ? b->ds.qrow : b->ds.prow;
    const uint32_t* c = which ? b->ds.qcol : b->ds.pcol;
    const float2* w = which ? b->ds.qw : b->ds.pw;
    if (rowptr) RET(copy_out(b, rowptr, r, sizeof(int64_t) * (size_t)(b->N + 1), where));
    if (index) RET(copy_out(b, index, c, sizeof(uint32_t) * (size_t)b->S, where));
    if (weight) RET(copy_out(b, weight, w, sizeof(float2) * (size_t)b->S, where));
    return DTB_OK;
}

int dtb_block_get_csr_entries(dtb_block* b, int which, int64_t first, int64_t count, uint32_t* index, float* weight,
                              int where)
{
    if (!b || (which != 0 && which != 1)) return fail(DTB_ERR_ARG, "bad argument");
    if ((which == 0 && !b->has_pull) || (which == 1 && !b->has_push)) return fail(DTB_ERR_STATE, "CSR not built");
    if (first < 0 || count < 0 || first > b->S || count > b->S - first)
        return fail(DTB_ERR_ARG, "entries [%lld, %lld) outside [0, %lld)", (long long)first, (long long)(first + count),
                    (long long)b->S);
    DeviceGuard g(b->device);
    const uint32_t* c = which ? b->ds.qcol : b->ds.pcol;
    const float2* w = which ? b->ds.qw : b->ds.pw;
    if (index && count) RET(copy_out(b, index, c + first, sizeof(uint32_t) * (size_t)count, where));
    if (weight && count) RET(copy_out(b, weight, w + first, sizeof(float2) * (size_t)count, where));
    return DTB_OK;
}

int dtb_block_set(dtb_block* b, int field, const void* src, int where)
{
    if (!b || !src) return fail(DTB_ERR_ARG, "null argument");
    DeviceGuard g(b->device);
    const DevState& s = b->ds;
    const int64_t N = b->N;
    const cudaMemcpyKind k = where == DTB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    switch (field) {
    case DTB_FIELD_V: CK(cudaMemcpyAsync(s.V, src, sizeof(float) * N, k, b->stream)); break;
    case DTB_FIELD_T_LAST: CK(cudaMemcpyAsync(s.tlast, src, sizeof(float) * N, k, b->stream)); break;
    case DTB_FIELD_J: {
        RET(discard_bins(b));
        if (!b->d_export) RET(dalloc(b, &b->d_export, (size_t)N * 4));
        CK(cudaMemcpyAsync(b->d_export, src, sizeof(float) * 4 * N, k, b->stream));
        k_J_from_planar<<<grid_for(N, 256), 256, 0, b->stream>>>(s, b->d_export);
        CK(cudaGetLastError());
        break;
    }
    case DTB_FIELD_T: CK(cudaMemcpyAsync(&s.ctl->t, src, sizeof(float), k, b->stream)); break;
    case DTB_FIELD_WINDOW_SPIKES:
        CK(cudaMemcpyAsync(s.win_spk, src, sizeof(unsigned long long) * (size_t)b->n_sub, k, b->stream));
        break;
    case DTB_FIELD_STEP: {
        uint64_t v;
        if (where == DTB_HOST) std::memcpy(&v, src, 8);
        else CK(cudaMemcpy(&v, src, 8, cudaMemcpyDeviceToHost));
        b->steps = v;
        CK(cudaMemcpyAsync(&s.ctl->steps_done, &b->steps, sizeof(uint64_t), cudaMemcpyHostToDevice, b->stream));
        break;
    }
    default: return fail(DTB_ERR_ARG, "field %d cannot be set", field);
    }
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

// The reference computes I_syn at the end of a step (models/block.py:140;
// cuda/src/block.cpp update_I_synaptic_gpu) and the next membrane update uses
// that stored value, so a parameter change takes effect on I_syn one step
// later.  The fused kernels recompute I_syn at the update: before parameters
// change, the current I_syn (old parameters) is kept for the next update.
static int keep_current_isyn(dtb_block* b)
{
    DevState& s = b->ds;
    if (b->override_pending || b->N <= 0) return DTB_OK;
    RET(flush_bins(b));
    if (!b->d_iui_override) RET(dalloc(b, &b->d_iui_override, (size_t)b->N * 4));
    k_export_current<<<grid_for(b->N, 256), 256, 0, b->stream>>>(s, b->d_iui_override, s.isyn_override);
    CK(cudaGetLastError());
    const uint32_t one = 1u;
    CK(cudaMemcpyAsync(&s.ctl->use_isyn_override, &one, sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    b->override_pending = true;
    b->override_live = true;
    return DTB_OK;
}

int dtb_block_update_property(dtb_block* b, const float* property, const float* decay)
{
    if (!b || !property) return fail(DTB_ERR_ARG, "null argument");
    RET(check_property(b->N, property, "dtb_block_update_property"));
    DeviceGuard g(b->device);
    DevState& s = b->ds;
    RET(keep_current_isyn(b));   // keep the current synaptic current (computed with the old parameters)
    std::vector<uint32_t> cls;
    RET(build_classes(b, b->N, property, decay, cls));
    RET(upload_class_tables(b));
    CK(cudaMemcpy(const_cast<uint32_t*>(s.cls), cls.data(), sizeof(uint32_t) * (size_t)b->N, cudaMemcpyHostToDevice));
    RET(upload_tile_classes(b, cls));
    if (!s.st_spk) RET(ensure_stats(b, 256));
    if (b->bold_R == 0) RET(rebuild_groups(b, nullptr));
    b->class_prop_base.clear();
    s.gnrn = nullptr;   // the new matrix holds every neuron's g_ui: gamma factors no longer apply
    drop_graphs(b);     // captured graphs hold the update's form for the old gnrn
    for (auto& ge : b->graph) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
    b->override_pending = true;
    return DTB_OK;
}

// Re-derives the device parameters of every dirty class from its current row
// (decay again from tau when a tau column moved) and uploads the table.
static int rebuild_dirty_classes(dtb_block* b, const std::vector<char>& dirty,
                                 const std::vector<char>* tau_set = nullptr)
{
    for (int c = 0; c < b->n_classes; ++c) {
        if (!dirty[(size_t)c]) continue;
        auto& row = b->class_prop[(size_t)c];
        float dc[4] = {b->class_decay[(size_t)c][0], b->class_decay[(size_t)c][1], b->class_decay[(size_t)c][2],
                       b->class_decay[(size_t)c][3]};
        bool tau_changed = false;
        for (int k = 18; k < 22; ++k) tau_changed |= row[(size_t)k] != b->class_prop_base[(size_t)c][(size_t)k];
        if (tau_set) tau_changed |= (*tau_set)[(size_t)c] != 0;
        if (tau_changed) { default_decay(row.data(), b->dt, dc); b->class_decay[(size_t)c] = {dc[0], dc[1], dc[2], dc[3]}; }
        ParamClass p = make_class(row.data(), dc, b->dt);
        p.sub = b->classes[(size_t)c].sub;
        p.member = b->classes[(size_t)c].member;
        b->classes[(size_t)c] = p;
    }
    CK(cudaMemcpyAsync(const_cast<ParamClass*>(b->ds.pc), b->classes.data(), sizeof(ParamClass) * b->classes.size(),
                       cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

int dtb_block_scale_property_by_subblock(dtb_block* b, int n, const int32_t* sub, const int32_t* col, const float* value)
{
    if (!b || n < 0 || (n > 0 && (!sub || !col || !value))) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(b->device);
    for (int i = 0; i < n; ++i)
        if (col[i] < 0 || col[i] >= DTB_NPROP || col[i] == 3) return fail(DTB_ERR_ARG, "column %d cannot be scaled", col[i]);
    if (n > 0) RET(keep_current_isyn(b));
    if (b->class_prop_base.empty()) b->class_prop_base = b->class_prop;
    for (int i = 0; i < n; ++i) {
        if (col[i] < 0 || col[i] >= DTB_NPROP || col[i] == 3) return fail(DTB_ERR_ARG, "column %d cannot be scaled", col[i]);
    }
    // classes of every subblock (a subblock can span several classes)
    std::unordered_map<int32_t, std::vector<int32_t>> by_sub;
    for (int c = 0; c < b->n_classes; ++c) by_sub[b->classes[(size_t)c].sub].push_back(c);
    std::vector<char> dirty((size_t)b->n_classes, 0);
    for (int i = 0; i < n; ++i) {
        auto it = by_sub.find(sub[i]);
        if (it == by_sub.end()) continue;
        for (int32_t c : it->second) {
            auto& row = b->class_prop[(size_t)c];
            volatile float v = b->class_prop_base[(size_t)c][(size_t)col[i]] * value[i];
            row[(size_t)col[i]] = v;
            dirty[(size_t)c] = 1;
        }
    }
    return rebuild_dirty_classes(b, dirty);
}

int dtb_block_gamma_property_by_subblock(dtb_block* b, int n, const int32_t* sub, const int32_t* col,
                                         const float* alpha, const float* beta)
{
    if (!b || n < 0 || (n > 0 && (!sub || !col || !alpha || !beta))) return fail(DTB_ERR_ARG, "bad argument");
    if (n == 0) return DTB_OK;
    for (int i = 0; i < n; ++i) {
        if (!(alpha[i] >= 0.0f) || !(beta[i] > 0.0f)) return fail(DTB_ERR_ARG, "request %d: need alpha >= 0, beta > 0", i);
        const bool g_col = col[i] >= 10 && col[i] < 14;
        const bool delta = alpha[i] >= 1e6f;   // relative spread 1/sqrt(alpha) <= 1e-3
        if (col[i] < 0 || col[i] >= DTB_NPROP || col[i] == 1 || col[i] == 3)
            return fail(DTB_ERR_ARG, "column %d cannot be gamma-distributed", col[i]);
        if (!g_col && !delta)
            return fail(DTB_ERR_ARG, "column %d: per-neuron values are kept for g_ui (columns 10-13) only; "
                        "other columns take the delta limit (alpha >= 1e6)", col[i]);
    }
    DeviceGuard g(b->device);
    RET(keep_current_isyn(b));   // the new values reach I_syn one step later, as in the reference
    if (b->class_prop_base.empty()) b->class_prop_base = b->class_prop;
    std::unordered_map<int32_t, std::vector<int32_t>> by_sub;
    for (int c = 0; c < b->n_classes; ++c) by_sub[b->classes[(size_t)c].sub].push_back(c);
    std::vector<char> dirty((size_t)b->n_classes, 0), tau_set((size_t)b->n_classes, 0);
    std::vector<int32_t> req((size_t)std::max(1, b->n_sub) * 4, -1);
    std::vector<double> ha, hb;
    bool any_g = false;
    for (int i = 0; i < n; ++i) {
        auto it = by_sub.find(sub[i]);
        if (it == by_sub.end()) continue;
        const bool g_col = col[i] >= 10 && col[i] < 14;
        // the sampled values become the base that later subblock scalings multiply
        const float v = g_col ? 1.0f : (float)((double)alpha[i] / (double)beta[i]);
        for (int32_t c : it->second) {
            b->class_prop[(size_t)c][(size_t)col[i]] = v;
            b->class_prop_base[(size_t)c][(size_t)col[i]] = v;
            dirty[(size_t)c] = 1;
            if (col[i] >= 18) tau_set[(size_t)c] = 1;
        }
        if (g_col && sub[i] >= 0 && sub[i] < b->n_sub) {
            req[(size_t)sub[i] * 4 + (size_t)(col[i] - 10)] = (int32_t)ha.size();
            ha.push_back(alpha[i]);
            hb.push_back(beta[i]);
            any_g = true;
        }
    }
    if (any_g) {
        if (!b->d_gnrn) {
            RET(dalloc(b, &b->d_gnrn, (size_t)std::max<int64_t>(b->N, 1)));
            k_fill4<<<grid_for(b->N, 256), 256, 0, b->stream>>>(b->d_gnrn, b->N, make_float4(1.f, 1.f, 1.f, 1.f));
            CK(cudaGetLastError());
        }
        if (!b->ds.gnrn) {   // re-activated after update_property: start again from factor 1
            k_fill4<<<grid_for(b->N, 256), 256, 0, b->stream>>>(b->d_gnrn, b->N, make_float4(1.f, 1.f, 1.f, 1.f));
            CK(cudaGetLastError());
        }
        int32_t* dreq = nullptr; double* da = nullptr; double* db = nullptr;
        cudaError_t e = cudaMalloc(&dreq, sizeof(int32_t) * req.size());
        if (e == cudaSuccess) e = cudaMalloc(&da, sizeof(double) * ha.size());
        if (e == cudaSuccess) e = cudaMalloc(&db, sizeof(double) * hb.size());
        if (e == cudaSuccess) e = cudaMemcpyAsync(dreq, req.data(), sizeof(int32_t) * req.size(), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(da, ha.data(), sizeof(double) * ha.size(), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(db, hb.data(), sizeof(double) * hb.size(), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) {
            b->ds.gnrn = b->d_gnrn;
            drop_graphs(b);   // captured graphs hold the plain form of the update
            k_gamma<<<grid_for(b->N, 256), 256, 0, b->stream>>>(b->ds, dreq, da, db, b->gamma_calls, b->d_gnrn);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        cudaFree(dreq); cudaFree(da); cudaFree(db);
        if (e != cudaSuccess) return fail(DTB_ERR_CUDA, "gamma sampling: %s", cudaGetErrorString(e));
        b->gamma_calls++;
        drop_graphs(b);   // graphs hold the state by value
    }
    return rebuild_dirty_classes(b, dirty, &tau_set);
}

int dtb_block_set_input_spikes(dtb_block* b, int64_t n_src, const uint32_t* neurons, int64_t T, const uint8_t* spikes)
{
    if (!b || n_src < 0 || (n_src > 0 && (!neurons || !spikes || T < 1))) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(b->device);
    DevState& s = b->ds;
    CK(cudaStreamSynchronize(b->stream));   // the previous buffers are no longer in use
    drop_graphs(b);
    s.n_src = 0;
    s.forced_active = nullptr;
    dfree(b, s.forced_mask); dfree(b, s.src_neuron); dfree(b, s.src_raster); dfree(b, s.src_val);
    if (n_src == 0) return DTB_OK;
    std::vector<uint32_t> mask((size_t)s.n_words, 0u);
    for (int64_t i = 0; i < n_src; ++i) {
        if (neurons[i] >= (uint64_t)b->N) return fail(DTB_ERR_ARG, "input %lld: neuron %u out of range", (long long)i, neurons[i]);
        uint32_t& w = mask[neurons[i] >> 5];
        if (w & (1u << (neurons[i] & 31))) return fail(DTB_ERR_ARG, "input neuron %u given twice", neurons[i]);
        w |= 1u << (neurons[i] & 31);
    }
    const int64_t words = (n_src + 31) / 32;
    std::vector<uint32_t> raster((size_t)(T * words), 0u);   // [T][words], from [n_src][T] bytes
    for (int64_t i = 0; i < n_src; ++i)
        for (int64_t t = 0; t < T; ++t)
            if (spikes[i * T + t]) raster[(size_t)(t * words + (i >> 5))] |= 1u << (i & 31);
    uint32_t *dn = nullptr, *dr = nullptr, *dm = nullptr, *dv = nullptr;
    RET(dalloc(b, &dn, (size_t)n_src));
    RET(dalloc(b, &dr, raster.size()));
    RET(dalloc(b, &dm, (size_t)s.n_words));
    RET(dalloc(b, &dv, (size_t)s.n_words));
    CK(cudaMemcpy(dn, neurons, sizeof(uint32_t) * (size_t)n_src, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dr, raster.data(), sizeof(uint32_t) * raster.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dm, mask.data(), sizeof(uint32_t) * mask.size(), cudaMemcpyHostToDevice));
    s.n_src = n_src; s.src_neuron = dn; s.src_raster = dr; s.src_words = words; s.src_T = T;
    s.src_from = b->steps;
    s.src_val = dv;
    s.forced_active = dv;
    s.forced_mask = dm;
    drop_graphs(b);
    return DTB_OK;
}

int dtb_block_update_conn_weight(dtb_block* b, int64_t n, const uint8_t* channel, const uint32_t* post,
                                 const uint32_t* pre, const float* value)
{
    if (!b || n < 0 || (n > 0 && (!channel || !post || !pre || !value))) return fail(DTB_ERR_ARG, "bad argument");
    if (n == 0) return DTB_OK;
    for (int64_t i = 0; i < n; ++i)
        if (channel[i] > 3) return fail(DTB_ERR_ARG, "channel must be 0..3");
    DeviceGuard g(b->device);
    uint8_t* dch = nullptr; uint32_t* dpo = nullptr; uint32_t* dpr = nullptr; float* dv = nullptr; unsigned* miss = nullptr;
    cudaError_t e = cudaMalloc(&dch, (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dpo, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dpr, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&dv, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&miss, 4);
    unsigned hmiss = 0;
    if (e == cudaSuccess) {
        cudaMemcpy(dch, channel, (size_t)n, cudaMemcpyHostToDevice);
        cudaMemcpy(dpo, post, 4 * (size_t)n, cudaMemcpyHostToDevice);
        cudaMemcpy(dpr, pre, 4 * (size_t)n, cudaMemcpyHostToDevice);
        cudaMemcpy(dv, value, 4 * (size_t)n, cudaMemcpyHostToDevice);
        cudaMemset(miss, 0, 4);
        k_update_weight<<<grid_for(n, 128), 128, 0, b->stream>>>(b->ds, n, dch, dpo, dpr, dv,
                                                                const_cast<float2*>(b->ds.pw),
                                                                const_cast<float2*>(b->ds.qw), miss);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
        if (e == cudaSuccess) e = cudaMemcpy(&hmiss, miss, 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(dch); cudaFree(dpo); cudaFree(dpr); cudaFree(dv); cudaFree(miss);
    if (e != cudaSuccess) return fail(DTB_ERR_CUDA, "update_conn_weight: %s", cudaGetErrorString(e));
    if (hmiss) return fail(DTB_ERR_ARG, "update_conn_weight: %u synapses not found", hmiss);
    return DTB_OK;
}

// Checkpoint format: "DTBCKPT1", N (i64), steps (u64), t (f32), override flag (u32),
// then V[N], J as stored (excitatory pairs [N] float2, then inhibitory pairs),
// t_last[N], and I_syn override[N] if the flag is set.
int dtb_block_save(dtb_block* b, const char* path)
{
    if (!b || !path) return fail(DTB_ERR_ARG, "null argument");
    DeviceGuard g(b->device);
    const int64_t N = b->N;
    std::vector<float> V((size_t)N), T((size_t)N), I((size_t)N);
    std::vector<float4> J((size_t)N);
    float t = 0.0f;
    RET(flush_bins(b));
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemcpy(V.data(), b->ds.V, 4 * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(J.data(), b->ds.J2, 8 * N, cudaMemcpyDeviceToHost));                       // AMPA, NMDA plane
    CK(cudaMemcpy(reinterpret_cast<float2*>(J.data()) + N, b->ds.J2 + b->ds.j_ps, 8 * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(T.data(), b->ds.tlast, 4 * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&t, &b->ds.ctl->t, 4, cudaMemcpyDeviceToHost));
    const uint32_t ov = b->override_pending ? 1u : 0u;
    if (ov) CK(cudaMemcpy(I.data(), b->ds.isyn_override, 4 * N, cudaMemcpyDeviceToHost));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(DTB_ERR_IO, "cannot write %s", path);
    bool ok = std::fwrite("DTBCKPT1", 1, 8, f) == 8;
    ok = ok && std::fwrite(&N, 8, 1, f) == 1 && std::fwrite(&b->steps, 8, 1, f) == 1 && std::fwrite(&t, 4, 1, f) == 1 &&
         std::fwrite(&ov, 4, 1, f) == 1;
    ok = ok && std::fwrite(V.data(), 4, (size_t)N, f) == (size_t)N;
    ok = ok && std::fwrite(J.data(), 16, (size_t)N, f) == (size_t)N;
    ok = ok && std::fwrite(T.data(), 4, (size_t)N, f) == (size_t)N;
    if (ov) ok = ok && std::fwrite(I.data(), 4, (size_t)N, f) == (size_t)N;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(DTB_ERR_IO, "write failed: %s", path);
    return DTB_OK;
}

int dtb_block_load(dtb_block* b, const char* path)
{
    if (!b || !path) return fail(DTB_ERR_ARG, "null argument");
    DeviceGuard g(b->device);
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(DTB_ERR_IO, "cannot read %s", path);
    char magic[8];
    int64_t N = 0;
    uint64_t steps = 0;
    float t = 0.0f;
    uint32_t ov = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "DTBCKPT1", 8) == 0;
    ok = ok && std::fread(&N, 8, 1, f) == 1 && std::fread(&steps, 8, 1, f) == 1 && std::fread(&t, 4, 1, f) == 1 &&
         std::fread(&ov, 4, 1, f) == 1;
    if (!ok || N != b->N || ov > 1) { std::fclose(f); return fail(DTB_ERR_FORMAT, "%s is not a checkpoint of this network", path); }
    std::vector<float> V((size_t)N), T((size_t)N), I((size_t)N);
    std::vector<float4> J((size_t)N);
    ok = std::fread(V.data(), 4, (size_t)N, f) == (size_t)N && std::fread(J.data(), 16, (size_t)N, f) == (size_t)N &&
         std::fread(T.data(), 4, (size_t)N, f) == (size_t)N;
    if (ok && ov) ok = std::fread(I.data(), 4, (size_t)N, f) == (size_t)N;
    std::fclose(f);
    if (!ok) return fail(DTB_ERR_FORMAT, "truncated checkpoint %s", path);
    RET(discard_bins(b));
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaMemcpy(b->ds.V, V.data(), 4 * N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->ds.J2, J.data(), 8 * N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->ds.J2 + b->ds.j_ps, reinterpret_cast<const float2*>(J.data()) + N, 8 * N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->ds.tlast, T.data(), 4 * N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&b->ds.ctl->t, &t, 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&b->ds.ctl->steps_done, &steps, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(&b->ds.ctl->use_isyn_override, &ov, 4, cudaMemcpyHostToDevice));
    if (ov) CK(cudaMemcpy(b->ds.isyn_override, I.data(), 4 * N, cudaMemcpyHostToDevice));
    b->steps = steps;
    b->override_pending = false;
    b->override_live = ov != 0;
    return DTB_OK;
}

// ------------------------------------------------------------ BOLD (standalone)
static int bold_init_state(dtb_bold* m)
{
    const int64_t R = m->R;
    const unsigned gr = grid_for(R, 256);
    if (m->dtype == 0) {
        k_fill<float><<<gr, 256, 0, m->stream>>>((float*)m->s, R, 0.0f);
        k_fill<float><<<gr, 256, 0, m->stream>>>((float*)m->q, R, 0.0f);
        k_fill<float><<<gr, 256, 0, m->stream>>>((float*)m->v, R, 1.0f);
        k_fill<float><<<gr, 256, 0, m->stream>>>((float*)m->f, R, 1.0f);
    } else {
        k_fill<double><<<gr, 256, 0, m->stream>>>((double*)m->s, R, 0.0);
        k_fill<double><<<gr, 256, 0, m->stream>>>((double*)m->q, R, 0.0);
        k_fill<double><<<gr, 256, 0, m->stream>>>((double*)m->v, R, 1.0);
        k_fill<double><<<gr, 256, 0, m->stream>>>((double*)m->f, R, 1.0);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->stream));
    return DTB_OK;
}

static void bold_free(dtb_bold* m)
{
    if (!m) return;
    DeviceGuard g(m->device);
    void* ps[] = {m->s, m->q, m->v, m->f, m->tmp_u, m->tmp_o, m->tmp_w};
    for (void* p : ps) if (p) cudaFree(p);
    delete m;
}

int dtb_bold_create(int64_t n_regions, int dtype, double epsilon, double tao_s, double tao_f, double tao_0, double alpha,
                    double E_0, double V_0, double delta_t, int device, dtb_bold** out)
{
    if (!out || n_regions <= 0 || (dtype != 0 && dtype != 1)) return fail(DTB_ERR_ARG, "bad argument");
    *out = nullptr;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(DTB_ERR_ARG, "device out of range");
    DeviceGuard g(device);
    dtb_bold* m = new dtb_bold();
    m->device = device; m->R = n_regions; m->dtype = dtype;
    m->eps = epsilon; m->ts = tao_s; m->tf = tao_f; m->t0 = tao_0; m->alpha = alpha; m->E0 = E_0; m->V0 = V_0; m->dt = delta_t;
    const size_t el = dtype ? 8 : 4;
    void** ps[] = {&m->s, &m->q, &m->v, &m->f, &m->tmp_u, &m->tmp_o};
    for (void** p : ps) {
        if (cudaMalloc(p, el * (size_t)n_regions) != cudaSuccess) {
            cudaGetLastError();
            bold_free(m);
            return fail(DTB_ERR_NOMEM, "BOLD state allocation failed");
        }
    }
    int rc = bold_init_state(m);
    if (rc != DTB_OK) { bold_free(m); return rc; }
    *out = m;
    return DTB_OK;
}

int dtb_bold_destroy(dtb_bold* m)
{
    bold_free(m);
    return DTB_OK;
}

int dtb_bold_set_stream(dtb_bold* m, void* stream)
{
    if (!m) return fail(DTB_ERR_ARG, "null handle");
    m->stream = (cudaStream_t)stream;
    return DTB_OK;
}

int dtb_bold_run(dtb_bold* m, const void* u, void* out, int where)
{
    if (!m || !u || !out) return fail(DTB_ERR_ARG, "null argument");
    DeviceGuard g(m->device);
    const size_t bytes = (m->dtype ? 8 : 4) * (size_t)m->R;
    const void* du = u;
    void* dout = out;
    if (where == DTB_HOST) {
        CK(cudaMemcpyAsync(m->tmp_u, u, bytes, cudaMemcpyHostToDevice, m->stream));
        du = m->tmp_u;
        dout = m->tmp_o;
    }
    const unsigned gr = grid_for(m->R, 128);
    if (m->dtype == 0)
        k_bold_run<float><<<gr, 128, 0, m->stream>>>(m->R, (const float*)du, (float*)m->s, (float*)m->q, (float*)m->v,
                                                     (float*)m->f, (float*)dout, bold_scalars<float>(m));
    else
        k_bold_run<double><<<gr, 128, 0, m->stream>>>(m->R, (const double*)du, (double*)m->s, (double*)m->q,
                                                      (double*)m->v, (double*)m->f, (double*)dout,
                                                      bold_scalars<double>(m));
    CK(cudaGetLastError());
    if (where == DTB_HOST) {
        CK(cudaMemcpyAsync(out, m->tmp_o, bytes, cudaMemcpyDeviceToHost, m->stream));
        CK(cudaStreamSynchronize(m->stream));
    }
    return DTB_OK;
}

int dtb_bold_run_steps(dtb_bold* m, const void* u, int n_steps, double u_floor, void* out, int where)
{
    if (!m || !u || !out || n_steps < 0) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(m->device);
    const size_t bytes = (m->dtype ? 8 : 4) * (size_t)m->R;
    const void* du = u;
    void* dout = out;
    if (where == DTB_HOST) {
        CK(cudaMemcpyAsync(m->tmp_u, u, bytes, cudaMemcpyHostToDevice, m->stream));
        du = m->tmp_u;
        dout = m->tmp_o;
    }
    const unsigned gr = grid_for(m->R, 128);
    if (m->dtype == 0)
        k_bold_run_steps<float><<<gr, 128, 0, m->stream>>>(m->R, (const float*)du, n_steps, (float)u_floor,
                                                           (float*)m->s, (float*)m->q, (float*)m->v, (float*)m->f,
                                                           (float*)dout, bold_scalars<float>(m));
    else
        k_bold_run_steps<double><<<gr, 128, 0, m->stream>>>(m->R, (const double*)du, n_steps, u_floor,
                                                            (double*)m->s, (double*)m->q, (double*)m->v,
                                                            (double*)m->f, (double*)dout, bold_scalars<double>(m));
    CK(cudaGetLastError());
    if (where == DTB_HOST) {
        CK(cudaMemcpyAsync(out, m->tmp_o, bytes, cudaMemcpyDeviceToHost, m->stream));
        CK(cudaStreamSynchronize(m->stream));
    }
    return DTB_OK;
}

int dtb_bold_state_update(dtb_bold* m, const void* w, int64_t E, int64_t Rp, int64_t S, int where)
{
    if (!m || !w) return fail(DTB_ERR_ARG, "null argument");
    if (E * Rp != m->R || S < 4) return fail(DTB_ERR_ARG, "state_update: w must be [E][R/E][>=4] with E*Rp == R");
    DeviceGuard g(m->device);
    const size_t el = m->dtype ? 8 : 4;
    const size_t bytes = el * (size_t)m->R * (size_t)S;
    const void* dw = w;
    if (where == DTB_HOST) {
        if (m->tmp_w_bytes < bytes) {
            if (m->tmp_w) cudaFree(m->tmp_w);
            m->tmp_w = nullptr;
            m->tmp_w_bytes = 0;
            CK(cudaMalloc(&m->tmp_w, bytes));
            m->tmp_w_bytes = bytes;
        }
        CK(cudaMemcpyAsync(m->tmp_w, w, bytes, cudaMemcpyHostToDevice, m->stream));
        dw = m->tmp_w;
    }
    const unsigned gr = grid_for(m->R, 128);
    if (m->dtype == 0)
        k_bold_state_update<float><<<gr, 128, 0, m->stream>>>(m->R, S, (const float*)dw, (float*)m->s, (float*)m->q,
                                                              (float*)m->v, (float*)m->f, 1e-05f);
    else
        k_bold_state_update<double><<<gr, 128, 0, m->stream>>>(m->R, S, (const double*)dw, (double*)m->s,
                                                               (double*)m->q, (double*)m->v, (double*)m->f, 1e-05);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->stream));
    return DTB_OK;
}

int dtb_bold_get(dtb_bold* m, int field, void* dst, int where)
{
    if (!m || !dst || field < 0 || field > 3) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(m->device);
    void* src[4] = {m->s, m->q, m->v, m->f};
    const size_t bytes = (m->dtype ? 8 : 4) * (size_t)m->R;
    CK(cudaMemcpyAsync(dst, src[field], bytes, where == DTB_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                       m->stream));
    CK(cudaStreamSynchronize(m->stream));
    return DTB_OK;
}

int dtb_bold_set(dtb_bold* m, int field, const void* srcp, int where)
{
    if (!m || !srcp || field < 0 || field > 3) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(m->device);
    void* dst[4] = {m->s, m->q, m->v, m->f};
    const size_t bytes = (m->dtype ? 8 : 4) * (size_t)m->R;
    CK(cudaMemcpyAsync(dst[field], srcp, bytes, where == DTB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                       m->stream));
    CK(cudaStreamSynchronize(m->stream));
    return DTB_OK;
}

// ------------------------------------------------------------ block-attached BOLD
int dtb_block_attach_bold(dtb_block* b, int n_regions, const int32_t* sub_to_region, double epsilon, double tao_s,
                          double tao_f, double tao_0, double alpha, double E_0, double V_0, double delta_t)
{
    if (!b || n_regions <= 0 || !sub_to_region || !(delta_t > 0.0)) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(b->device);
    std::vector<double> rn((size_t)n_regions, 0.0);
    for (int i = 0; i < b->n_sub; ++i) {
        const int r = sub_to_region[i];
        if (r >= n_regions) return fail(DTB_ERR_ARG, "sub_to_region[%d] = %d out of range", i, r);
        if (r >= 0) rn[(size_t)r] += (double)b->sub_count[(size_t)i];
    }
    BoldDev& bd = b->ds.bold;
    int32_t* sr = nullptr; double* drn = nullptr; double* st = nullptr;
    RET(dalloc(b, &sr, (size_t)std::max(1, b->n_sub)));
    RET(dalloc(b, &drn, (size_t)n_regions));
    RET(dalloc(b, &st, (size_t)n_regions * 6));
    if (b->n_sub) CK(cudaMemcpy(sr, sub_to_region, sizeof(int32_t) * b->n_sub, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(drn, rn.data(), sizeof(double) * n_regions, cudaMemcpyHostToDevice));
    std::vector<double> init((size_t)n_regions * 6, 0.0);
    for (int r = 0; r < n_regions; ++r) { init[(size_t)(2 * n_regions + r)] = 1.0; init[(size_t)(3 * n_regions + r)] = 1.0; }
    CK(cudaMemcpy(st, init.data(), sizeof(double) * init.size(), cudaMemcpyHostToDevice));
    bd.n_regions = n_regions;
    bd.sub_region = sr;
    bd.region_n = drn;
    bd.s = st; bd.q = st + n_regions; bd.v = st + 2 * n_regions; bd.f = st + 3 * n_regions;
    bd.act = st + 4 * n_regions; bd.out = st + 5 * n_regions;
    bd.epsilon = epsilon; bd.tao_s = tao_s; bd.tao_f = tao_f; bd.tao_0 = tao_0; bd.div_alpha = 1.0 / alpha;
    bd.E0 = E_0; bd.V0 = V_0; bd.delta_t = delta_t;
    b->bold_R = n_regions;
    RET(rebuild_groups(b, sub_to_region));
    for (auto& ge : b->graph) if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
    return DTB_OK;
}

int dtb_block_set_samples(dtb_block* b, int n, const uint32_t* idx, int64_t capacity_steps)
{
    if (!b || n < 0 || (n > 0 && (!idx || capacity_steps < 1))) return fail(DTB_ERR_ARG, "bad argument");
    DeviceGuard g(b->device);
    DevState& s = b->ds;
    for (int i = 0; i < n; ++i)
        if (idx[i] >= (uint64_t)b->N) return fail(DTB_ERR_ARG, "sample %d: neuron %u out of range", i, idx[i]);
    CK(cudaStreamSynchronize(b->stream));   // the previous buffers are no longer in use
    drop_graphs(b);
    s.n_samples = 0;
    b->samples_written = 0;
    dfree(b, s.samples); dfree(b, s.samp_spk); dfree(b, s.samp_v);
    if (n == 0) return DTB_OK;
    uint32_t* di = nullptr; uint8_t* sp = nullptr; float* sv = nullptr;
    RET(dalloc(b, &di, (size_t)n));
    RET(dalloc(b, &sp, (size_t)n * (size_t)capacity_steps));
    RET(dalloc(b, &sv, (size_t)n * (size_t)capacity_steps));
    CK(cudaMemcpy(di, idx, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    s.samples = di; s.samp_spk = sp; s.samp_v = sv; s.samp_cap = capacity_steps; s.n_samples = n;
    b->samples_from = b->steps;
    drop_graphs(b);
    return DTB_OK;
}

int dtb_block_get_samples(dtb_block* b, uint8_t* spikes, float* v, int64_t* rows, int where)
{
    if (!b || !rows) return fail(DTB_ERR_ARG, "null argument");
    const DevState& s = b->ds;
    if (s.n_samples <= 0) { *rows = 0; return DTB_OK; }
    DeviceGuard g(b->device);
    const int64_t total = (int64_t)(b->steps - b->samples_from);
    const int64_t nr = std::min<int64_t>(total, s.samp_cap);
    *rows = nr;
    if (nr <= 0) return DTB_OK;
    // chronological order: the oldest kept row first
    const int64_t first_step = (int64_t)b->steps - nr;
    const int64_t r0 = first_step % s.samp_cap;
    const int64_t n1 = std::min<int64_t>(nr, s.samp_cap - r0);
    const cudaMemcpyKind k = where == DTB_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const size_t ns = (size_t)s.n_samples;
    if (spikes) {
        CK(cudaMemcpyAsync(spikes, s.samp_spk + r0 * ns, n1 * ns, k, b->stream));
        if (nr > n1) CK(cudaMemcpyAsync(spikes + n1 * ns, s.samp_spk, (nr - n1) * ns, k, b->stream));
    }
    if (v) {
        CK(cudaMemcpyAsync(v, s.samp_v + r0 * ns, n1 * ns * 4, k, b->stream));
        if (nr > n1) CK(cudaMemcpyAsync(v + n1 * ns, s.samp_v, (nr - n1) * ns * 4, k, b->stream));
    }
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

int dtb_block_set_bold(dtb_block* b, int field, const double* src, int where)
{
    if (!b || !src || field < 0 || field > 3) return fail(DTB_ERR_ARG, "bad argument");
    if (b->bold_R == 0) return fail(DTB_ERR_STATE, "no BOLD model attached");
    DeviceGuard g(b->device);
    const BoldDev& bd = b->ds.bold;
    double* dst[4] = {bd.s, bd.q, bd.v, bd.f};
    CK(cudaMemcpyAsync(dst[field], src, sizeof(double) * b->bold_R,
                       where == DTB_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return DTB_OK;
}

int dtb_block_get_bold(dtb_block* b, int field, double* dst, int where)
{
    if (!b || !dst || field < 0 || field > 5) return fail(DTB_ERR_ARG, "bad argument");
    if (b->bold_R == 0) return fail(DTB_ERR_STATE, "no BOLD model attached");
    DeviceGuard g(b->device);
    const BoldDev& bd = b->ds.bold;
    const double* src[6] = {bd.s, bd.q, bd.v, bd.f, bd.out, bd.act};
    return copy_out(b, dst, src[field], sizeof(double) * b->bold_R, where);
}

}  // extern "C"
