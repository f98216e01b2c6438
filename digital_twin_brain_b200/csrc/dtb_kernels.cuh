// Kernels of libdtb (sm_100a).
//
// Step pipeline of one time step k (models/block.py:116-150):
//   update_k  : I_syn(V,J) -> V, threshold, refractory, Philox noise,
//               bitmask of spikes|noise, J <- J*decay (pending), stats.
//   propagate : push  — k_scatter: every set bit of the bitmask scatters its
//               outgoing row with float2 atomics into the pending J;
//               pull  — k_step<GATHER>: every postsynaptic row sums the
//               weights of its firing presynaptic neurons in row order
//               (torch.sparse.mm's order, bit-identical) and adds them to
//               the pending J.  The pull gather of step k is fused with the
//               update of step k+1 (k_step<true,true>), so a run of n pull
//               steps is update, n-1 fused kernels and one gather-only kernel.
// The last CTA of every update kernel folds the per-subblock statistics,
// runs the per-region BOLD step when one is attached, and advances the
// device clock (steps_done, t) — no extra launch per step.
#pragma once

#include "dtb_device.cuh"

namespace dtb {

// ------------------------------------------------------------ neuron math
// Operation order of models/block.py:83-111 with round-to-nearest float32
// intrinsics so that no multiply-add is contracted.

__device__ __forceinline__ float isyn_g(float4 g, float4 Vu, float v, float4 J)
{
    const float i0 = __fmul_rn(__fmul_rn(g.x, __fsub_rn(Vu.x, v)), J.x);
    const float i1 = __fmul_rn(__fmul_rn(g.y, __fsub_rn(Vu.y, v)), J.y);
    const float i2 = __fmul_rn(__fmul_rn(g.z, __fsub_rn(Vu.z, v)), J.z);
    const float i3 = __fmul_rn(__fmul_rn(g.w, __fsub_rn(Vu.w, v)), J.w);
    return __fadd_rn(__fadd_rn(__fadd_rn(i0, i1), i2), i3);
}

__device__ __forceinline__ float4 iui_g(float4 g, float4 Vu, float v, float4 J)
{
    return make_float4(__fmul_rn(__fmul_rn(g.x, __fsub_rn(Vu.x, v)), J.x),
                       __fmul_rn(__fmul_rn(g.y, __fsub_rn(Vu.y, v)), J.y),
                       __fmul_rn(__fmul_rn(g.z, __fsub_rn(Vu.z, v)), J.z),
                       __fmul_rn(__fmul_rn(g.w, __fsub_rn(Vu.w, v)), J.w));
}

__device__ __forceinline__ float isyn_of(const ParamClass& p, float v, float4 J) { return isyn_g(p.g, p.Vu, v, J); }

__device__ __forceinline__ ParamClass load_class(const ParamClass* __restrict__ pc, uint32_t c)
{
    const float4* src = reinterpret_cast<const float4*>(pc + c);
    ParamClass p;
    float4* dst = reinterpret_cast<float4*>(&p);
#pragma unroll
    for (int i = 0; i < 6; ++i) dst[i] = __ldg(src + i);
    return p;
}

__device__ __forceinline__ float4 add4(float4 a, float4 b)
{
    return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}

__device__ __forceinline__ float4 mul4(float4 a, float4 b)
{
    return make_float4(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z), __fmul_rn(a.w, b.w));
}

// J of neuron n as {AMPA, NMDA, GABAa, GABAb} (streaming access: once per step).
__device__ __forceinline__ float4 load_J(const DevState& s, int64_t n)
{
    const float2 a = __ldcs(s.J2 + n * s.j_es);
    const float2 b = __ldcs(s.J2 + s.j_ps + n * s.j_es);
    return make_float4(a.x, a.y, b.x, b.y);
}

// j_keep: the update's J stores keep their L2 lines (normal priority) so that the
// push scatter that follows finds part of J in L2 for its read-modify-writes;
// otherwise they stream (evict first) like the rest of the state.
__device__ __forceinline__ void store_J(const DevState& s, int64_t n, float4 J)
{
    if (s.j_keep) {
        __stcg(s.J2 + n * s.j_es, make_float2(J.x, J.y));
        __stcg(s.J2 + s.j_ps + n * s.j_es, make_float2(J.z, J.w));
    } else {
        __stcs(s.J2 + n * s.j_es, make_float2(J.x, J.y));
        __stcs(s.J2 + s.j_ps + n * s.j_es, make_float2(J.z, J.w));
    }
}

// Synaptic events propagated by a warp or CTA, into one of kEvParts counters.
__device__ __forceinline__ void add_events(const DevState& s, unsigned long long ev, uint32_t key)
{
    if (!ev) return;
    if (s.ev_part) atomicAdd(s.ev_part + (key & (kEvParts - 1)), ev);
    else atomicAdd(&s.ctl->events, ev);
}

__device__ __forceinline__ bool test_bit(const uint32_t* __restrict__ bits, int64_t n)
{
    return (__ldg(bits + (n >> 5)) >> (n & 31)) & 1u;
}

// ------------------------------------------------------------ pull gather
// Sum of the weights of row n whose presynaptic neuron is set in `bits`,
// accumulated strictly in row order from +0 (sparse.mm order). All lanes
// return the same value.
__device__ __forceinline__ float4 gather_row(const DevState& s, const uint32_t* __restrict__ bits, int64_t n,
                                             int lane, uint32_t& events)
{
    const int64_t e0 = __ldg(s.prow + n);
    const int64_t e1 = __ldg(s.prow + n + 1);
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    for (int64_t e = e0; e < e1; e += 32) {
        const int64_t idx = e + lane;
        const bool valid = idx < e1;
        const uint32_t c = valid ? __ldg(s.pcol + idx) : 0u;
        const bool act = valid && test_bit(bits, c & kIndexMask);
        unsigned m = __ballot_sync(0xffffffffu, act);
        events += __popc(m);
        float2 w = make_float2(0.0f, 0.0f);
        if (act) w = __ldg(s.pw + idx);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const float wx = __shfl_sync(0xffffffffu, w.x, l);
            const float wy = __shfl_sync(0xffffffffu, w.y, l);
            const uint32_t cl = __shfl_sync(0xffffffffu, c, l);
            if (cl & kKindBit) { a2 = __fadd_rn(a2, wx); a3 = __fadd_rn(a3, wy); }
            else { a0 = __fadd_rn(a0, wx); a1 = __fadd_rn(a1, wy); }
        }
    }
    return make_float4(a0, a1, a2, a3);
}

// Sum of one neuron's c <= kSlotCap ordered-push contributions in ascending
// pull-row position (the order gather_row adds them).  Two terms added to +0
// give the same float in either order, so only c >= 3 needs the ordering.
__device__ __forceinline__ void slot_add(uint4 v, float& a0, float& a1, float& a2, float& a3)
{
    const float wx = __uint_as_float(v.z), wy = __uint_as_float(v.w);
    if (v.x & kKindBit) { a2 = __fadd_rn(a2, wx); a3 = __fadd_rn(a3, wy); }
    else { a0 = __fadd_rn(a0, wx); a1 = __fadd_rn(a1, wy); }
}

// One or two contributions (already loaded): any order gives the same float.
__device__ __forceinline__ float4 slot_pair_sum(uint4 v0, uint4 v1, uint32_t c)
{
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    slot_add(v0, a0, a1, a2, a3);
    if (c == 2u) slot_add(v1, a0, a1, a2, a3);
    return make_float4(a0, a1, a2, a3);
}

__device__ __forceinline__ float4 slot_sum(const uint4* __restrict__ sl, uint32_t c)
{
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    auto add = [&](uint4 v) {
        const float wx = __uint_as_float(v.z), wy = __uint_as_float(v.w);
        if (v.x & kKindBit) { a2 = __fadd_rn(a2, wx); a3 = __fadd_rn(a3, wy); }
        else { a0 = __fadd_rn(a0, wx); a1 = __fadd_rn(a1, wy); }
    };
    if (c <= 2u) {
        add(__ldcs(sl));
        if (c == 2u) add(__ldcs(sl + 1));
    } else {
        uint32_t last = 0u;
        for (uint32_t r = 0; r < c; ++r) {
            uint4 best = make_uint4(0u, 0u, 0u, 0u);
            uint32_t bp = 0xffffffffu;
            for (uint32_t k = 0; k < c; ++k) {
                const uint4 v = sl[k];
                const uint32_t p = v.x & kIndexMask;
                if ((r == 0u || p > last) && p < bp) { bp = p; best = v; }
            }
            add(best);
            last = bp;
        }
    }
    return make_float4(a0, a1, a2, a3);
}

// Sum of the pull entries a neuron's position masks mark, in ascending position
// (the order gather_row adds them): excitatory and inhibitory pairs are summed
// separately, as gather_row's two accumulator pairs are.  Up to 8 weights are
// loaded before they are added.
__device__ __forceinline__ float4 mask_sum(const DevState& s, int64_t n, uint4 ex, uint4 in)
{
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    const float2* __restrict__ pw = s.pw + __ldg(s.prow + n);
#pragma unroll
    for (int kind = 0; kind < 2; ++kind) {
        const uint4 m4 = kind ? in : ex;
        uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
        float x = 0.0f, y = 0.0f;
#pragma unroll
        for (int wi = 0; wi < 4; ++wi) {
            uint32_t word = mw[wi];
            while (word) {
                uint32_t pos[8];
                int k = 0;
                while (word && k < 8) {
                    const int bit = __ffs(word) - 1;
                    word &= word - 1u;
                    pos[k++] = (uint32_t)(wi * 32 + bit);
                }
                float2 w[8];
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    if (i < k) w[i] = __ldg(pw + pos[i]);
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    if (i < k) { x = __fadd_rn(x, w[i].x); y = __fadd_rn(y, w[i].y); }
            }
        }
        if (kind) { a.z = x; a.w = y; } else { a.x = x; a.y = y; }
    }
    return a;
}

// ------------------------------------------------------------ BOLD step
// models/bold_model_pytorch.py:43-78 in float64 for region r with input u
// (q before v before f_in before s, f_in clamped at 0).
__device__ __forceinline__ void bold_region_step(const BoldDev& b, int r, double u)
{
    double fi = b.f[r], si = b.s[r], qi = b.q[r], vi = b.v[r];
    const double ds = ((b.epsilon * u) - si / b.tao_s) - (fi - 1.0) / b.tao_f;
    const double qpart = fi > 0.0 ? (1.0 - pow(1.0 - b.E0, 1.0 / fi)) : 1.0;
    const double dq = (((fi * qpart) / b.E0) - qi * pow(vi, b.div_alpha - 1.0)) / b.tao_0;
    qi = qi + dq * b.delta_t;
    const double dv = (fi - pow(vi, b.div_alpha)) / b.tao_0;
    vi = vi + dv * b.delta_t;
    fi = fi + si * b.delta_t;
    fi = fi > 0.0 ? fi : 0.0;
    si = si + ds * b.delta_t;
    b.s[r] = si; b.q[r] = qi; b.v[r] = vi; b.f[r] = fi;
    b.out[r] = b.V0 * ((7.0 * b.E0 * (1.0 - qi) + 2.0 * (1.0 - qi / vi)) + (2.0 * b.E0 - 0.2) * (1.0 - vi));
}

// ------------------------------------------------------------ epilogue
// Runs in the last CTA of an update kernel: per-subblock statistics of step
// `steps_done` (models/block.py:144-150), BOLD (simulation/simulation.py:
// 269-279 + models/bold_model_pytorch.py:43-78 in float64), clock advance.
__device__ void step_epilogue(const DevState& s, unsigned long long steps_done, float t)
{
    Ctl* ctl = s.ctl;
    const unsigned long long row = steps_done - ctl->run_base;
    const bool write = row < (unsigned long long)ctl->stats_cap;
    if (s.stats_ext) {   // k_stats folds the statistics right after this kernel
        if (threadIdx.x == 0) {
            if (write) s.st_nact[row] = atomicExch(s.unmapped_nact, 0u);
            ctl->t = t;
            ctl->use_isyn_override = 0u;
            ctl->done = 0u;
            ctl->steps_done = steps_done + 1ull;
            __threadfence();
        }
        return;
    }
    __shared__ unsigned long long sh_nact;
    if (threadIdx.x == 0) sh_nact = atomicExch(s.unmapped_nact, 0u);
    if (s.bold.n_regions > 0)
        for (int r = threadIdx.x; r < s.bold.n_regions; r += blockDim.x) s.bold.act[r] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < s.n_sub; i += blockDim.x) {
        const uint32_t spk = atomicExch(s.sub_spk + i, 0u);
        const uint32_t nact = atomicExch(s.sub_nact + i, 0u);
        const unsigned long long vb =
            atomicExch(reinterpret_cast<unsigned long long*>(s.sub_vsum + i), 0ull);
        const double vsum = __longlong_as_double((long long)vb);
        const uint32_t cnt = s.sub_count[i];
        if (s.win_spk) s.win_spk[i] += spk;
        if (write) {
            s.st_spk[row * s.n_sub + i] = (float)spk;
            s.st_mean[row * s.n_sub + i] = cnt ? (float)(vsum / (double)cnt) : __int_as_float(0x7fc00000);
        }
        atomicAdd(&sh_nact, (unsigned long long)nact);
        if (s.bold.n_regions > 0) {
            const int r = s.bold.sub_region[i];
            if (r >= 0) atomicAdd(s.bold.act + r, (double)spk);
        }
    }
    __syncthreads();
    if (s.bold.n_regions > 0) {
        const BoldDev& b = s.bold;
        for (int r = threadIdx.x; r < b.n_regions; r += blockDim.x) {
            const double act = b.region_n[r] > 0.0 ? b.act[r] / b.region_n[r] : 0.0;
            b.act[r] = act;
            bold_region_step(b, r, act > 1e-5 ? act : 1e-5);
        }
    }
    if (threadIdx.x == 0) {
        if (write) s.st_nact[row] = (uint32_t)sh_nact;
        ctl->t = t;
        ctl->use_isyn_override = 0u;
        ctl->done = 0u;
        ctl->steps_done = steps_done + 1ull;
        __threadfence();
    }
}

// ------------------------------------------------------------ statistics kernel
// For networks with many subblocks or regions (ensembles): one thread per
// group (a BOLD region with its subblocks, or a lone subblock) folds the
// accumulators of the step just taken into the per-step rows and the window
// totals, and runs the region's BOLD step.  Launched right after each update.
__global__ void __launch_bounds__(256) k_stats(DevState s)
{
    const Ctl* ctl = s.ctl;
    const unsigned long long row = ctl->steps_done - 1ull - ctl->run_base;   // clock already advanced
    const bool write = row < (unsigned long long)ctl->stats_cap;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t nact_sum = 0;
    if (g < s.n_groups) {
        double spk_sum = 0.0;
        for (int k = s.grp_ptr[g]; k < s.grp_ptr[g + 1]; ++k) {
            const int i = s.grp_sub[k];
            const uint32_t spk = atomicExch(s.sub_spk + i, 0u);
            nact_sum += atomicExch(s.sub_nact + i, 0u);
            const double vsum = __longlong_as_double(
                (long long)atomicExch(reinterpret_cast<unsigned long long*>(s.sub_vsum + i), 0ull));
            const uint32_t cnt = s.sub_count[i];
            if (s.win_spk) s.win_spk[i] += spk;
            if (write) {
                s.st_spk[row * s.n_sub + i] = (float)spk;
                s.st_mean[row * s.n_sub + i] = cnt ? (float)(vsum / (double)cnt) : __int_as_float(0x7fc00000);
            }
            spk_sum += (double)spk;
        }
        const int r = s.grp_region[g];
        if (r >= 0 && s.bold.n_regions > 0) {
            const BoldDev& b = s.bold;
            const double act = b.region_n[r] > 0.0 ? spk_sum / b.region_n[r] : 0.0;
            b.act[r] = act;
            bold_region_step(b, r, act > 1e-5 ? act : 1e-5);
        }
    }
    const uint32_t w = __reduce_add_sync(0xffffffffu, nact_sum);
    if ((threadIdx.x & 31) == 0 && w && write) atomicAdd(s.st_nact + row, w);
}

// ------------------------------------------------------------ samples
// cuda/src/stage/sample.cpp:8-26 / stat_result.cpp:283-305: spike and V of the
// sampled neurons after the step just taken, into a ring of steps.
__global__ void k_samples(DevState s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_samples) return;
    const unsigned long long step = s.ctl->steps_done - 1ull;   // clock already advanced
    const int64_t row = (int64_t)(step % (unsigned long long)s.samp_cap);
    const uint32_t n = s.samples[i];
    s.samp_spk[row * s.n_samples + i] = (uint8_t)((s.abits[n >> 5] >> (n & 31)) & 1u);
    s.samp_v[row * s.n_samples + i] = s.V[n];
}

// ------------------------------------------------------------ staged state loads
// Bulk asynchronous copies (cp.async.bulk, the TMA engine; no multicast) of a
// tile's V, t_last and both J planes into shared memory, issued by lane 0 one
// tile ahead, so that the loads of tile k+1 are in flight while tile k computes
// (class ids come from the per-tile table, or, for a tile of mixed classes, from
// global memory).  Completion is counted on a per-warp, per-buffer mbarrier.
// 3 KB per buffer: eight warps' double buffers (48 KB) fit four CTAs per SM.
constexpr int kStageBytes = kWarpNeurons * (4 + 4 + 8 + 8);       // 3072 per tile buffer
constexpr int kStagedSmem = (kStepThreads / 32) * 2 * kStageBytes;
constexpr uint32_t kErrStageTimeout = 1u;                        // Ctl::err bit: a staged copy was given up on
constexpr uint32_t kErrStageDrain = 2u;                          // Ctl::err bit: ... and had not landed at exit
constexpr uint32_t kErrGeneralSkipped = 4u;                      // Ctl::err bit: an update needing the general form ran plain

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void stage_issue(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

// Lane 0: the four copies of tile `base` into buffer `buf` (16-byte aligned, whole tile):
// V at 0, t_last at 512, J plane 0 at 1024, J plane 1 at 2048.
__device__ __forceinline__ void stage_tile(const DevState& s, int64_t base, unsigned char* buf, uint32_t mbar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic reads of buf first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"((uint32_t)kStageBytes)
                 : "memory");
    const uint32_t d = smem_u32(buf);
    stage_issue(d, s.V + base, kWarpNeurons * 4, mbar);
    stage_issue(d + kWarpNeurons * 4, s.tlast + base, kWarpNeurons * 4, mbar);
    stage_issue(d + kWarpNeurons * 8, s.J2 + base, kWarpNeurons * 8, mbar);
    stage_issue(d + kWarpNeurons * 16, s.J2 + s.j_ps + base, kWarpNeurons * 8, mbar);
}

// Bounded wait for a buffer's copies: at most `limit` polls; false after the limit (the
// caller then loads from global).  limit 0 gives up at once (tests of the fallback).
__device__ __forceinline__ bool stage_wait(uint32_t mbar, uint32_t parity, uint32_t limit)
{
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

// ------------------------------------------------------------ binned push: fold
// CTA-wide: the events the push scatter appended to bin c (one bin = one chunk of
// 2^bin_shift neurons) are summed into acc[2^bin_shift] (float4 per neuron:
// AMPA, NMDA, GABAa, GABAb) with shared-memory atomics; the bin's count is reset
// for the next scatter.  Events beyond the bin's capacity were added to J by the
// scatter itself.  n_raw = the bin's count, read by the caller one chunk ahead;
// the first entries are loaded before the barrier that frees acc.  Every thread
// of the CTA calls it (three barriers).
constexpr int kFoldBatch = 8;   // entries per thread in flight

// Staged bin fold (kGatherBins with staged state): the first kBinStageMax entries of the
// next chunk's bin are bulk-copied into one of two shared buffers one chunk ahead (index
// array, then weight pairs); entries past it are read from global memory by the fold.
constexpr uint32_t kBinStageMax = 1216;                         // a multiple of 8 (16-byte copies)
constexpr int kBinStageBytes = (int)kBinStageMax * 10;
constexpr int kBinStagedSmem = kStagedSmem + 2 * kBinStageBytes;

// entries of a bin with n_raw appended events that the staged copy covers
__device__ __forceinline__ uint32_t bin_stage_n(const DevState& s, uint32_t n_raw)
{
    const uint32_t lst = kBinStageMax < (s.bin_cap & ~7u) ? kBinStageMax : (s.bin_cap & ~7u);
    const uint32_t n = n_raw < s.bin_cap ? n_raw : s.bin_cap;
    return n < lst ? n : lst;
}

// One thread: the copies of the first n entries of bin c (rounded up to whole 16-byte
// units: the bin capacity is a multiple of 8) into buf, completion counted on mbar.
__device__ __forceinline__ void stage_bin(const DevState& s, int64_t c, uint32_t n, unsigned char* buf, uint32_t mbar)
{
    const uint32_t nr = (n + 7u) & ~7u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic reads of buf first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(mbar), "r"(nr * 10u) : "memory");
    if (nr) {
        const uint32_t d = smem_u32(buf);
        stage_issue(d, s.bin_idx + c * (int64_t)s.bin_cap, nr * 2u, mbar);
        stage_issue(d + kBinStageMax * 2u, s.bin_w + c * (int64_t)s.bin_cap, nr * 8u, mbar);
    }
}

__device__ __forceinline__ void fold_bin(const DevState& s, int64_t c, float4* acc, uint32_t n_raw)
{
    const int chunk_n = 1 << s.bin_shift;
    const uint32_t n = n_raw < s.bin_cap ? n_raw : s.bin_cap;
    const uint16_t* __restrict__ bi = s.bin_idx + c * (int64_t)s.bin_cap;
    const float2* __restrict__ bw = s.bin_w + c * (int64_t)s.bin_cap;
    float* af = reinterpret_cast<float*>(acc);
    uint32_t x[kFoldBatch];
    float2 w[kFoldBatch];
#pragma unroll
    for (int u = 0; u < kFoldBatch; ++u) {
        const uint32_t i = threadIdx.x + u * kStepThreads;
        x[u] = 0u;
        w[u] = make_float2(0.f, 0.f);
        if (i < n) { x[u] = __ldcs(bi + i); w[u] = __ldcs(bw + i); }
    }
    __syncthreads();   // every warp is done with the previous chunk's sums
    for (int i = threadIdx.x; i < chunk_n; i += kStepThreads) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (threadIdx.x == 0 && n_raw) s.bin_cnt[c] = 0u;
    __syncthreads();
    for (uint32_t i0 = 0;; i0 += kStepThreads * kFoldBatch) {
#pragma unroll
        for (int u = 0; u < kFoldBatch; ++u) {
            if (i0 + threadIdx.x + u * kStepThreads < n) {
                float* a = af + ((x[u] & 0x7fffu) << 2) + ((x[u] >> 15) << 1);
                atomicAdd(a, w[u].x);
                atomicAdd(a + 1, w[u].y);
            }
        }
        const uint32_t i1 = i0 + kStepThreads * kFoldBatch;
        if (i1 >= n) break;
#pragma unroll
        for (int u = 0; u < kFoldBatch; ++u) {
            const uint32_t i = i1 + threadIdx.x + u * kStepThreads;
            if (i < n) { x[u] = __ldcs(bi + i); w[u] = __ldcs(bw + i); }
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------ step kernel
// Persistent: the grid is sized to the resident CTAs, and every warp streams a
// contiguous run of 128-neuron tiles (tiles_per_warp of them).  In a tile a
// lane owns neurons n = base + 32 j + lane, j = 0..3: coalesced loads, one
// Philox call per lane (its four words), one bitmask word per j.  Per-subblock
// statistics are kept in registers while consecutive tiles stay in one
// subblock, so the CTA-wide barrier and the done-count happen once per CTA.
// MINB = resident CTAs per SM the register budget is sized for (2: no spills,
// 3: more warps, a few spills); the autotuner picks per network.  FORCED = the
// general form: teacher-forced or input spikes, the I_syn override of the step
// after a property change, gamma-distributed g_ui; the plain form leaves their
// branches out of the neuron update (fewer registers and instructions).
//
// STAGED with kGatherBins (bins of 1024 neurons: one tile per warp per chunk): the
// chunk's eight tiles are in the warps' stage buffers before the fold, and the
// bin's events are added by shared-memory atomics straight into their J planes
// there (no separate sums, two CTA barriers per chunk); the bin's entries are
// loaded while the warps wait for their copies.
template <int GATHER, bool UPDATE, bool FORCED, int MINB = 2, bool STAGED = false>
__global__ void __launch_bounds__(kStepThreads, MINB) k_step(DevState s, int tiles_per_warp)
{
    static_assert(!STAGED || GATHER == 0 || (GATHER == kGatherBins && UPDATE),
                  "staged loads are for the update without gather, or with the bin fold");
    constexpr bool kBinStaged = STAGED && GATHER == kGatherBins;
    constexpr int kWarps = kStepThreads / 32;
    extern __shared__ __align__(128) unsigned char stage_smem[];   // STAGED: [warp][2][kStageBytes]
    __shared__ __align__(8) unsigned long long stage_bar[kWarps][2];
    __shared__ int sh_sub[kWarps];
    __shared__ uint32_t sh_spk[kWarps];
    __shared__ uint32_t sh_nact[kWarps];
    __shared__ double sh_vsum[kWarps];
    __shared__ unsigned long long sh_ev[kWarps];
    __shared__ int sh_last;
    __shared__ uint32_t sh_buf[kWarps];   // kBinStaged: each warp's stage buffer of the chunk (byte offset)
    __shared__ __align__(8) unsigned long long bin_bar[2];   // kBinStaged: the bin buffers' copies

    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int64_t warp_id = (int64_t)blockIdx.x * kWarps + wid;
    const unsigned long long steps_done = s.ctl->steps_done;
    const int64_t ntiles = (s.N + kWarpNeurons - 1) / kWarpNeurons;
    const int64_t tile0 = warp_id * tiles_per_warp;
    const int64_t tile1 = tile0 + tiles_per_warp < ntiles ? tile0 + tiles_per_warp : ntiles;
    // kGatherBins: tiles_per_warp is the number of chunks (2^bin_shift neurons, one push
    // bin each) per CTA.  The CTA folds chunk c's bin into bacc, then warp wid updates
    // tiles wid*tpw_b .. wid*tpw_b + tpw_b - 1 of the chunk.
    float4* bacc = reinterpret_cast<float4*>(stage_smem);
    const int tpw_b = GATHER == kGatherBins ? (1 << (s.bin_shift - 7)) / kWarps : 1;   // bin_shift >= 10
    const int64_t chunk_tiles = (int64_t)tpw_b * kWarps;
    const int64_t bc0 = (int64_t)blockIdx.x * tiles_per_warp;
    int64_t n_iter = tile1 > tile0 ? tile1 - tile0 : 0;
    int64_t bc1 = bc0;
    uint32_t bin_next = 0u;   // count of the next chunk's bin, read one chunk ahead
    if (GATHER == kGatherBins) {
        const int64_t nchunks = (ntiles + chunk_tiles - 1) / chunk_tiles;
        bc1 = bc0 + tiles_per_warp < nchunks ? bc0 + tiles_per_warp : nchunks;
        n_iter = bc1 > bc0 ? (bc1 - bc0) * tpw_b : 0;
        if (bc0 < bc1) bin_next = __ldcg(s.bin_cnt + bc0);
    }

    // update-phase constants (models/block.py:133-142)
    const Ctl* ctl = s.ctl;
    const float t = UPDATE ? __fadd_rn(ctl->t, s.dt) : 0.0f;
    const float noise_rate = ctl->noise_rate;
    const int isolated = ctl->isolated;
    const bool use_override = UPDATE && FORCED && ctl->use_isyn_override != 0u;
    uint32_t* obits = s.bits[steps_done & 1ull];
    const uint32_t* gbits = s.bits[(steps_done - 1ull) & 1ull];

    // warp-level statistics carried across tiles (identical in every lane, except acc_v: each
    // lane's own V sum, reduced over the warp when it is flushed)
    int cur_sub = -1;
    uint32_t acc_spk = 0, acc_nact = 0;
    double acc_v = 0.0;
    unsigned long long acc_ev = 0;
    bool flushed = false;

    // STAGED: whole tiles are copied one ahead into two per-warp buffers (the second J
    // plane must start on 16 bytes: the host stages only split planes with an even stride)
    unsigned char* my_stage = stage_smem + (size_t)wid * 2 * kStageBytes;
    bool stage_off = false;      // a copy was given up on: no more copies from this warp
    int bad_sb = 0;              // ... the buffer it targets and the phase it belongs to
    uint32_t bad_parity = 0;
    if (STAGED) {
        if (lane == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&stage_bar[wid][0])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&stage_bar[wid][1])) : "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int64_t first = kBinStaged ? bc0 * kWarps + wid : tile0;
            if (n_iter > 0 && (first + 1) * kWarpNeurons <= s.N)
                stage_tile(s, first * kWarpNeurons, my_stage, smem_u32(&stage_bar[wid][0]));
        }
        __syncwarp();
    }
    // kBinStaged: counts of the current and next chunk's bins, copies issued per bin buffer,
    // copies given up on (drained at exit); CTA-uniform
    unsigned char* bin_sm = stage_smem + kStagedSmem;
    uint32_t cnt_cur = 0u, cnt_nxt = 0u;
    uint32_t bin_npar = 0u;   // bit b: phase parity of the next copy into bin buffer b
    uint32_t bin_pend = 0u;   // bit b: the latest copy into bin buffer b was given up on
    bool bins_off = false, cur_staged = false;
    if (kBinStaged) {
        if (bc0 < bc1) cnt_cur = __ldcg(s.bin_cnt + bc0);
        if (bc0 + 1 < bc1) cnt_nxt = __ldcg(s.bin_cnt + bc0 + 1);
        if (threadIdx.x == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bin_bar[0])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&bin_bar[1])) : "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            if (bc0 < bc1) stage_bin(s, bc0, bin_stage_n(s, cnt_cur), bin_sm, smem_u32(&bin_bar[0]));
        }
        if (bc0 < bc1) { bin_npar = 1u; cur_staged = true; }
        __syncthreads();   // the barriers' initialisation before any wait
    }

    for (int64_t iter = 0; iter < n_iter; ++iter) {
        int64_t tile = tile0 + iter;
        int64_t bchunk = 0;
        const int it = (int)iter;   // the warp's tile sequence number: stage buffer and phase
        const int sb = it & 1;
        bool staged = false;        // this tile's state is in stage_buf
        unsigned char* stage_buf = my_stage + sb * kStageBytes;
        if (kBinStaged) {   // CTA-uniform: every warp runs the same iterations, one tile each
            bchunk = bc0 + iter;
            tile = bchunk * kWarps + wid;
            const bool have = tile < ntiles;
            const int bb = it & 1;   // bin buffer of this chunk
            // the next chunk's bin entries, into the other bin buffer (its last reader, the
            // previous chunk's fold, finished before the previous barrier)
            const bool nxt_staged = !bins_off && bchunk + 1 < bc1;
            if (nxt_staged) {
                if (threadIdx.x == 0)
                    stage_bin(s, bchunk + 1, bin_stage_n(s, cnt_nxt), bin_sm + (bb ^ 1) * kBinStageBytes,
                              smem_u32(&bin_bar[bb ^ 1]));
                bin_npar ^= 1u << (bb ^ 1);
            }
            const uint32_t n_raw = cnt_cur;
            cnt_cur = cnt_nxt;
            cnt_nxt = bchunk + 2 < bc1 ? __ldcg(s.bin_cnt + bchunk + 2) : 0u;
            const uint32_t nb = n_raw < s.bin_cap ? n_raw : s.bin_cap;
            if (have) {
                const int64_t base = tile * kWarpNeurons;
                if (!stage_off && base + kWarpNeurons <= s.N) {
                    const bool ok = stage_wait(smem_u32(&stage_bar[wid][sb]), (uint32_t)((it >> 1) & 1),
                                               s.stage_wait_limit);
                    staged = __all_sync(0xffffffffu, ok);
                    if (!staged) {   // as below: flag, stop copying, keep off the buffer
                        if (lane == 0) atomicOr(&s.ctl->err, kErrStageTimeout);
                        stage_off = true;
                        bad_sb = sb;
                        bad_parity = (uint32_t)((it >> 1) & 1);
                    }
                }
                if (stage_off && sb == bad_sb) stage_buf = my_stage + (sb ^ 1) * kStageBytes;
                if (!staged) {   // a partial tile, or a copy given up on: the lanes load it
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int k = j * 32 + lane;
                        const int64_t n = base + k;
                        if (n >= s.N) continue;
                        reinterpret_cast<float*>(stage_buf)[k] = __ldcs(s.V + n);
                        reinterpret_cast<float*>(stage_buf + kWarpNeurons * 4)[k] = __ldcs(s.tlast + n);
                        reinterpret_cast<float2*>(stage_buf + kWarpNeurons * 8)[k] = __ldcs(s.J2 + n);
                        reinterpret_cast<float2*>(stage_buf + kWarpNeurons * 16)[k] = __ldcs(s.J2 + s.j_ps + n);
                    }
                }
                // the next chunk's tile of this warp, into the buffer this warp has finished with
                const int64_t nt = tile + kWarps;
                if (!stage_off && lane == 0 && iter + 1 < n_iter && (nt + 1) * kWarpNeurons <= s.N)
                    stage_tile(s, nt * kWarpNeurons, my_stage + (sb ^ 1) * kStageBytes,
                               smem_u32(&stage_bar[wid][sb ^ 1]));
            }
            if (lane == 0) sh_buf[wid] = (uint32_t)(stage_buf - stage_smem);
            // this chunk's staged bin entries (every thread waits: the copies' data is then
            // visible to it), and every tile of the chunk staged
            bool ok = true;
            if (cur_staged)
                ok = stage_wait(smem_u32(&bin_bar[bb]), ((bin_npar >> bb) & 1u) ^ 1u, s.stage_wait_limit);
            const bool bad = __syncthreads_or(!ok);
            uint32_t n_st = 0u;
            if (cur_staged) {
                if (bad) {   // given up on: the entries come from global memory, no more bin copies
                    if (threadIdx.x == 0) atomicOr(&s.ctl->err, kErrStageTimeout);
                    bins_off = true;
                    bin_pend |= 1u << bb;
                } else {
                    n_st = bin_stage_n(s, n_raw);
                }
            }
            cur_staged = nxt_staged;
            if (threadIdx.x == 0 && n_raw) s.bin_cnt[bchunk] = 0u;
            // fold: entry = local neuron (10 bits: warp, lane-neuron) | kind << 15, added into the
            // staged J planes
            auto fold_add = [&](uint32_t x, float2 w) {
                const uint32_t l = x & 0x3ffu;
                float* a = reinterpret_cast<float*>(stage_smem + sh_buf[l >> 7] + kWarpNeurons * 8 +
                                                    (x >> 15) * (kWarpNeurons * 8)) + 2 * (l & 127u);
                atomicAdd(a, w.x);
                atomicAdd(a + 1, w.y);
            };
            {
                const uint16_t* sbi = reinterpret_cast<const uint16_t*>(bin_sm + bb * kBinStageBytes);
                const float2* sbw = reinterpret_cast<const float2*>(bin_sm + bb * kBinStageBytes + kBinStageMax * 2);
                for (uint32_t i = threadIdx.x; i < n_st; i += kStepThreads) fold_add(sbi[i], sbw[i]);
            }
            if (nb > n_st) {   // the rest of the bin from global memory, kFoldBatch entries per thread in flight
                const uint16_t* __restrict__ bi = s.bin_idx + bchunk * (int64_t)s.bin_cap;
                const float2* __restrict__ bw = s.bin_w + bchunk * (int64_t)s.bin_cap;
                for (uint32_t i0 = n_st; i0 < nb; i0 += kStepThreads * kFoldBatch) {
                    uint32_t x[kFoldBatch];
                    float2 w[kFoldBatch];
#pragma unroll
                    for (int u = 0; u < kFoldBatch; ++u) {
                        const uint32_t i = i0 + threadIdx.x + u * kStepThreads;
                        x[u] = 0u;
                        w[u] = make_float2(0.f, 0.f);
                        if (i < nb) { x[u] = __ldcs(bi + i); w[u] = __ldcs(bw + i); }
                    }
#pragma unroll
                    for (int u = 0; u < kFoldBatch; ++u)
                        if (i0 + threadIdx.x + u * kStepThreads < nb) fold_add(x[u], w[u]);
                }
            }
            __syncthreads();   // the chunk's events are in the staged J planes
            staged = true;
            if (!have) continue;
        } else if (GATHER == kGatherBins) {   // CTA-uniform: every warp runs the same iterations
            const int64_t ci = iter / tpw_b;
            const int jj = (int)(iter - ci * tpw_b);
            bchunk = bc0 + ci;
            if (jj == 0) {
                const uint32_t n_raw = bin_next;
                if (bchunk + 1 < bc1) bin_next = __ldcg(s.bin_cnt + bchunk + 1);
                fold_bin(s, bchunk, bacc, n_raw);
            }
            tile = bchunk * chunk_tiles + (int64_t)wid * tpw_b + jj;
            if (tile >= ntiles) continue;
        }
        const int64_t base = tile * kWarpNeurons;
        float4 Jn[4];
        if (STAGED && !kBinStaged) {
            if (!stage_off && base + kWarpNeurons <= s.N) {
                const bool ok = stage_wait(smem_u32(&stage_bar[wid][sb]), (uint32_t)((it >> 1) & 1),
                                           s.stage_wait_limit);
                staged = __all_sync(0xffffffffu, ok);
                if (!staged) {
                    // copy given up on: flag it, issue no further copies, and keep off its
                    // buffer (the copy may still land there) until the drain at exit
                    if (lane == 0) atomicOr(&s.ctl->err, kErrStageTimeout);
                    stage_off = true;
                    bad_sb = sb;
                    bad_parity = (uint32_t)((it >> 1) & 1);
                }
            }
            if (stage_off && sb == bad_sb) stage_buf = my_stage + (sb ^ 1) * kStageBytes;
            // the next tile's copy, into the buffer the previous tile has finished with
            if (!stage_off && lane == 0 && tile + 1 < tile1 && (tile + 2) * kWarpNeurons <= s.N)
                stage_tile(s, base + kWarpNeurons, my_stage + (sb ^ 1) * kStageBytes,
                           smem_u32(&stage_bar[wid][sb ^ 1]));
        }
        if (GATHER == kGatherMasks) {
            // The warp lists every marked pull entry of its 128 neurons (a lane's entries
            // contiguous, neuron by neuron, excitatory then inhibitory, ascending position),
            // loads their weights together, then every lane adds its own in that order.
            uint16_t* lrel = reinterpret_cast<uint16_t*>(stage_smem + (size_t)wid * kMaskList * 10);
            float2* lw = reinterpret_cast<float2*>(stage_smem + (size_t)wid * kMaskList * 10 + kMaskList * 2);
            const int64_t rbase = __ldg(s.prow + base);             // entries relative to the tile's first row
            uint4 mx[4], mi[4];
            int nx[4], ni[4];
            int mine = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                mx[j] = mi[j] = make_uint4(0u, 0u, 0u, 0u);
                if (n < s.N) {
                    uint4* pm = reinterpret_cast<uint4*>(s.pmask + n * (2 * kMaskWords));
                    mx[j] = __ldcs(pm);
                    mi[j] = __ldcs(pm + 1);
                }
                nx[j] = __popc(mx[j].x) + __popc(mx[j].y) + __popc(mx[j].z) + __popc(mx[j].w);
                ni[j] = __popc(mi[j].x) + __popc(mi[j].y) + __popc(mi[j].z) + __popc(mi[j].w);
                mine += nx[j] + ni[j];
            }
            int incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            const bool listed = total <= kMaskList;
            float4 sum[4];
            if (listed) {
                int at = incl - mine;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (nx[j] + ni[j] == 0) continue;
                    const int64_t n = base + j * 32 + lane;
                    const uint32_t rel0 = (uint32_t)(__ldg(s.prow + n) - rbase);
#pragma unroll
                    for (int kind = 0; kind < 2; ++kind) {
                        const uint4 m4 = kind ? mi[j] : mx[j];
                        const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
                        for (int wi = 0; wi < 4; ++wi) {
                            uint32_t word = mw[wi];
                            while (word) {
                                const int bit = __ffs(word) - 1;
                                word &= word - 1u;
                                lrel[at++] = (uint16_t)(rel0 + (uint32_t)(wi * 32 + bit));
                            }
                        }
                    }
                }
                __syncwarp();
                const float2* __restrict__ pwt = s.pw + rbase;
                for (int i = lane; i < total; i += 32) lw[i] = __ldg(pwt + lrel[i]);
                __syncwarp();
                int rd = incl - mine;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
                    for (int k = 0; k < nx[j]; ++k) { const float2 w = lw[rd++]; a.x = __fadd_rn(a.x, w.x); a.y = __fadd_rn(a.y, w.y); }
                    for (int k = 0; k < ni[j]; ++k) { const float2 w = lw[rd++]; a.z = __fadd_rn(a.z, w.x); a.w = __fadd_rn(a.w, w.y); }
                    sum[j] = a;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (n >= s.N) continue;
                if (nx[j] + ni[j]) {
                    uint4* pm = reinterpret_cast<uint4*>(s.pmask + n * (2 * kMaskWords));
                    pm[0] = make_uint4(0u, 0u, 0u, 0u);
                    pm[1] = make_uint4(0u, 0u, 0u, 0u);
                    if (!listed) sum[j] = mask_sum(s, n, mx[j], mi[j]);   // a tile with many inputs
                } else {
                    sum[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                Jn[j] = add4(load_J(s, n), sum[j]);   // models/block.py:71-73
            }
            __syncwarp();   // the list is reused by the next tile
            if (!UPDATE) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t n = base + j * 32 + lane;
                    if (n < s.N) store_J(s, n, Jn[j]);
                }
                continue;
            }
        } else if (GATHER == kGatherSlots) {
            float4 sum[4];
            uint32_t ovf = 0u;   // bit j: neuron j of this lane got more contributions than slots
            // counts of the lane's four neurons, then their first two slots, all in flight together
            uint32_t cnt[4];
            uint4 s0[4], s1[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                cnt[j] = n < s.N ? __ldcs(s.slot_cnt + n) : 0u;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                sum[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                s0[j] = s1[j] = make_uint4(0u, 0u, 0u, 0u);
                if (cnt[j]) s.slot_cnt[n] = 0u;
                if (cnt[j] >= 1u && cnt[j] <= kSlotCap) s0[j] = __ldcs(s.slots + n * kSlotCap);
                if (cnt[j] == 2u) s1[j] = __ldcs(s.slots + n * kSlotCap + 1);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (cnt[j] == 0u) continue;
                if (cnt[j] > kSlotCap) ovf |= 1u << j;
                else if (cnt[j] <= 2u) sum[j] = slot_pair_sum(s0[j], s1[j], cnt[j]);
                else sum[j] = slot_sum(s.slots + n * kSlotCap, cnt[j]);
            }
            // overflowing rows: the warp gathers them whole, in row order
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                unsigned m = __ballot_sync(0xffffffffu, (ovf >> j) & 1u);
                while (m) {
                    const int l = __ffs(m) - 1;
                    m &= m - 1;
                    uint32_t ev = 0;
                    const float4 a = gather_row(s, gbits, base + j * 32 + l, lane, ev);
                    if (lane == l) sum[j] = a;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (n < s.N) Jn[j] = add4(load_J(s, n), sum[j]);   // models/block.py:71-73
            }
            if (!UPDATE) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t n = base + j * 32 + lane;
                    if (n < s.N) store_J(s, n, Jn[j]);
                }
                continue;
            }
        } else if (GATHER == kGatherStream) {
            // The warp streams the pull entries of its 128 rows in 32-entry chunks (coalesced
            // index loads, 4 chunks in flight), tests their presynaptic bits and, for the
            // firing ones, adds the weights to the row sums in entry order: the row order of
            // gather_row, for every row at once.  Lane 0 does the (rare) additions.
            int64_t* rp = reinterpret_cast<int64_t*>(stage_smem + (size_t)wid * kStreamWarpBytes);
            float4* acc = reinterpret_cast<float4*>(stage_smem + (size_t)wid * kStreamWarpBytes + 129 * 8 + 8);
            const int nrows = (int)(s.N - base < kWarpNeurons ? s.N - base : kWarpNeurons);
            for (int i = lane; i <= nrows; i += 32) rp[i] = __ldg(s.prow + base + i);
            for (int i = lane; i < kWarpNeurons; i += 32) acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            __syncwarp();
            const int64_t e0 = rp[0], e1 = rp[nrows];
            uint32_t events = 0;
            constexpr int UC = 4;
            for (int64_t c = e0; c < e1; c += 32 * UC) {
                uint32_t col[UC];
                bool act[UC];
#pragma unroll
                for (int u = 0; u < UC; ++u) {
                    const int64_t e = c + u * 32 + lane;
                    col[u] = e < e1 ? __ldcs(s.pcol + e) : 0u;
                }
#pragma unroll
                for (int u = 0; u < UC; ++u) {
                    const int64_t e = c + u * 32 + lane;
                    act[u] = e < e1 && test_bit(gbits, col[u] & kIndexMask);
                }
#pragma unroll
                for (int u = 0; u < UC; ++u) {
                    unsigned m = __ballot_sync(0xffffffffu, act[u]);
                    if (!m) continue;
                    const int64_t e = c + u * 32 + lane;
                    float2 w = make_float2(0.f, 0.f);
                    int r = 0;
                    if (act[u]) {
                        w = __ldg(s.pw + e);
                        int lo = 0, hi = nrows;              // rp[lo] <= e < rp[hi]
                        while (hi - lo > 1) {
                            const int mid = (lo + hi) >> 1;
                            if (rp[mid] <= e) lo = mid; else hi = mid;
                        }
                        r = lo;
                    }
                    events += __popc(m);
                    while (m) {
                        const int l = __ffs(m) - 1;
                        m &= m - 1;
                        const float wx = __shfl_sync(0xffffffffu, w.x, l);
                        const float wy = __shfl_sync(0xffffffffu, w.y, l);
                        const uint32_t cl = __shfl_sync(0xffffffffu, col[u], l);
                        const int rl = __shfl_sync(0xffffffffu, r, l);
                        if (lane == 0) {
                            float4 a = acc[rl];
                            if (cl & kKindBit) { a.z = __fadd_rn(a.z, wx); a.w = __fadd_rn(a.w, wy); }
                            else { a.x = __fadd_rn(a.x, wx); a.y = __fadd_rn(a.y, wy); }
                            acc[rl] = a;
                        }
                    }
                }
            }
            __syncwarp();
            acc_ev += events;   // synaptic events of the step gathered
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (n < s.N) Jn[j] = add4(load_J(s, n), acc[j * 32 + lane]);   // models/block.py:71-73
            }
            __syncwarp();   // the row pointers and sums are rewritten by the next tile
            if (!UPDATE) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t n = base + j * 32 + lane;
                    if (n < s.N) store_J(s, n, Jn[j]);
                }
                continue;
            }
        } else if (GATHER == kGatherBins && !kBinStaged) {
            const float4* acc = bacc + (base - bchunk * chunk_tiles * kWarpNeurons);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (n < s.N) Jn[j] = add4(load_J(s, n), acc[j * 32 + lane]);
            }
            if (!UPDATE) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t n = base + j * 32 + lane;
                    if (n < s.N) store_J(s, n, Jn[j]);
                }
                continue;
            }
        } else if (GATHER == kGatherRows) {
            float4 sum[4];
            uint32_t events = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                sum[j] = make_float4(0.f, 0.f, 0.f, 0.f);
                for (int r = 0; r < 32; ++r) {
                    const int64_t n = base + j * 32 + r;
                    if (n >= s.N) break;
                    const float4 a = gather_row(s, gbits, n, lane, events);
                    if (lane == r) sum[j] = a;
                }
            }
            acc_ev += events;   // synaptic events of the step gathered
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t n = base + j * 32 + lane;
                if (n < s.N) Jn[j] = add4(load_J(s, n), sum[j]);   // models/block.py:71-73
            }
            if (!UPDATE) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int64_t n = base + j * 32 + lane;
                    if (n < s.N) store_J(s, n, Jn[j]);
                }
                continue;
            }
        }

        // ---- update of step `steps_done`
        // Phase 1: every load of the lane's four neurons before any store, so their
        // latencies overlap (the stores below could alias them).  Streaming hints:
        // the state is touched once per step.
        bool valid[4];
        float v_in[4], tl_in[4];
        float4 J_in[4];
        uint32_t c_in[4];
        const uint32_t tcls = s.tile_cls ? __ldg(s.tile_cls + tile) : kMixedTile;   // the tile's class, or kMixedTile
        const bool mixed = tcls == kMixedTile;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t n = base + j * 32 + lane;
            valid[j] = n < s.N;
            c_in[j] = 0u;          // class 0 exists whenever N > 0: keeps the shuffle below in bounds
            if (valid[j]) {
                if (STAGED) {
                    // the tile's state lives in the stage buffer: the copies' (or, for a
                    // partial tile, this lane's own loads, written below)
                    if (!staged) {
                        const int k = j * 32 + lane;
                        reinterpret_cast<float*>(stage_buf)[k] = __ldcs(s.V + n);
                        reinterpret_cast<float*>(stage_buf + kWarpNeurons * 4)[k] = __ldcs(s.tlast + n);
                        reinterpret_cast<float2*>(stage_buf + kWarpNeurons * 8)[k] = __ldcs(s.J2 + n);
                        reinterpret_cast<float2*>(stage_buf + kWarpNeurons * 16)[k] = __ldcs(s.J2 + s.j_ps + n);
                    }
                } else {
                    v_in[j] = __ldcs(s.V + n);
                    tl_in[j] = __ldcs(s.tlast + n);
                    c_in[j] = mixed ? __ldcs(s.cls + n) : tcls;
                    if (!GATHER) J_in[j] = load_J(s, n);
                }
            }
        }
        if (STAGED) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                c_in[j] = !valid[j] ? 0u
                          : mixed   ? __ldcs(s.cls + base + j * 32 + lane)
                                    : tcls;
        }
        // Noise words: counter {tile*32 + lane, stream, step}; inside an ensemble the
        // tile and stream are the member's own (members start on 128-neuron tiles),
        // so a member draws the same noise as when it is simulated alone.
        const uint32_t c0 = __shfl_sync(0xffffffffu, c_in[0], 0);
        uint64_t qtile = (uint64_t)tile;
        uint32_t stream = s.stream_id;
        if (s.member_start) {
            const int m = __ldg(&s.pc[c0].member);
            if (m >= 0) {
                qtile = (uint64_t)((base - __ldg(s.member_start + m)) / kWarpNeurons);
                stream += (uint32_t)m;
            }
        }
        const U4 rnd = philox4x32_10(U4{(uint32_t)(qtile * 32 + lane), stream, (uint32_t)steps_done,
                                        (uint32_t)(steps_done >> 32)},
                                     (uint32_t)s.seed, (uint32_t)(s.seed >> 32));
        const uint32_t words[4] = {rnd.x, rnd.y, rnd.z, rnd.w};

        // Phase 2: arithmetic (models/block.py:83-111 order), each neuron stored as
        // soon as it is computed (all loads were issued above).  When the tile's 128
        // neurons share one parameter class (classes are region x E/I ranges), the
        // class is loaded once for the warp.
        uint32_t act_m = 0, nav_m = 0;      // bit j: neuron j of this lane
        int mysub0 = -1;
        bool lane_uni = true;               // all of this lane's valid neurons in mysub0
        double vsum_lane = 0.0;
        auto neuron = [&](int j, const ParamClass& p) {
            const int64_t n = base + j * 32 + lane;
            float v, tl;
            float4 J;
            if (STAGED) {
                const int k = j * 32 + lane;
                v = reinterpret_cast<const float*>(stage_buf)[k];
                tl = reinterpret_cast<const float*>(stage_buf + kWarpNeurons * 4)[k];
                const float2 a = reinterpret_cast<const float2*>(stage_buf + kWarpNeurons * 8)[k];
                const float2 b2 = reinterpret_cast<const float2*>(stage_buf + kWarpNeurons * 16)[k];
                J = make_float4(a.x, a.y, b2.x, b2.y);
            } else {
                v = v_in[j];
                tl = tl_in[j];
                J = GATHER ? Jn[j] : J_in[j];
            }
            float isyn;
            if (FORCED) {   // the general form: the I_syn override, gamma-distributed g_ui
                if (use_override) isyn = s.isyn_override[n];
                else if (s.gnrn) isyn = isyn_g(mul4(p.g, __ldcs(s.gnrn + n)), p.Vu, v, J);
                else isyn = isyn_of(p, v, J);
            } else {
                isyn = isyn_of(p, v, J);
            }
            const float mainp = __fmul_rn(-p.gL, __fsub_rn(v, p.VL));
            const float cd = __fadd_rn(__fadd_rn(mainp, isyn), p.Iext);
            const float vn = __fadd_rn(v, __fmul_rn(p.rCdt, cd));
            const bool notsat = t >= __fadd_rn(tl, p.Tref);
            const float vs = notsat ? vn : p.Vreset;
            bool a = vs >= p.Vth;
            // torch.minimum(vs, V_th): NaN when either is NaN (one compare-or-NaN test and a select)
            const float vmin = (vs < p.Vth || isnan(vs)) ? vs : p.Vth;
            if (FORCED && s.forced_active && (!s.forced_mask || ((__ldg(s.forced_mask + (n >> 5)) >> (n & 31)) & 1u)))
                a = (__ldg(s.forced_active + (n >> 5)) >> (n & 31)) & 1u;
            const float rate = noise_rate >= 0.0f ? noise_rate : p.noise;
            const bool nz = u01(words[j]) < rate;
            bool na = isolated ? nz : (nz || a);
            if (FORCED && s.forced_new) na = (__ldg(s.forced_new + (n >> 5)) >> (n & 31)) & 1u;
            __stcs(s.V + n, vmin);
            store_J(s, n, mul4(J, p.decay));
            if (a) s.tlast[n] = t;
            act_m |= (uint32_t)a << j;
            nav_m |= (uint32_t)na << j;
            if (j == 0) mysub0 = p.sub;
            else if (p.sub != mysub0) lane_uni = false;
            vsum_lane += (double)vmin;
            if (p.sub < 0 || p.sub >= s.n_sub) {
                lane_uni = false;
                if (na) atomicAdd(s.unmapped_nact, 1u);
            }
        };
        bool same = true;   // a tile of one class (known from the tile table, or checked)
        if (mixed) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (valid[j]) same = same && (c_in[j] == c0);
        }
        if (!mixed || __all_sync(0xffffffffu, same)) {
            // one class for the warp's tile, loaded once into registers (a per-warp shared
            // copy read field by field measured slower: 0.230 against 0.224 ms)
            const ParamClass p = load_class(s.pc, c0);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (valid[j]) neuron(j, p);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (valid[j]) neuron(j, s.pc[c_in[j]]);   // fields read from the (L1-cached) table as used
        }

        uint32_t cnt_spk = 0, cnt_nact = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t ma = __ballot_sync(0xffffffffu, (act_m >> j) & 1u);
            const uint32_t mn = __ballot_sync(0xffffffffu, (nav_m >> j) & 1u);
            const int64_t wi = tile * 4 + j;
            if (lane == 0) { s.abits[wi] = ma; obits[wi] = mn; }
            cnt_spk += __popc(ma);
            cnt_nact += __popc(mn);
        }

        // ---- per-subblock statistics
        const int sub0 = __shfl_sync(0xffffffffu, mysub0, 0);
        const bool uni = __all_sync(0xffffffffu, lane_uni && (mysub0 == sub0 || !valid[0])) && sub0 >= 0 &&
                         sub0 < s.n_sub;
        if (uni) {
            // the V sum stays per lane across the subblock's tiles; the warp reduces it when
            // the subblock changes and at the end
            if (sub0 != cur_sub) {
                double vw = acc_v;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) vw += __shfl_xor_sync(0xffffffffu, vw, o);
                if (cur_sub >= 0 && lane == 0) {
                    atomicAdd(s.sub_spk + cur_sub, acc_spk);
                    atomicAdd(s.sub_nact + cur_sub, acc_nact);
                    atomicAdd(s.sub_vsum + cur_sub, vw);
                    flushed = true;
                }
                cur_sub = sub0; acc_spk = 0; acc_nact = 0; acc_v = 0.0;
            }
            acc_spk += cnt_spk; acc_nact += cnt_nact; acc_v += vsum_lane;
        } else {
            // mixed subblocks in this tile: per-neuron atomics (classes re-read from L1)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (!valid[j]) continue;
                const int sb = s.pc[c_in[j]].sub;
                if (sb >= 0 && sb < s.n_sub) {
                    if ((act_m >> j) & 1u) atomicAdd(s.sub_spk + sb, 1u);
                    if ((nav_m >> j) & 1u) atomicAdd(s.sub_nact + sb, 1u);
                    atomicAdd(s.sub_vsum + sb, (double)__ldcg(s.V + base + j * 32 + lane));
                }
            }
            __threadfence();   // this lane's atomics before the CTA's done-count
        }
        if (STAGED) __syncwarp();   // every lane is done with the buffer before lane 0 refills it
    }
    if (flushed) __threadfence();
    if (kBinStaged && threadIdx.x == 0) {
        // bin copies given up on must land before this CTA's shared memory is released
#pragma unroll
        for (int b = 0; b < 2; ++b)
            if (((bin_pend >> b) & 1u) && !stage_wait(smem_u32(&bin_bar[b]), ((bin_npar >> b) & 1u) ^ 1u, 1u << 22))
                atomicOr(&s.ctl->err, kErrStageDrain);
    }
    if (STAGED && stage_off) {
        // a copy given up on must land before this CTA's shared memory is released
        if (lane == 0 && !stage_wait(smem_u32(&stage_bar[wid][bad_sb]), bad_parity, 1u << 22))
            atomicOr(&s.ctl->err, kErrStageDrain);
        __syncwarp();
    }

    // ---- CTA merge: one barrier, one set of atomics, one done-count per CTA
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc_v += __shfl_xor_sync(0xffffffffu, acc_v, o);   // the lanes' V sums
    if (lane == 0) { sh_sub[wid] = cur_sub; sh_spk[wid] = acc_spk; sh_nact[wid] = acc_nact; sh_vsum[wid] = acc_v; sh_ev[wid] = acc_ev; }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long ev = 0;
        int cur = -1; uint32_t cs = 0, cn = 0; double cv = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            ev += sh_ev[w];
            const int sb = sh_sub[w];
            if (!UPDATE || sb < 0) continue;
            if (sb != cur) {
                if (cur >= 0) {
                    atomicAdd(s.sub_spk + cur, cs); atomicAdd(s.sub_nact + cur, cn); atomicAdd(s.sub_vsum + cur, cv);
                }
                cur = sb; cs = 0; cn = 0; cv = 0.0;
            }
            cs += sh_spk[w]; cn += sh_nact[w]; cv += sh_vsum[w];
        }
        if (cur >= 0) { atomicAdd(s.sub_spk + cur, cs); atomicAdd(s.sub_nact + cur, cn); atomicAdd(s.sub_vsum + cur, cv); }
        add_events(s, ev, blockIdx.x);
        // the plain form (FORCED false) has neither the I_syn override nor gamma g_ui: the host
        // routes such steps to the general form; a step that reached the plain one is flagged
        // (read before the done-count: the last CTA's epilogue clears the override flag)
        if (UPDATE && !FORCED && (s.ctl->use_isyn_override != 0u || s.gnrn != nullptr))
            atomicOr(&s.ctl->err, kErrGeneralSkipped);
        if (UPDATE) {
            __threadfence();   // the CTA's statistics before its done-count
            const unsigned prev = atomicAdd(&s.ctl->done, 1u);
            sh_last = (prev == gridDim.x - 1u);
        }
    }
    if (!UPDATE) return;
    __syncthreads();
    if (sh_last) {
        __threadfence();
        step_epilogue(s, steps_done, t);
    }
}

// ------------------------------------------------------------ push scatter
// cuda/src/stage/presynaptic_voltage.cpp:152-266 restated for one device.
// A warp owns `wpw` bitmask words (32*wpw presynaptic neurons).  It lists the
// set bits in shared memory, then takes them 32 rows at a time: every lane
// loads one row's bounds, a warp scan turns the row lengths into offsets, and
// the lanes walk the concatenated synapses of the 32 rows together (four
// independent index/weight loads in flight per lane), each synapse adding its
// weight pair to the pending J with one float2 atomic.  The synapse stream is
// read with evict-first hints so it does not push the J lines out of L2; a
// small `wpw` keeps the rows scattered at any moment inside a narrow window
// of neurons, whose intra-region targets then share L2-resident J lines.  No
// CTA-wide barrier; the synaptic events (row lengths) are counted per warp.
constexpr int kScatterThreads = 256;
constexpr int kScatterMaxWords = 32;

constexpr int kScatterUnroll = 8;   // synapses in flight per lane
constexpr int kScatterJ = 0, kScatterSlots = 1, kScatterMasks = 2;

// MINB: resident CTAs per SM the registers are budgeted for; the row lists take
// wpw * 32 entries per warp of dynamic shared memory.
template <int MODE, int MINB = 1>
__global__ void __launch_bounds__(kScatterThreads, MINB) k_scatter(DevState s, int wpw)
{
    extern __shared__ uint32_t sh_rows_dyn[];
    const unsigned long long steps_done = s.ctl->steps_done;
    const uint32_t* __restrict__ bits = s.bits[(steps_done - 1ull) & 1ull];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    // rev_scatter: CTAs take the bitmask from its end, so that the first rows scattered
    // target the neurons the update wrote last, whose J lines may still be in L2
    const int64_t bid = s.rev_scatter ? (int64_t)(gridDim.x - 1u - blockIdx.x) : (int64_t)blockIdx.x;
    const int64_t warp_global = (bid * blockDim.x + threadIdx.x) >> 5;
    const int64_t w0 = warp_global * wpw;
    uint32_t* rows = sh_rows_dyn + (size_t)wid * wpw * 32;
    uint32_t word = (lane < wpw && w0 + lane < s.n_words) ? __ldcs(bits + w0 + lane) : 0u;
    // list the set bits of the window in neuron order
    const int cnt = __popc(word);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int pos = incl - cnt;
    while (word) {
        const int b = __ffs(word) - 1;
        word &= word - 1;
        rows[pos++] = (uint32_t)((w0 + lane) * 32 + b);
    }
    __syncwarp();
    unsigned long long warp_events = 0;
    for (int r0 = 0; r0 < total; r0 += 32) {
        const bool has = r0 + lane < total;
        int64_t e0 = 0, len = 0;
        if (has) {
            const uint32_t pre = rows[r0 + lane];
            e0 = __ldcs(s.qrow + pre);
            len = __ldcs(s.qrow + pre + 1) - e0;
        }
        // inclusive scan of the row lengths
        int64_t off = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, off, o);
            if (lane >= o) off += y;
        }
        const int64_t T = __shfl_sync(0xffffffffu, off, 31);
        warp_events += (unsigned long long)T;
        const int64_t start = off - len;           // exclusive offset of this lane's row
        for (int64_t v0 = 0; v0 < T; v0 += 32 * kScatterUnroll) {
            uint32_t c[kScatterUnroll];
            float2 w[kScatterUnroll];
            uint32_t ppos[kScatterUnroll];
            bool ok[kScatterUnroll];
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const int64_t v = v0 + u * 32 + lane;
                // row of v: number of rows whose inclusive offset is <= v
                int lo = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1) {
                    const int64_t val = __shfl_sync(0xffffffffu, off, lo + step - 1);
                    if (val <= v) lo += step;
                }
                const int src = lo < 31 ? lo : 31;
                const int64_t rs = __shfl_sync(0xffffffffu, start, src);
                const int64_t re0 = __shfl_sync(0xffffffffu, e0, src);
                ok[u] = v < T;
                if (ok[u]) {
                    const int64_t e = re0 + (v - rs);
                    c[u] = __ldcs(s.qcol + e);
                    if (MODE != kScatterMasks) w[u] = __ldcs(s.qw + e);
                    if (MODE != kScatterJ) ppos[u] = __ldcs(s.qpos + e);
                }
            }
            if (MODE == kScatterMasks) {
#pragma unroll
                for (int u = 0; u < kScatterUnroll; ++u)
                    if (ok[u])
                        atomicOr(s.pmask + (int64_t)(c[u] & kIndexMask) * (2 * kMaskWords) +
                                     ((c[u] & kKindBit) ? kMaskWords : 0) + (ppos[u] >> 5),
                                 1u << (ppos[u] & 31));
            } else if (MODE == kScatterSlots) {
                // every slot claim of the batch first, so their round trips overlap
                uint32_t k[kScatterUnroll];
#pragma unroll
                for (int u = 0; u < kScatterUnroll; ++u)
                    k[u] = ok[u] ? atomicAdd(s.slot_cnt + (c[u] & kIndexMask), 1u) : kSlotCap;
#pragma unroll
                for (int u = 0; u < kScatterUnroll; ++u)
                    if (k[u] < kSlotCap)
                        __stcg(s.slots + (int64_t)(c[u] & kIndexMask) * kSlotCap + k[u],
                               make_uint4(ppos[u] | (c[u] & kKindBit), 0u, __float_as_uint(w[u].x),
                                          __float_as_uint(w[u].y)));
            } else {
#pragma unroll
                for (int u = 0; u < kScatterUnroll; ++u)
                    if (ok[u])
                        atomicAdd(s.J2 + (int64_t)(c[u] >> 31) * s.j_ps + (int64_t)(c[u] & kIndexMask) * s.j_es, w[u]);
            }
        }
    }
    if (lane == 0) add_events(s, warp_events, (uint32_t)warp_global);
}

// ------------------------------------------------------------ binned push scatter
// cuda/src/stage/presynaptic_voltage.cpp:152-266 (every synapse of a firing row
// adds its weight pair to its postsynaptic neuron), with the additions staged:
// instead of one L2 float atomic per synaptic event, events are appended to the
// bin of their postsynaptic neuron (2^bin_shift neurons per bin) and the next
// update folds each bin in shared memory (fold_bin).
//
// A persistent CTA takes rounds of `wpr` bitmask words (grid-strided), lists the
// round's firing rows and their bounds in shared memory, and walks the
// concatenated synapses of those rows in slices of kBinSlice events (8 per
// thread, coalesced index/weight loads).  Bins within a window of kBinWin bins
// around the round's own neurons (the neuron's region and its neighbours: most
// synapses stay inside the region) are staged: shared-memory atomics rank every
// event inside its bin, a CTA-wide scan of the window's counts gives each bin its
// run in a shared staging buffer, one global atomic per bin reserves the run in
// the bin, and the runs are written out coalesced.  Events outside the window, or
// past their bin's capacity, go to J with a float2 atomic.
constexpr int kBinThreads = 256;
constexpr int kBinEPT = 8;                                  // events per thread and slice
constexpr int kBinSlice = kBinThreads * kBinEPT;            // 2048
constexpr int kBinMaxWords = 256;                           // bitmask words per round (one per thread)
constexpr int kBinMaxRows = 2048;                           // firing rows listed at once (a sub-round)
constexpr int kBinWin = 1024;                               // bins staged per round
constexpr int kBinWinPerThread = kBinWin / kBinThreads;
constexpr uint32_t kBinSkip = 0xffffffffu;

// Dynamic shared memory of k_bin_scatter (offsets multiples of 16).
constexpr int kBinOffW = 0;                                               // float2 [kBinSlice]
constexpr int kBinOffE0 = kBinOffW + 8 * kBinSlice;                       // u32 [kBinMaxRows], rel. to the round's first row
constexpr int kBinOffRow = kBinOffE0 + 4 * kBinMaxRows;                   // i32 [kBinMaxRows + 1]
constexpr int kBinOffDst = kBinOffRow + ((4 * (kBinMaxRows + 1) + 15) & ~15);   // u32 [kBinSlice]
constexpr int kBinOffCnt = kBinOffDst + 4 * kBinSlice;                    // u32 [kBinWin] counts, then run offsets
constexpr int kBinOffG = kBinOffCnt + 4 * kBinWin;                        // u32 [kBinWin] run position in the bin
constexpr int kBinOffIdx = kBinOffG + 4 * kBinWin;                        // u16 [kBinSlice]
constexpr int kBinSmem = kBinOffIdx + 2 * kBinSlice;                      // 53264 bytes: four CTAs per SM

// Exclusive prefix sum over the CTA (kBinThreads threads); *total gets the sum.
__device__ __forceinline__ int bin_block_scan(int v, int* sh_warp, int* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sh_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int x = lane < kBinThreads / 32 ? sh_warp[lane] : 0;
        int xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, xi, o);
            if (lane >= o) xi += y;
        }
        if (lane < kBinThreads / 32) sh_warp[lane] = xi - x;   // exclusive warp offsets
        if (lane == 31) sh_warp[kBinThreads / 32] = xi;
    }
    __syncthreads();
    const int r = sh_warp[wid] + incl - v;
    *total = sh_warp[kBinThreads / 32];
    __syncthreads();   // sh_warp is reused by the next scan
    return r;
}

__global__ void __launch_bounds__(kBinThreads, 4) k_bin_scatter(DevState s, int wpr)
{
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ int sh_warp[kBinThreads / 32 + 1];
    float2* st_w = reinterpret_cast<float2*>(bsm + kBinOffW);
    uint32_t* row_e0 = reinterpret_cast<uint32_t*>(bsm + kBinOffE0);
    int32_t* row_off = reinterpret_cast<int32_t*>(bsm + kBinOffRow);
    uint32_t* st_dst = reinterpret_cast<uint32_t*>(bsm + kBinOffDst);
    uint32_t* row_pre = st_dst;                                    // listing only (before the slices)
    uint32_t* w_cnt = reinterpret_cast<uint32_t*>(bsm + kBinOffCnt);
    uint32_t* w_g = reinterpret_cast<uint32_t*>(bsm + kBinOffG);
    uint16_t* st_idx = reinterpret_cast<uint16_t*>(bsm + kBinOffIdx);

    const int tid = threadIdx.x;
    const unsigned long long steps_done = s.ctl->steps_done;
    const uint32_t* __restrict__ bits = s.bits[(steps_done - 1ull) & 1ull];
    const int B = s.bin_shift;
    const uint32_t lmask = (1u << B) - 1u;
    const uint32_t cap = s.bin_cap;
    const int64_t n_rounds = (s.n_words + wpr - 1) / wpr;
    unsigned long long cta_events = 0;

#pragma unroll
    for (int q = 0; q < kBinWinPerThread; ++q) w_cnt[tid * kBinWinPerThread + q] = 0u;
    __syncthreads();

    for (int64_t r = blockIdx.x; r < n_rounds; r += gridDim.x) {
        // ---- the round's firing rows in neuron order, listed in sub-rounds of at most
        //      kBinMaxRows rows (a prefix of the remaining words: at most 32 rows per word);
        //      the window of staged bins around them
        const int64_t rw0 = r * wpr;
        const uint32_t word_all = (tid < wpr && rw0 + tid < s.n_words) ? __ldcs(bits + rw0 + tid) : 0u;
        for (int wstart = 0; wstart < wpr;) {
        const int64_t w0 = rw0 + wstart;
        const int64_t n0 = w0 * 32 < s.N ? w0 * 32 : s.N;
        int64_t wb = (n0 >> B) - kBinWin / 2;
        if (wb > s.n_bins - kBinWin) wb = s.n_bins - kBinWin;
        if (wb < 0) wb = 0;
        const int64_t e_base = __ldg(s.qrow + n0);
        const bool mine_w = tid >= wstart && tid < wpr;
        const int cw = mine_w ? __popc(word_all) : 0;
        int all_rows;
        const int excl = bin_block_scan(cw, sh_warp, &all_rows);
        const bool take = mine_w && excl + cw <= kBinMaxRows;
        const int wend = wstart + __syncthreads_count(take);
        if (take) {
            uint32_t word = word_all;
            int pos = excl;
            while (word) {
                const int b = __ffs(word) - 1;
                word &= word - 1u;
                row_pre[pos++] = (uint32_t)((rw0 + tid) * 32 + b);
            }
        }
        (void)all_rows;
        if (take && tid == wend - 1) sh_warp[kBinThreads / 32] = excl + cw;   // rows of this sub-round
        __syncthreads();
        const int nrows = sh_warp[kBinThreads / 32];
        int len[kBinMaxRows / kBinThreads];
        int mine = 0;
#pragma unroll
        for (int q = 0; q < kBinMaxRows / kBinThreads; ++q) {
            const int i = tid * (kBinMaxRows / kBinThreads) + q;
            len[q] = 0;
            if (i < nrows) {
                const uint32_t pre = row_pre[i];
                const int64_t e0 = __ldg(s.qrow + pre);
                len[q] = (int)(__ldg(s.qrow + pre + 1) - e0);
                row_e0[i] = (uint32_t)(e0 - e_base);
                mine += len[q];
            }
        }
        int T;
        int ex = bin_block_scan(mine, sh_warp, &T);
#pragma unroll
        for (int q = 0; q < kBinMaxRows / kBinThreads; ++q) {
            const int i = tid * (kBinMaxRows / kBinThreads) + q;
            if (i < nrows) { row_off[i] = ex; ex += len[q]; }
        }
        if (tid == 0) row_off[nrows] = T;
        cta_events += (unsigned long long)T;
        __syncthreads();

        // ---- slices of kBinSlice events
        for (int v0 = 0; v0 < T; v0 += kBinSlice) {
            uint32_t c[kBinEPT], rk[kBinEPT];
            float2 w[kBinEPT];
#pragma unroll
            for (int u = 0; u < kBinEPT; ++u) {
                const int v = v0 + u * kBinThreads + tid;
                c[u] = kBinSkip;
                if (v < T) {
                    int lo = 0, hi = nrows;   // row_off[lo] <= v < row_off[hi]
                    while (hi - lo > 1) {
                        const int mid = (lo + hi) >> 1;
                        if (row_off[mid] <= v) lo = mid; else hi = mid;
                    }
                    const int64_t e = e_base + (int64_t)row_e0[lo] + (v - row_off[lo]);
                    c[u] = __ldcs(s.qcol + e);
                    w[u] = __ldcs(s.qw + e);
                }
            }
            // rank every event inside its window bin; events outside the window go to J now
#pragma unroll
            for (int u = 0; u < kBinEPT; ++u) {
                rk[u] = 0u;
                if (c[u] == kBinSkip) continue;
                const uint32_t post = c[u] & kIndexMask;
                const int64_t wi = (int64_t)(post >> B) - wb;
                if (wi >= 0 && wi < kBinWin) {
                    rk[u] = atomicAdd(w_cnt + wi, 1u);
                } else {
                    atomicAdd(s.J2 + (int64_t)(c[u] >> 31) * s.j_ps + (int64_t)post * s.j_es, w[u]);
                    c[u] = kBinSkip;
                }
            }
            __syncthreads();
            // window bins: run offsets in the staging buffer (scan) and runs reserved in the bins
            uint32_t cn[kBinWinPerThread];
            int sum = 0;
#pragma unroll
            for (int q = 0; q < kBinWinPerThread; ++q) { cn[q] = w_cnt[tid * kBinWinPerThread + q]; sum += (int)cn[q]; }
            int tot;
            int lo = bin_block_scan(sum, sh_warp, &tot);
            uint32_t g[kBinWinPerThread];
#pragma unroll
            for (int q = 0; q < kBinWinPerThread; ++q)
                g[q] = cn[q] ? atomicAdd(s.bin_cnt + wb + tid * kBinWinPerThread + q, cn[q]) : 0u;
#pragma unroll
            for (int q = 0; q < kBinWinPerThread; ++q) {
                w_cnt[tid * kBinWinPerThread + q] = (uint32_t)lo;
                w_g[tid * kBinWinPerThread + q] = g[q];
                lo += (int)cn[q];
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < kBinEPT; ++u) {
                if (c[u] == kBinSkip) continue;
                const uint32_t post = c[u] & kIndexMask;
                const uint32_t bin = post >> B;
                const int wi = (int)((int64_t)bin - wb);
                const uint32_t lp = w_cnt[wi] + rk[u];
                const uint32_t gp = w_g[wi] + rk[u];
                if (gp < cap) {
                    st_dst[lp] = bin * cap + gp;
                    st_w[lp] = w[u];
                    st_idx[lp] = (uint16_t)((post & lmask) | ((c[u] >> 31) << 15));
                } else {   // bin full: straight into J
                    st_dst[lp] = kBinSkip;
                    atomicAdd(s.J2 + (int64_t)(c[u] >> 31) * s.j_ps + (int64_t)post * s.j_es, w[u]);
                }
            }
            __syncthreads();
            for (int i = tid; i < tot; i += kBinThreads) {
                const uint32_t d = st_dst[i];
                if (d != kBinSkip) {
                    s.bin_idx[d] = st_idx[i];
                    s.bin_w[d] = st_w[i];
                }
            }
#pragma unroll
            for (int q = 0; q < kBinWinPerThread; ++q) w_cnt[tid * kBinWinPerThread + q] = 0u;
            __syncthreads();
        }
        wstart = wend;
        }
    }
    if (tid == 0) add_events(s, cta_events, blockIdx.x);
}

// ------------------------------------------------------------ exports

// ctl->events = the sum of the event counters (one CTA of kEvParts threads).
__global__ void __launch_bounds__(kEvParts) k_sum_events(const unsigned long long* __restrict__ part, Ctl* ctl)
{
    __shared__ unsigned long long sh[kEvParts / 32];
    unsigned long long v = part[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = sh[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) ctl->events = v;
    }
}

__global__ void k_export_J(const DevState s, float* __restrict__ out)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= s.N) return;
    const float4 J = load_J(s, n);
    out[n] = J.x; out[s.N + n] = J.y; out[2 * s.N + n] = J.z; out[3 * s.N + n] = J.w;
}

// I_ui [4][N] and I_syn [N] from the current V and J (models/block.py:83-87).
__global__ void k_export_current(const DevState s, float* __restrict__ iui, float* __restrict__ isyn)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= s.N) return;
    const ParamClass p = load_class(s.pc, s.cls[n]);
    const float v = s.V[n];
    const float4 J = load_J(s, n);
    const float4 g = s.gnrn ? mul4(p.g, s.gnrn[n]) : p.g;
    if (iui) {
        const float4 i = iui_g(g, p.Vu, v, J);
        iui[n] = i.x; iui[s.N + n] = i.y; iui[2 * s.N + n] = i.z; iui[3 * s.N + n] = i.w;
    }
    if (isyn) isyn[n] = isyn_g(g, p.Vu, v, J);
}

__global__ void k_bits_to_u8(const uint32_t* __restrict__ bits, int64_t N, uint8_t* __restrict__ out)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    out[n] = (uint8_t)((bits[n >> 5] >> (n & 31)) & 1u);
}

__global__ void k_u8_to_bits(const uint8_t* __restrict__ in, int64_t N, uint32_t* __restrict__ bits, int64_t n_words)
{
    const int64_t wi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (wi >= n_words) return;
    uint32_t w = 0;
    for (int b = 0; b < 32; ++b) {
        const int64_t n = wi * 32 + b;
        if (n < N && in[n]) w |= (1u << b);
    }
    bits[wi] = w;
}

// This step's input spikes: column (steps_done - src_from) of the raster, as
// bits of the input neurons in src_val (cleared beforehand).
__global__ void k_src_bits(const DevState s)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_src) return;
    const unsigned long long col = s.ctl->steps_done - s.src_from;
    if (col >= (unsigned long long)s.src_T) return;   // the host refuses runs past the raster
    const uint32_t w = __ldg(s.src_raster + (int64_t)col * s.src_words + (i >> 5));
    if ((w >> (i & 31)) & 1u) {
        const uint32_t n = s.src_neuron[i];
        atomicOr(s.src_val + (n >> 5), 1u << (n & 31));
    }
}

__global__ void k_J_from_planar(DevState s, const float* __restrict__ in)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= s.N) return;
    store_J(s, n, make_float4(in[n], in[s.N + n], in[2 * s.N + n], in[3 * s.N + n]));
}

// ------------------------------------------------------------ weights
// models/block.py:172-177: set channel weights of existing synapses.
__global__ void k_update_weight(DevState s, int64_t n, const uint8_t* __restrict__ ch,
                                const uint32_t* __restrict__ post, const uint32_t* __restrict__ pre,
                                const float* __restrict__ val, float2* pw, float2* qw, unsigned* missing)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t kb = (ch[i] >= 2) ? kKindBit : 0u;
    const int half = ch[i] & 1;
    const uint32_t po = post[i], pr = pre[i];
    bool found = false;
    if (pw && po < s.N) {
        for (int64_t e = s.prow[po]; e < s.prow[po + 1]; ++e) {
            if (s.pcol[e] == (pr | kb)) {
                float* w = reinterpret_cast<float*>(pw + e);
                w[half] = val[i];
                found = true;
                break;
            }
        }
    }
    if (qw && pr < s.N) {
        bool f2 = false;
        for (int64_t e = s.qrow[pr]; e < s.qrow[pr + 1]; ++e) {
            if (s.qcol[e] == (po | kb)) {
                float* w = reinterpret_cast<float*>(qw + e);
                w[half] = val[i];
                f2 = true;
                break;
            }
        }
        found = found || f2;
    }
    if (!found) atomicAdd(missing, 1u);
}

// ------------------------------------------------------------ BOLD
// models/bold_model_pytorch.py:43-78, one thread per region. Python scalars
// are rounded to T where the tensor expression consumes them.
template <typename T>
struct BoldScalars {
    T eps, ts, tf, t0, E0, V0, dt, base, exq, exv, k7, k2, one_em5;
};

__device__ __forceinline__ float dpow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double dpow(double a, double b) { return pow(a, b); }

template <typename T>
__global__ void k_bold_run(int64_t R, const T* __restrict__ u, T* s, T* q, T* v, T* f, T* __restrict__ out,
                           BoldScalars<T> c)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R) return;
    T fi = f[i], si = s[i], qi = q[i], vi = v[i];
    const T one = (T)1;
    const T ds = ((u[i] * c.eps) - si / c.ts) - (fi - one) / c.tf;
    const T qpart = fi > (T)0 ? (one - dpow(c.base, (one / fi) * one)) : one;
    const T dq = (((fi * qpart) / c.E0) - qi * dpow(vi, c.exq)) / c.t0;
    qi = qi + dq * c.dt;
    const T dv = (fi - dpow(vi, c.exv)) / c.t0;
    vi = vi + dv * c.dt;
    fi = fi + si * c.dt;
    fi = fi > (T)0 ? fi : (T)0;
    si = si + ds * c.dt;
    s[i] = si; q[i] = qi; v[i] = vi; f[i] = fi;
    out[i] = ((c.k7 * (one - qi) + (one - qi / vi) * (T)2) + c.k2 * (one - vi)) * c.V0;
}

// n_steps Euler steps of BOLD.run with a constant input per region
// (u_r = max(u[r], floor)), outputs the last step's signal.
template <typename T>
__global__ void k_bold_run_steps(int64_t R, const T* __restrict__ u, int n_steps, T floor_u, T* s, T* q, T* v, T* f,
                                 T* __restrict__ out, BoldScalars<T> c)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R) return;
    T fi = f[i], si = s[i], qi = q[i], vi = v[i];
    const T one = (T)1;
    const T ui = u[i] > floor_u ? u[i] : floor_u;
    for (int k = 0; k < n_steps; ++k) {
        const T ds = ((ui * c.eps) - si / c.ts) - (fi - one) / c.tf;
        const T qpart = fi > (T)0 ? (one - dpow(c.base, (one / fi) * one)) : one;
        const T dq = (((fi * qpart) / c.E0) - qi * dpow(vi, c.exq)) / c.t0;
        qi = qi + dq * c.dt;
        const T dv = (fi - dpow(vi, c.exv)) / c.t0;
        vi = vi + dv * c.dt;
        fi = fi + si * c.dt;
        fi = fi > (T)0 ? fi : (T)0;
        si = si + ds * c.dt;
    }
    s[i] = si; q[i] = qi; v[i] = vi; f[i] = fi;
    out[i] = ((c.k7 * (one - qi) + (one - qi / vi) * (T)2) + c.k2 * (one - vi)) * c.V0;
}

template <typename T>
__device__ __forceinline__ T max_nan(T x, T c) { return (x != x) ? x : (x < c ? c : x); }

// bold_model_pytorch.py:34-41
template <typename T>
__global__ void k_bold_state_update(int64_t R, int64_t S, const T* __restrict__ w, T* s, T* q, T* v, T* f, T c)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R) return;
    const T* row = w + i * S;
    s[i] = row[0];
    q[i] = max_nan(row[1], c);
    v[i] = max_nan(row[2], c);
    f[i] = max_nan(row[3], c);
}

template <typename T>
__global__ void k_fill(T* p, int64_t n, T val)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = val;
}

// ------------------------------------------------------------ generator
// Counter-based synthetic network, restated on the CPU by
// oracle/oracle.c:oracle_gen_rows.  One warp per postsynaptic row.
struct GenArgs {
    int64_t N;
    int R;
    const int64_t* region_start;  // [R+1]
    const int64_t* region_n_exc;  // [R]
    const int32_t* src_base;      // [R] first candidate source region of a row of region r
    const int32_t* src_count;     // [R] number of candidate source regions
    const int64_t* cum_off;       // [R] offset of region r's cumulative row in cum_flat
    const float* cum_flat;
    const int32_t* region_member; // [R]
    const int64_t* member_start;  // [M] first neuron of every member
    const uint64_t* member_seed;  // [M] generator key of every member
    int K, Kp;                    // in-degree, next power of two
    float w_scale;
    uint32_t* pcol;               // [N*K]
    float2* pw;                   // [N*K]
    uint32_t* outdeg;             // [N] (nullable) out-degree counts
    unsigned* err;                // rows that could not draw K sources
};

constexpr uint32_t kTagSrc = 0xF0000001u;
constexpr uint32_t kTagW = 0xF0000002u;
constexpr int kGenWarps = 4;

__device__ __forceinline__ int region_of(const int64_t* __restrict__ rs, int R, int64_t n)
{
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(rs + mid) <= n) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kGenWarps * 32) k_gen_rows(GenArgs g)
{
    extern __shared__ unsigned long long gsm[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * kGenWarps + wid;
    if (i >= g.N) return;
    unsigned long long* chosen = gsm + (size_t)wid * g.Kp;
    const int ri = region_of(g.region_start, g.R, i);
    const float* crow = g.cum_flat + __ldg(g.cum_off + ri);
    const int cnt_src = __ldg(g.src_count + ri), base_src = __ldg(g.src_base + ri);
    const int mem = __ldg(g.region_member + ri);
    const uint64_t li = (uint64_t)(i - __ldg(g.member_start + mem));   // member-local row index
    const uint64_t key = __ldg(g.member_seed + mem);
    const uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
    int have = 0;
    uint32_t attempt = 0;
    const uint32_t limit = (uint32_t)(64 * g.K + 1024);
    bool failed = false;
    while (have < g.K) {
        if (attempt > limit) { failed = true; break; }
        const U4 o = philox4x32_10(U4{(uint32_t)li, kTagSrc, attempt, (uint32_t)(li >> 32)}, k0, k1);
        ++attempt;
        const uint32_t ws[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (have >= g.K) break;
            const float ur = u01(ws[2 * h]);
            int cntr = 0;
            for (int j = lane; j < cnt_src - 1; j += 32) cntr += (__ldg(crow + j) <= ur) ? 1 : 0;
            const int r = base_src + __reduce_add_sync(0xffffffffu, cntr);
            const int64_t rs0 = __ldg(g.region_start + r);
            const int64_t size = __ldg(g.region_start + r + 1) - rs0;
            if (size <= 0) continue;
            const uint64_t off = ((uint64_t)ws[2 * h + 1] * (uint64_t)size) >> 32;
            const int64_t src = rs0 + (int64_t)off;
            if (src == i) continue;
            bool dup = false;
            for (int k = lane; k < have; k += 32) dup |= ((int64_t)(chosen[k] >> 1) == src);
            if (__any_sync(0xffffffffu, dup)) continue;
            const unsigned long long kb = ((int64_t)off >= __ldg(g.region_n_exc + r)) ? 1ull : 0ull;
            if (lane == 0) chosen[have] = ((unsigned long long)src << 1) | kb;
            __syncwarp();
            ++have;
        }
    }
    if (failed) {
        if (lane == 0) atomicAdd(g.err, 1u);
        for (int k = have + lane; k < g.K; k += 32) chosen[k] = 0ull;
        __syncwarp();
    }
    for (int k = g.K + lane; k < g.Kp; k += 32) chosen[k] = ~0ull;
    __syncwarp();
    // bitonic sort of chosen[0..Kp)
    for (int size = 2; size <= g.Kp; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int idx = lane; idx < g.Kp; idx += 32) {
                const int p = idx ^ stride;
                if (p > idx) {
                    const unsigned long long a = chosen[idx], b = chosen[p];
                    const bool up = (idx & size) == 0;
                    if ((a > b) == up) { chosen[idx] = b; chosen[p] = a; }
                }
            }
            __syncwarp();
        }
    }
    const int64_t rowbase = i * (int64_t)g.K;
    for (int j = lane; j < g.K; j += 32) {
        const unsigned long long e = chosen[j];
        const uint32_t src = (uint32_t)(e >> 1);
        g.pcol[rowbase + j] = src | ((e & 1ull) ? kKindBit : 0u);
        const U4 o = philox4x32_10(U4{(uint32_t)li, kTagW, (uint32_t)(j >> 1), (uint32_t)(li >> 32)}, k0, k1);
        const uint32_t a = (j & 1) ? o.z : o.x;
        const uint32_t b = (j & 1) ? o.w : o.y;
        g.pw[rowbase + j] = make_float2(u01(a) * g.w_scale, u01(b) * g.w_scale);
        if (g.outdeg) atomicAdd(g.outdeg + src, 1u);
    }
}

// ------------------------------------------------------------ CSR transpose
// Exclusive scan of u32 counts into i64 row pointers (three passes).
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long* sh, long long& total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        long long w = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        sh[lane] = w;
    }
    __syncthreads();
    total = sh[(blockDim.x >> 5) - 1];
    const long long before = wid ? sh[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in, int64_t n,
                                                             int64_t* __restrict__ out, long long* __restrict__ tile_sum)
{
    __shared__ long long sh[32];
    const int64_t t0 = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    long long v[kScanItems];
    long long local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (t0 + k < n) ? (long long)in[t0 + k] : 0;
        local += v[k];
    }
    long long total;
    long long ex = block_exclusive_scan(local, sh, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (t0 + k < n) out[t0 + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(long long* tile_sum, int64_t ntiles)
{
    __shared__ long long sh[32];
    long long carry = 0;
    for (int64_t b = 0; b < ntiles; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const long long v = (i < ntiles) ? tile_sum[i] : 0;
        long long total;
        const long long ex = block_exclusive_scan(v, sh, total);
        if (i < ntiles) tile_sum[i] = ex + carry;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) tile_sum[ntiles] = carry;
}

__global__ void k_scan_add(int64_t* out, int64_t n, const long long* __restrict__ tile_sum, int64_t ntiles)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_sum[i / kScanTile];
    if (i == 0) out[n] = tile_sum[ntiles];
}

// Fill the push CSR from the pull CSR (unordered within a row; sorted next).
// Out-degree of every presynaptic neuron from the pull CSR (counts[N] zeroed).
__global__ void k_count_outdeg(int64_t S, const uint32_t* __restrict__ pcol, uint32_t* counts)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < S) atomicAdd(counts + (pcol[e] & kIndexMask), 1u);
}

__global__ void k_fill_push(int64_t N, const int64_t* __restrict__ prow, const uint32_t* __restrict__ pcol,
                            const float2* __restrict__ pw, const int64_t* __restrict__ qrow, uint32_t* cursor,
                            uint32_t* qcol, float2* qw, uint16_t* qpos)
{
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= N) return;
    for (int64_t e = prow[i] + lane; e < prow[i + 1]; e += 32) {
        const uint32_t c = pcol[e];
        const uint32_t src = c & kIndexMask;
        const uint32_t pos = atomicAdd(cursor + src, 1u);
        const int64_t d = qrow[src] + pos;
        qcol[d] = (uint32_t)i | (c & kKindBit);
        qw[d] = pw[e];
        if (qpos) qpos[d] = (uint16_t)(e - prow[i]);
    }
}

// Sort every push row by postsynaptic index (warp per row, rows up to
// kSortCap entries in shared memory; longer rows are flagged).
constexpr int kSortCap = 2048;
static_assert(kSortCap <= 2048, "the row slot takes 11 bits of the sort key");
constexpr int kSortWarps = 4;

__global__ void __launch_bounds__(kSortWarps * 32) k_sort_push_rows(int64_t N, const int64_t* __restrict__ qrow,
                                                                    uint32_t* qcol, float2* qw, uint16_t* qpos,
                                                                    unsigned* too_long)
{
    extern __shared__ unsigned long long ssm[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int64_t r = (int64_t)blockIdx.x * kSortWarps + wid;
    if (r >= N) return;
    const int64_t e0 = qrow[r], e1 = qrow[r + 1];
    const int64_t len = e1 - e0;
    if (len <= 1) return;
    if (len > kSortCap) { if (lane == 0) atomicAdd(too_long, 1u); return; }
    // key = post << 32 | kind bit | pull-row position << 11 | slot: rows are ordered by
    // (postsynaptic neuron, kind, position in its pull row), a deterministic order even
    // when one pair of neurons has several synapses
    unsigned long long* key = ssm + (size_t)wid * kSortCap;
    float2* wtmp = reinterpret_cast<float2*>(ssm + (size_t)kSortWarps * kSortCap) + (size_t)wid * kSortCap;
    uint16_t* ptmp = reinterpret_cast<uint16_t*>(ssm + (size_t)2 * kSortWarps * kSortCap) + (size_t)wid * kSortCap;
    int Kp = 1;
    while (Kp < len) Kp <<= 1;
    for (int k = lane; k < Kp; k += 32) {
        unsigned long long kk = ~0ull;
        if (k < len) {
            const uint32_t c = qcol[e0 + k];
            kk = ((unsigned long long)(c & kIndexMask) << 32) | (unsigned long long)(c & kKindBit) |
                 (qpos ? ((unsigned long long)qpos[e0 + k] << 11) : 0ull) | (unsigned long long)k;
            wtmp[k] = qw[e0 + k];
            if (qpos) ptmp[k] = qpos[e0 + k];
        }
        key[k] = kk;
    }
    __syncwarp();
    for (int size = 2; size <= Kp; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int idx = lane; idx < Kp; idx += 32) {
                const int p = idx ^ stride;
                if (p > idx) {
                    const unsigned long long a = key[idx], b = key[p];
                    const bool up = (idx & size) == 0;
                    if ((a > b) == up) { key[idx] = b; key[p] = a; }
                }
            }
            __syncwarp();
        }
    }
    for (int k = lane; k < len; k += 32) {
        const unsigned long long kk = key[k];
        qcol[e0 + k] = (uint32_t)(kk >> 32) | (uint32_t)(kk & kKindBit);
        qw[e0 + k] = wtmp[(int)(kk & 0x7ffull)];
        if (qpos) qpos[e0 + k] = ptmp[(int)(kk & 0x7ffull)];
    }
}

// ------------------------------------------------------------ gamma-distributed properties
// cuda/src/stage/property.cpp:313-471 (gamma_kernel / sample_gamma): every
// neuron of a subblock draws its own value Gamma(alpha, 1) / beta.  Method of
// Marsaglia & Tsang, "A simple method for generating gamma variables", ACM
// TOMS 26(3), 2000 (squeeze test, then the log test; alpha < 1 through
// G(alpha) = G(alpha + 1) U^(1/alpha)).  Normals by the Box-Muller transform
// (Box & Muller 1958).  All arithmetic in double; uniforms from Philox4x32-10
// with counter {n_lo, n_hi, attempt, tag} and key {seed_lo, seed_hi ^ 'GAMM'}
// (tag = 0x80000000 | receptor << 24 | call number), 64 attempts at most (the
// acceptance rate is above 95 % per attempt), after which the mode d is used.
constexpr uint32_t kGammaKeyXor = 0x47414D4Du;

__host__ __device__ inline double gamma_u24(uint32_t x, int open_zero)
{
    return ((double)(x >> 8) + (open_zero ? 1.0 : 0.0)) * (1.0 / 16777216.0);
}

__device__ inline double gamma_unit(double alpha, uint64_t seed, uint64_t n, uint32_t tag)
{
    if (!(alpha > 0.0)) return 0.0;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32) ^ kGammaKeyXor;
    double scale = 1.0;
    if (alpha < 1.0) {
        const U4 r = philox4x32_10(U4{(uint32_t)n, (uint32_t)(n >> 32), 0xffffffffu, tag}, k0, k1);
        scale = pow(gamma_u24(r.x, 1), 1.0 / alpha);
        alpha += 1.0;
    }
    const double d = alpha - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    for (uint32_t it = 0; it < 64u; ++it) {
        const U4 r = philox4x32_10(U4{(uint32_t)n, (uint32_t)(n >> 32), it, tag}, k0, k1);
        const double u1 = gamma_u24(r.x, 1), u2 = gamma_u24(r.y, 0);
        const double x = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        const double y = 1.0 + c * x;
        if (y <= 0.0) continue;
        const double v = y * y * y;
        const double u = gamma_u24(r.z, 1);
        const double xx = x * x;
        if (u < 1.0 - 0.0331 * xx * xx) return scale * d * v;
        if (log(u) < 0.5 * xx + d * (1.0 - v + log(v))) return scale * d * v;
    }
    return scale * d;
}

// req[sub * 4 + u] = request index for receptor u of subblock sub, or -1.
__global__ void k_gamma(const DevState s, const int32_t* __restrict__ req, const double* __restrict__ alpha,
                        const double* __restrict__ beta, uint32_t call, float4* __restrict__ g)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= s.N) return;
    const int sub = s.pc[s.cls[n]].sub;
    if (sub < 0 || sub >= s.n_sub) return;
    float4 v = g[n];
    float* vp = reinterpret_cast<float*>(&v);
    bool any = false;
    for (int u = 0; u < 4; ++u) {
        const int r = req[(int64_t)sub * 4 + u];
        if (r < 0) continue;
        const uint32_t tag = 0x80000000u | ((uint32_t)u << 24) | (call & 0x00ffffffu);
        vp[u] = (float)(gamma_unit(alpha[r], s.seed, (uint64_t)n, tag) / beta[r]);
        any = true;
    }
    if (any) g[n] = v;
}

__global__ void k_fill4(float4* p, int64_t n, float4 val)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = val;
}

}  // namespace dtb
