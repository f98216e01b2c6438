// Device-side data structures and helpers shared by the kernels of libdtb.
//
// Layout in HBM (one network = one handle):
//   V[N] f32, J as two float2 planes (AMPA/NMDA pairs, then GABAa/GABAb pairs:
//   one 32-byte sector holds four neurons' pair, which the push atomics hit),
//   t_last[N] f32,
//   cls[N] u32 -> ParamClass table (deduplicated property rows),
//   spike bitmasks: new_active (double buffered by step parity) and active,
//   ceil(N/128)*4 words each (one warp owns 128 neurons = 4 words),
//   pull CSR: prow[N+1] i64, pcol[S] u32 (pre | bit31 = GABA pair), pw[S] float2,
//   push CSR: qrow[N+1] i64, qcol[S] u32 (post | bit31 = GABA pair), qw[S] float2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dtb {

constexpr uint32_t kKindBit = 0x80000000u;
constexpr uint32_t kIndexMask = 0x7fffffffu;
constexpr int kWarpNeurons = 128;      // neurons owned by one warp in the step kernels
constexpr uint32_t kSlotCap = 8;       // ordered-push contributions kept per neuron and step
constexpr int kGatherRows = 1;         // k_step gathers whole pull rows
constexpr int kGatherSlots = 2;        // k_step sums its ordered-push slots
constexpr int kGatherMasks = 3;        // k_step sums the pull entries its position masks mark
constexpr int kGatherStream = 4;       // k_step streams its tile's pull entries, chunk by chunk
constexpr int kGatherBins = 5;         // k_step folds its chunk's binned push events (CTA-wide, shared memory)
constexpr int kBinMinShift = 10;       // binned push: 2^bin_shift neurons per bin (= update chunk), 10..13
constexpr int kBinMaxShift = 13;
constexpr int kBinMaxBins = 1 << 22;  // bins per network (u32 entry addresses: bins x capacity < 2^32)
constexpr int kStreamWarpBytes = 129 * 8 + 8 + 128 * 16;   // row pointers (+pad) and row sums per warp
constexpr int kMaskWords = 4;          // position-mask words per kind: in-degree up to 128
constexpr int kMaskList = 256;         // marked entries a warp gathers together per tile
constexpr uint32_t kMixedTile = 0xffffffffu;   // tile_cls of a tile whose neurons have different classes
constexpr int kStepThreads = 256;      // 8 warps, 1024 neurons per CTA
constexpr int kEvParts = 1024;         // event counters: many warps add at once, one address would serialise

// One deduplicated row of the 22-column property matrix
// (generation/make_block.py:394-432) with the derived constants the step uses.
struct __align__(16) ParamClass {
    float4 g;       // g_ui           cols 10-13
    float4 Vu;      // V_ui           cols 14-17
    float4 decay;   // exp(-dt/tau_ui), tau cols 18-21
    float gL;       // col 6
    float VL;       // col 7
    float rCdt;     // (1/C) * dt, C col 4 (torch: C.reciprocal() * dt)
    float Vth;      // col 8
    float Vreset;   // col 9
    float Tref;     // col 5
    float Iext;     // col 2
    float noise;    // col 0 (per-neuron noise rate, cuda/src/stage/spike.cpp:157)
    int32_t sub;    // col 3 (subblock index)
    float C;        // col 4
    int32_t member; // ensemble member (noise stream offset), -1 outside ensembles
    float pad1;
};
static_assert(sizeof(ParamClass) == 96, "ParamClass layout");

// Control block in device memory; read by every step kernel, advanced by the
// last CTA of each update kernel.
struct Ctl {
    unsigned long long steps_done;   // number of completed updates (Philox step counter)
    // per-run parameters, written by the host as one 16-byte copy
    unsigned long long run_base;     // steps_done at the start of the current run (stats row 0)
    float noise_rate;                // >= 0: scalar rate; < 0: per-class rate
    int32_t isolated;                // block.run(isolated=...)
    float t;                         // block.t after the last update (float32 accumulation)
    uint32_t done;                   // CTAs finished in the current update kernel
    uint32_t stats_cap;              // rows of the per-step stats buffers
    uint32_t use_isyn_override;      // next update takes I_syn from isyn_override
    uint32_t err;                    // sticky error flags
    uint32_t pad;
    unsigned long long events;       // synaptic events propagated since creation
};
static_assert(sizeof(Ctl) == 56, "Ctl layout");

struct RunParams {
    unsigned long long run_base;
    float noise_rate;
    int32_t isolated;
};
static_assert(sizeof(RunParams) == 16, "RunParams layout");

struct BoldDev {
    int n_regions;               // 0: no BOLD attached
    const int32_t* sub_region;   // [n_sub] -> region or -1
    const double* region_n;      // [R] neurons in region
    double* s; double* q; double* v; double* f; double* act; double* out;   // [R]
    double epsilon, tao_s, tao_f, tao_0, div_alpha, E0, V0, delta_t;
};

struct DevState {
    int64_t N;
    int64_t n_words;            // bitmask words (multiple of 4)
    float* V;
    float2* J2;                 // receptor pairs: pair p of neuron n at J2[p * j_ps + n * j_es]
    int64_t j_ps;               // plane stride (float2 units): N for the split layout, 1 for [N][4]
    int64_t j_es;               // neuron stride (float2 units): 1 for the split layout, 2 for [N][4]
    int j_keep;                 // J stores at normal L2 priority (else evict-first)
    int rev_scatter;            // the atomic scatter walks the bitmask from its end
    float* tlast;
    float* isyn_override;       // [N] used once after update_property
    const uint32_t* cls;
    const uint32_t* tile_cls;   // [ceil(N/128)] the class every neuron of a 128-neuron tile shares, else
                                // kMixedTile (nullable: every tile then reads its per-neuron ids)
    const ParamClass* pc;
    const float4* gnrn;         // [N] per-neuron factors of g_ui (gamma-distributed properties; nullable)
    const int64_t* member_start;  // [M] first neuron of every ensemble member (nullable)
    uint32_t* bits[2];          // new_active bitmask by step parity
    uint32_t* abits;            // active bitmask of the latest update
    const uint32_t* forced_active;   // teacher forcing bitmasks (nullable)
    const uint32_t* forced_new;
    const uint32_t* forced_mask;     // neurons forced_active applies to (nullable: every neuron)
    // input neurons (models/block.py:37-50, :104-109): their spikes replay a raster
    int64_t n_src;
    const uint32_t* src_neuron;      // [n_src]
    const uint32_t* src_raster;      // [T][src_words] bits by input ordinal
    int64_t src_words;
    int64_t src_T;
    unsigned long long src_from;     // step at which column 0 is replayed
    uint32_t* src_val;               // [n_words] this step's input spikes (forced_active while inputs are set)
    // pull CSR
    const int64_t* prow; const uint32_t* pcol; const float2* pw;
    // push CSR
    const int64_t* qrow; const uint32_t* qcol; const float2* qw;
    const uint16_t* qpos;       // [S] position of every push entry inside its pull row (nullable)
    // ordered push (bit-exact pull order at push cost): pending contributions per neuron
    uint32_t* slot_cnt;         // [N] contributions written since the neuron last consumed them
    uint4* slots;               // [N][kSlotCap] {pull-row position | kind bit, 0, w.x bits, w.y bits}
    uint32_t* pmask;            // [N][2][kMaskWords] pull-row positions that fired (excitatory, inhibitory)
    // binned push: the scatter appends every synaptic event {neuron within bin | kind << 15, w} to the bin of
    // its postsynaptic neuron; the next update folds each bin into its chunk in shared memory
    uint16_t* bin_idx;          // [n_bins][bin_cap]
    float2* bin_w;              // [n_bins][bin_cap]
    uint32_t* bin_cnt;          // [n_bins] events appended (may exceed bin_cap: the rest went to J by atomics)
    int64_t n_bins;
    uint32_t bin_cap;           // entries per bin (n_bins * bin_cap < 2^32)
    int bin_shift;              // 2^bin_shift neurons per bin
    // statistics
    int n_sub;
    uint32_t* sub_spk;          // [n_sub] accumulators (active)
    uint32_t* sub_nact;         // [n_sub] accumulators (new_active)
    double* sub_vsum;           // [n_sub]
    const uint32_t* sub_count;  // [n_sub] neurons per subblock
    uint32_t* unmapped_nact;    // new_active of neurons whose subblock is out of range
    unsigned long long* win_spk; // [n_sub] spikes accumulated since the host last cleared them
    int stats_ext;              // 1: statistics and BOLD in k_stats (many subblocks / regions)
    const int32_t* grp_ptr;     // k_stats groups: [n_groups+1] into grp_sub
    const int32_t* grp_sub;     // subblocks of every group
    const int32_t* grp_region;  // [n_groups] BOLD region of the group or -1
    int n_groups;
    const uint32_t* samples;    // sampled neurons (cuda/src/stage/sample.cpp:8)
    int n_samples;
    int64_t samp_cap;           // ring rows
    uint8_t* samp_spk;          // [samp_cap][n_samples] spike (threshold crossing) of the step
    float* samp_v;              // [samp_cap][n_samples] V after the step
    float* st_spk;              // [stats_cap][n_sub]
    float* st_mean;             // [stats_cap][n_sub]
    uint32_t* st_nact;          // [stats_cap]
    Ctl* ctl;
    uint32_t stage_wait_limit;     // polls of a staged copy's mbarrier before the update gives up on it
    unsigned long long* ev_part;   // [kEvParts] synaptic event counters (summed into ctl->events on demand;
                                   // nullable: then the kernels add to ctl->events)
    uint64_t seed;
    uint32_t stream_id;
    float dt;
    BoldDev bold;
};

// ---------------------------------------------------------------- Philox
// Philox4x32-10, Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11 (round function and Weyl key schedule of the paper).
struct U4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo)
{
#ifdef __CUDA_ARCH__
    hi = __umulhi(a, b);
    lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(0xD2511F53u, c.x, hi0, lo0);
        mulhilo32(0xCD9E8D57u, c.z, hi1, lo1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
    }
    return c;
}

// 24-bit uniform in [0,1), exact in float32.
__host__ __device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

}  // namespace dtb
