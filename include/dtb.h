/*
 * dtb.h — C ABI of the B200-native Digital Twin Brain time-step library
 * (libdtb.so, built from digital_twin_brain_b200/csrc/).
 *
 * One handle (dtb_block) is one network resident on one GPU: neuron state,
 * parameter classes, pull CSR (by postsynaptic neuron) and push CSR (by
 * presynaptic neuron).  Every call returns 0 on success or a dtb_status code;
 * dtb_last_error() gives the message.  No call throws or exits.  The library
 * owns device memory; the caller owns every buffer it passes.  A handle is
 * used by one host thread at a time and issues all work on one CUDA stream
 * (dtb_block_set_stream).
 *
 * Pointers tagged `where` are host memory (DTB_HOST) or device memory on the
 * handle's device (DTB_DEVICE).
 *
 * Each entry point names the reference interface it replaces
 * (yeyeleijun/Digital_twin_brain, file:line).
 */
#ifndef DTB_H
#define DTB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTB_ABI_VERSION 1
#define DTB_NPROP 22 /* property columns, generation/make_block.py:394-432 */

typedef enum {
    DTB_OK = 0,
    DTB_ERR_ARG = 1,      /* bad argument (null, out of range, inconsistent sizes) */
    DTB_ERR_CUDA = 2,     /* CUDA runtime error */
    DTB_ERR_NOMEM = 3,    /* host or device allocation failed */
    DTB_ERR_IO = 4,       /* file could not be read or written */
    DTB_ERR_FORMAT = 5,   /* malformed npz / npy / checkpoint */
    DTB_ERR_STATE = 6,    /* call not valid in the handle's current state */
    DTB_ERR_LIMIT = 7     /* size beyond a documented limit */
} dtb_status;

typedef enum { DTB_HOST = 0, DTB_DEVICE = 1 } dtb_where;

/* Propagation method for a run: the per-step choice between the push scatter
 * (compacted spike list, float2 atomics) and the pull gather (spike bitmask,
 * row-ordered, bit-identical to torch.sparse.mm's accumulation order). */
typedef enum { DTB_MODE_AUTO = 0, DTB_MODE_PUSH = 1, DTB_MODE_PULL = 2 } dtb_mode;

typedef enum {
    DTB_FIELD_V = 0,          /* float[N]      block.V_i          models/block.py:56  */
    DTB_FIELD_J = 1,          /* float[4][N]   block.J_ui         models/block.py:57  */
    DTB_FIELD_I_UI = 2,       /* float[4][N]   block.I_ui         models/block.py:84  */
    DTB_FIELD_I_SYN = 3,      /* float[N]      block.I_syn        models/block.py:86  */
    DTB_FIELD_T_LAST = 4,     /* float[N]      block.t_ik_last    models/block.py:55  */
    DTB_FIELD_ACTIVE = 5,     /* uint8[N]      block.active       models/block.py:134 */
    DTB_FIELD_NEW_ACTIVE = 6, /* uint8[N]      spikes | noise     models/block.py:136 */
    DTB_FIELD_T = 7,          /* float[1]      block.t            models/block.py:58  */
    DTB_FIELD_STEP = 8,       /* uint64[1]     steps taken (Philox step counter) */
    DTB_FIELD_SUB_COUNT = 9,  /* uint32[n_sub] neurons per subblock */
    DTB_FIELD_EVENTS = 10,    /* uint64[1]     synaptic events propagated since creation */
    DTB_FIELD_WINDOW_SPIKES = 11, /* uint64[n_sub] spikes per subblock since last set (window totals,
                                    simulation/simulation.py:269-279 freqs summed over a TR) */
    DTB_FIELD_G_FACTOR = 12   /* float[N][4]  per-neuron g_ui factors after dtb_block_gamma_property_by_subblock */
} dtb_field;

typedef struct dtb_block dtb_block;
typedef struct dtb_bold dtb_bold;

/* Network from host arrays: the in-memory form of generation/read_block.py
 * (property [N,22] + COO synapses), i.e. models/block.py:30 block(node_property,
 * w_uij, delta_t).  Synapse e adds weight[e][0] to channel kind[e] and
 * weight[e][1] to channel kind[e]+1 of neuron post[e] when neuron pre[e]
 * fires (generation/read_block.py:68-74).  Entries are kept in the given
 * order inside every row of both CSRs (stable sorts), which is the order
 * torch.sparse.mm accumulates in. */
typedef struct {
    int64_t n_neurons;
    const float* property;   /* [N][22] row-major, host */
    const float* decay;      /* [N][4] exp(-dt/tau_ui) per neuron, host; NULL: expf on the host */
    int64_t n_synapses;
    const uint32_t* post;    /* [S] host */
    const uint32_t* pre;     /* [S] host */
    const uint8_t* kind;     /* [S] 0 = AMPA/NMDA, 2 = GABAa/GABAb, host */
    const float* weight;     /* [S][2] host */
    float dt;                /* ms */
    uint64_t seed;           /* Philox key of the noise stream */
    uint32_t stream_id;      /* Philox counter word 1 (ensemble member) */
    int device;              /* CUDA device ordinal */
    int build_push;          /* nonzero: also build the push CSR */
} dtb_block_desc;

/* Synthetic network generated on the GPU (counter-based Philox, identical to
 * the CPU restatement in oracle/oracle.c:oracle_gen_rows).  Regions own
 * neuron ranges [region_start[r], region_start[r+1]); the first
 * region_n_exc[r] are excitatory.  Each neuron draws K distinct presynaptic
 * neurons (never itself): source region from the cumulative row cum[r][*],
 * then a uniform neuron inside it.  Parameter class of a neuron = 2r
 * (excitatory) or 2r+1 (inhibitory), class parameters from
 * class_property[2R][22] (its column 3 is the subblock). */
typedef struct {
    int n_regions;
    const int64_t* region_start;   /* [R+1] host */
    const int64_t* region_n_exc;   /* [R] host */
    const float* cum;              /* [R][R] host, cumulative source-region distribution */
    int K;                         /* in-degree, 1..1024 */
    float w_scale;                 /* weights U[0,1) * w_scale */
    uint64_t gen_seed;
    const float* class_property;   /* [2R][22] host */
    const float* class_decay;      /* [2R][4] host; NULL: expf on the host */
    float dt;
    uint64_t seed;
    uint32_t stream_id;
    int device;
    int build_push;
    /* Ensembles of members (optional: all NULL / 0 for one network).  A row of
     * region r draws its source region among src_base[r] .. src_base[r] +
     * src_count[r] - 1 through the cumulative row cum_flat[cum_off[r] ..]
     * (then `cum` is unused).  Region r belongs to member region_member[r];
     * member m's neurons start at member_start[m] (a multiple of 128); its rows
     * are drawn with key member_seed[m] and member-local row indices, and its
     * noise with stream stream_id + m and member-local counters, so every
     * member equals the same network generated and simulated alone.  The
     * subblock of class c is class_property[c][3] (-1: not counted). */
    const int32_t* src_base;
    const int32_t* src_count;
    const int64_t* cum_off;
    const float* cum_flat;
    int32_t n_members;
    const int32_t* region_member;
    const int64_t* member_start;
    const uint64_t* member_seed;
} dtb_synth_desc;

typedef struct {
    int64_t n_neurons;
    int64_t n_synapses;
    int32_t n_subblocks;
    int32_t n_classes;
    int32_t has_pull;
    int32_t has_push;
    int64_t device_bytes;    /* device memory held by the handle */
    int64_t max_outdegree;
    int64_t max_indegree;
    int64_t kernel_launches; /* kernels enqueued so far (graph nodes counted) */
} dtb_block_info;

/* ---- library ------------------------------------------------------------ */

int dtb_abi_version(void);
/* Copies the calling thread's last error message (NUL-terminated). */
int dtb_last_error(char* buf, size_t len);

/* ---- block lifecycle ---------------------------------------------------- */

/* models/block.py:30-60 block.__init__; cuda/src/block.cpp:13-180
 * (BrainBlock ctor, init_connection_table_gpu, init_config_params_gpu,
 * init_all_stages_gpu); CSR order of cuda/src/configuration.cpp:575-828.
 * Initial state as block.py: V = (V_th + V_reset)/2, J = 0, t_last = 0, t = 0. */
int dtb_block_create(const dtb_block_desc* desc, dtb_block** out);

/* generation/make_block.py:206-323 (connect_for_single_sparse_block) +
 * :326-434 (generate_block_node_property), generated on the device. */
int dtb_block_create_synthetic(const dtb_synth_desc* desc, dtb_block** out);

/* cuda/src/configuration.cpp:748 parse_conn_table_from_numpy +
 * :961 parse_params_from_numpy: reads block_0.npz .. block_{n-1}.npz of
 * generation/make_block.py:473-479 from `dir` (one population per file, as
 * generation/read_block.py:12-97 reads them). */
int dtb_block_create_from_npz(const char* dir, float dt, uint64_t seed, uint32_t stream_id,
                              int device, int build_push, dtb_block** out);

int dtb_block_destroy(dtb_block* b);

/* cuda/src/block.cpp / dist_simulator.cpp:399-400 (the step's stream).
 * `stream` is a cudaStream_t; NULL selects the legacy default stream. */
int dtb_block_set_stream(dtb_block* b, void* stream);
int dtb_block_synchronize(dtb_block* b);
int dtb_block_get_info(const dtb_block* b, dtb_block_info* info);

/* ---- stepping ----------------------------------------------------------- */

/* n_steps x models/block.py:116-150 block.run(noise_rate, isolated).
 * noise_rate >= 0: that rate for every neuron (block.py:136);
 * noise_rate < 0: per-neuron rate from property column 0 (cuda/src/stage/spike.cpp:157).
 * Outputs per step (nullable): sum_out[n_steps][n_sub] spike count of every
 * subblock (noise excluded, block.py:148), mean_out[n_steps][n_sub] mean V
 * (block.py:147; NaN for an empty subblock), nact_out[n_steps] number of
 * neurons that propagated (spikes | noise).  All three at `where`. */
int dtb_block_run(dtb_block* b, int n_steps, float noise_rate, int isolated, int mode,
                  float* sum_out, float* mean_out, uint32_t* nact_out, int where);

/* One block.run in which this step's active and new_active sets are replaced
 * by the given uint8[N] arrays (teacher forcing; NULL keeps the computed
 * set).  Used to compare against a reference run step by step. */
int dtb_block_step_forced(dtb_block* b, float noise_rate, int isolated, int mode,
                          const uint8_t* forced_active, const uint8_t* forced_new_active,
                          float* sum_out, float* mean_out, int where);

/* Measurement hook (the per-iteration timers of cuda/tools/benchmark.cpp:
 * 2289-2316, per kernel): runs n_steps with CUDA events around every kernel
 * launch (no graphs) and writes out_ms[0] = mean duration of the kernels that
 * update neurons (fused with the gather in pull mode), out_ms[1] = mean
 * duration of the propagation-only kernels (push scatter, final gather),
 * out_ms[2] = mean wall time of a step on the stream, out_ms[3] = mean
 * synaptic events per step. */
int dtb_block_time_kernels(dtb_block* b, int n_steps, float noise_rate, int isolated, int mode, float* out_ms);

/* Schedule knobs (new: the reference has a fixed launch shape per kernel).
 * DTB_TUNE_SCATTER_WORDS   bitmask words per warp in the push scatter (1..32)
 * DTB_TUNE_CHUNK           steps per captured CUDA graph (1..4096)
 * DTB_TUNE_PULL_THRESHOLD_PPM  activity fraction (parts per million of the
 *                          neurons propagating per step) above which
 *                          DTB_MODE_AUTO pulls instead of pushing
 * DTB_TUNE_USE_GRAPHS      capture chunks in CUDA graphs (0/1)
 * DTB_TUNE_STEP_VARIANT    update kernel: 0 = registers for two resident
 *                          CTAs per SM (no spills), 1 = three, 2, 3 and 4 =
 *                          two, three and four with the state of the next
 *                          tile bulk-copied to shared memory while the
 *                          current one computes (default 3; the results are
 *                          bit-identical every way; a network whose J planes
 *                          do not allow the copies runs variant 0 or 1)
 * DTB_TUNE_PULL_METHOD     how DTB_MODE_PULL propagates (bit-identical every
 *                          way): 1 = every postsynaptic row gathers its firing
 *                          inputs; 2 = ordered push: firing rows scatter into
 *                          per-neuron slots that the next update sums in pull
 *                          order; 3 = ordered push: firing rows set one bit per
 *                          pull-row position in per-neuron masks (in-degree up
 *                          to 128) and the next update sums the marked pull
 *                          entries in order (2 and 3 need the push CSR); 4 =
 *                          streamed gather: every warp streams its 128 rows'
 *                          entries in coalesced chunks and adds the firing ones
 *                          in row order; 0 = slots while at most 10 % of the
 *                          neurons propagate, else the streamed gather
 * DTB_TUNE_J_CACHE         0 = the update streams J (evict first), 1 = its J
 *                          stores keep normal L2 priority for the scatter
 * DTB_TUNE_SCATTER_VARIANT push scatter registers: 0 = unbounded, 1 = budgeted
 *                          for six resident CTAs per SM
 * DTB_TUNE_PUSH_METHOD     how DTB_MODE_PUSH adds the weights of firing rows
 *                          (the order of the float additions differs, the sums
 *                          agree to rounding): 1 = one float2 atomic into J per
 *                          synaptic event; 2 = binned: every event is appended
 *                          to the bin of its postsynaptic neuron (a run of 2^B
 *                          neurons) and the next update adds each bin to its
 *                          neurons in shared memory, events past a bin's
 *                          capacity going to J by atomics; 0 = binned whenever
 *                          the network allows it (push CSR, at most 2^28
 *                          neurons) and its bins could be allocated; default 1,
 *                          dtb_block_autotune keeps the faster of 1 and 2
 * DTB_TUNE_BIN_WORDS       binned push: bitmask words (32 neurons each) whose
 *                          firing rows one scatter CTA takes per round (1..256)
 * DTB_TUNE_BIN_CAPACITY    binned push: bin entries per neuron of the bin
 *                          (1..1024, default 8; 10 bytes each); reallocates
 * DTB_TUNE_BIN_SHIFT       binned push: B (10..13), 0 = 10; reallocates; the update stages
 *                          its state (step variants 2..4) only with B = 10
 * DTB_TUNE_SCATTER_REVERSE atomic push scatter: 0 = CTAs take the bitmask from its start,
 *                          1 = from its end (the rows scattered first then target the
 *                          neurons whose J the update wrote last)
 * DTB_TUNE_STAGE_WAIT_LIMIT polls of a staged copy's completion barrier before the
 *                          update gives up on it (default 2^20; 0 gives up at once, for
 *                          tests): the update then loads that state from global memory,
 *                          stops staging for the rest of the launch and the next call that
 *                          reads results returns DTB_ERR_CUDA (the flag is cleared once
 *                          reported; the results themselves are exact) */
enum { DTB_TUNE_SCATTER_WORDS = 0, DTB_TUNE_CHUNK = 1, DTB_TUNE_PULL_THRESHOLD_PPM = 2, DTB_TUNE_USE_GRAPHS = 3,
       DTB_TUNE_STEP_VARIANT = 4, DTB_TUNE_PULL_METHOD = 5, DTB_TUNE_J_CACHE = 6, DTB_TUNE_SCATTER_VARIANT = 7,
       DTB_TUNE_PUSH_METHOD = 8, DTB_TUNE_BIN_WORDS = 9, DTB_TUNE_BIN_CAPACITY = 10, DTB_TUNE_BIN_SHIFT = 11,
       DTB_TUNE_STAGE_WAIT_LIMIT = 12, DTB_TUNE_SCATTER_REVERSE = 13 };
int dtb_block_set_tuning(dtb_block* b, int key, int64_t value);
int dtb_block_get_tuning(dtb_block* b, int key, int64_t* value);

/* Autotuner: times the step kernel's register budgets, the atomic push scatter at 1, 2, 4, ..., 32 bitmask words
 * per warp, the binned push at 64, 128 and 256 words per round (unless DTB_TUNE_PUSH_METHOD is 1) and the pull
 * gather on the live network (n_steps each; the simulation advances), keeps the fastest push method and shape
 * (DTB_TUNE_PUSH_METHOD becomes 1 or 2) and sets the
 * AUTO push/pull threshold from the measured costs at the current activity.
 * report (nullable, 6 floats): words per warp, push ms/step, pull ms/step,
 * activity fraction, threshold, step variant. */
int dtb_block_autotune(dtb_block* b, int n_steps, float noise_rate, float* report);

/* ---- state access ------------------------------------------------------- */

/* Getters of cuda/include/block.hpp:247-562 (get_*_gpu / get_*_cpu) and the
 * public tensors of models/block.py:55-58,84-86,134. */
int dtb_block_get(dtb_block* b, int field, void* dst, int where);
/* Copies the pull (which = 0, rows = postsynaptic neurons) or push (which = 1,
 * rows = presynaptic neurons) CSR: rowptr[N+1] int64, index[S] uint32 (the
 * other endpoint; bit 31 set for a GABAa/GABAb synapse), weight[S][2] float.
 * Any output may be NULL.  The layout of cuda/src/configuration.cpp:783-795
 * (rowptrs, colinds, float2 vals, connkinds) with the kind folded into bit 31. */
int dtb_block_get_csr(dtb_block* b, int which, int64_t* rowptr, uint32_t* index, float* weight, int where);
/* Entries [first, first + count) of the same CSR arrays (index[count], weight[count][2], either nullable):
 * rows of a network too large to copy whole (configuration.cpp reads its tables back by range,
 * cuda/src/configuration.cpp:214-341). */
int dtb_block_get_csr_entries(dtb_block* b, int which, int64_t first, int64_t count, uint32_t* index,
                              float* weight, int where);

/* Overwrite V, J, T_LAST, T or STEP (checkpoint restore, tests). */
int dtb_block_set(dtb_block* b, int field, const void* src, int where);

/* models/block.py:152-170 block.update_property: replace the [N][22]
 * property matrix (and optionally [N][4] decay).  As in the reference, the
 * synaptic current already computed from the old parameters drives the next
 * membrane update. */
int dtb_block_update_property(dtb_block* b, const float* property, const float* decay);

/* cuda/src/stage/property.cpp:146-257 update_prop_cols_kernel,
 * cuda/python/dist_blockwrapper_pytorch.py:446 mul_property_by_subblk
 * (accumulate=False): property column col[i] of every neuron in subblock
 * sub[i] becomes base_value * value[i], base = the value at creation. */
int dtb_block_scale_property_by_subblock(dtb_block* b, int n, const int32_t* sub, const int32_t* col,
                                         const float* value);

/* cuda/src/stage/property.cpp:313-471 (gamma_kernel), cuda/src/block.cpp:815-855
 * update_Gamma_Prop_Cols_gpu, client cuda/python/dist_blockwrapper_pytorch.py:460
 * gamma_property_by_subblk: property column col[i] of every neuron of
 * subblock sub[i] becomes its own draw of Gamma(alpha[i], 1) / beta[i].
 * g_ui columns (10-13) keep one value per neuron (a per-neuron factor on the
 * class value, which becomes 1); any other column takes the delta limit
 * alpha/beta and needs alpha >= 1e6 (the reference's near-delta use,
 * simulation/simulation.py:120-144).  The drawn values become the base of
 * later dtb_block_scale_property_by_subblock calls.  Sampler: Marsaglia &
 * Tsang (2000) on Philox4x32-10 in double precision; the stream is keyed by
 * the block seed, the neuron and a per-block call counter. */
int dtb_block_gamma_property_by_subblock(dtb_block* b, int n, const int32_t* sub, const int32_t* col,
                                         const float* alpha, const float* beta);

/* models/block.py:37-50, :104-109 (block with src): the n_src input neurons
 * `neurons` replay a spike raster, spikes[i][t] (uint8, [n_src][T]) being the
 * spike of input i at the t-th step from now; their other state evolves as
 * usual (noise still ORs into what they propagate).  As in the reference, a
 * raster of T columns serves T - 1 steps: running further fails.  n_src = 0
 * removes the inputs. */
int dtb_block_set_input_spikes(dtb_block* b, int64_t n_src, const uint32_t* neurons, int64_t T,
                               const uint8_t* spikes);

/* models/block.py:172-177 block.update_conn_weight: set the channel weight
 * of existing synapses (channel[i], post[i], pre[i]) to value[i]. */
int dtb_block_update_conn_weight(dtb_block* b, int64_t n, const uint8_t* channel, const uint32_t* post,
                                 const uint32_t* pre, const float* value);

/* Checkpoint of the dynamic state (V, J, t_last, pending I_syn, t, step).
 * No counterpart in the reference (it has none, cuda/protos/snn.proto:62
 * only offsets input-spike timestamps); a restored run continues
 * bit-identically because the noise counter is the step index. */
int dtb_block_save(dtb_block* b, const char* path);
int dtb_block_load(dtb_block* b, const char* path);

/* Sampled neurons (cuda/python/dist_blockwrapper_pytorch.py set_samples,
 * cuda/src/stage/sample.cpp:8): after every step the spike (threshold
 * crossing, noise excluded) and V of the n neurons idx[] are recorded in a
 * device ring of capacity_steps rows.  n = 0 stops sampling. */
int dtb_block_set_samples(dtb_block* b, int n, const uint32_t* idx, int64_t capacity_steps);
/* The recorded rows in step order, oldest first (at most capacity_steps):
 * spikes[rows][n] uint8, v[rows][n] float (either nullable), *rows = count. */
int dtb_block_get_samples(dtb_block* b, uint8_t* spikes, float* v, int64_t* rows, int where);

/* ---- BOLD (models/bold_model_pytorch.py) --------------------------------- */

/* BOLD.__init__ (bold_model_pytorch.py:12-25). dtype: 0 float32, 1 float64.
 * State starts as the reference's first run(): s=0, q=0, v=1, f_in=1. */
int dtb_bold_create(int64_t n_regions, int dtype, double epsilon, double tao_s, double tao_f, double tao_0,
                    double alpha, double E_0, double V_0, double delta_t, int device, dtb_bold** out);
int dtb_bold_destroy(dtb_bold* m);
int dtb_bold_set_stream(dtb_bold* m, void* stream);
/* BOLD.run (bold_model_pytorch.py:43-78): one Euler step, u -> out, both [R] of the model's dtype. */
int dtb_bold_run(dtb_bold* m, const void* u, void* out, int where);
/* n_steps x BOLD.run with a constant input u[r] (floored at u_floor, as
 * simulation/simulation.py:279 floors at 1e-5); out = the last step's
 * signal.  Integrates the hemodynamics of a window whose rate is forecast
 * instead of simulated. */
int dtb_bold_run_steps(dtb_bold* m, const void* u, int n_steps, double u_floor, void* out, int where);
/* BOLD.state_update (bold_model_pytorch.py:34-41): w is [E][Rp][S] of the
 * model's dtype with E*Rp == R; s = w[..,0], q = max(w[..,1],1e-5),
 * v = max(w[..,2],1e-5), f_in = max(w[..,3],1e-5). */
int dtb_bold_state_update(dtb_bold* m, const void* w, int64_t E, int64_t Rp, int64_t S, int where);
/* field: 0 s, 1 q, 2 v, 3 f_in; dst [R] of the model's dtype. */
int dtb_bold_get(dtb_bold* m, int field, void* dst, int where);
int dtb_bold_set(dtb_bold* m, int field, const void* src, int where);

/* Per-step BOLD driven by the block (simulation/simulation.py:269-279):
 * after every step, act[r] = (spikes of the subblocks mapped to region r) /
 * (neurons of those subblocks); BOLD.run(max(act, 1e-5)) in float64 with the
 * given delta_t (seconds per step, e.g. 1e-4 for dt = 0.1 ms).
 * sub_to_region[n_sub] (host) maps subblocks to regions (-1: none). */
int dtb_block_attach_bold(dtb_block* b, int n_regions, const int32_t* sub_to_region,
                          double epsilon, double tao_s, double tao_f, double tao_0, double alpha,
                          double E_0, double V_0, double delta_t);
/* field: 0 s, 1 q, 2 v, 3 f_in, 4 bold output of the last step, 5 act of the last step; double[R]. */
int dtb_block_get_bold(dtb_block* b, int field, double* dst, int where);
/* Overwrite the attached BOLD state (field 0 s, 1 q, 2 v, 3 f_in; double[R]): the
 * bold.state_update after an ensemble Kalman filter step
 * (data_assimilation/DataAssimilation.py:400). */
int dtb_block_set_bold(dtb_block* b, int field, const double* src, int where);

/* ---- surrogate forecast network ------------------------------------------- */

/* No counterpart in the reference (its EnKF forecast always runs the
 * simulator, data_assimilation/DataAssimilation.py:353-370).  A multilayer
 * perceptron in_dim -> hidden -> hidden -> 1 with GELU: BF16 weights for
 * compute, FP32 master weights, FP32 activations and accumulation; forward,
 * MSE backward and Adam are CUDA kernels.  Flat parameter order (FP32):
 * W1[hidden][in_dim], b1[hidden], W2[hidden][hidden], b2[hidden], W3[hidden], b3.
 * x / target / y / grad pointers are device memory; calls are asynchronous on
 * the handle's stream (dtb_mlp_set_stream). */
typedef struct dtb_mlp dtb_mlp;
int dtb_mlp_create(int in_dim, int hidden, uint64_t seed, int device, dtb_mlp** out);
int dtb_mlp_destroy(dtb_mlp* m);
int dtb_mlp_set_stream(dtb_mlp* m, void* stream);
int dtb_mlp_n_params(const dtb_mlp* m, int64_t* n);
int dtb_mlp_get_params(dtb_mlp* m, float* dst, int where);
int dtb_mlp_set_params(dtb_mlp* m, const float* src, int where);
/* y[B] = MLP(x[B][in_dim]) */
int dtb_mlp_forward(dtb_mlp* m, const float* x, int64_t B, float* y);
/* gradient of mean((MLP(x) - target)^2) into grad[n_params] and the loss into *loss (both nullable) */
int dtb_mlp_gradient(dtb_mlp* m, const float* x, const float* target, int64_t B, float* grad, float* loss);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8) on that loss */
int dtb_mlp_train_step(dtb_mlp* m, const float* x, const float* target, int64_t B, float lr, float* loss);
int dtb_mlp_last_error(char* buf, size_t len);

/* ---- one step without any allocation ------------------------------------ */

/* One parameter class (a deduplicated property row with its derived
 * constants), in the layout the step kernels read.  rC_dt = (1.0f / C) * dt
 * and decay[c] = expf(-dt / tau_c) (as float32 operations, tau_c = property
 * cols 18-21) reproduce models/block.py:71,92. */
typedef struct {
    float g[4];      /* g_ui (property cols 10-13) */
    float V_ui[4];   /* cols 14-17 */
    float decay[4];  /* exp(-dt / tau_ui), tau = cols 18-21 */
    float g_L, V_L;  /* cols 6, 7 */
    float rC_dt;     /* (1 / C) * dt, C = col 4 */
    float V_th, V_reset, T_ref, I_ext, noise_rate;  /* cols 8, 9, 5, 2, 0 */
    int32_t subblock;                               /* col 3, -1 when not a whole number >= 0 */
    float C, pad0, pad1;
} dtb_param_class;

/* A network whose device arrays all belong to the caller. */
typedef struct {
    int64_t n_neurons;                /* <= DTB_PREALLOC_MAX_NEURONS */
    int32_t n_subblocks;              /* <= DTB_PREALLOC_MAX_SUBBLOCKS */
    int32_t device;
    float* V;                         /* [N] in/out */
    float* J;                         /* [N][4] in/out (AMPA, NMDA, GABAa, GABAb per neuron) */
    float* t_last;                    /* [N] in/out */
    const uint32_t* cls;              /* [N] class of every neuron */
    const dtb_param_class* classes;   /* class table */
    const uint32_t* sub_count;        /* [n_subblocks] neurons per subblock (divides the mean V) */
    const int64_t* rowptr;            /* pull CSR: [N+1], rows = postsynaptic neurons */
    const uint32_t* index;            /* [S] presynaptic neuron | bit 31 for a GABAa/GABAb synapse */
    const float* weight;              /* [S][2] */
    float dt;
    uint64_t seed;
    uint32_t stream_id;
} dtb_prealloc_net;

#define DTB_PREALLOC_MAX_NEURONS (1 << 22)
#define DTB_PREALLOC_MAX_SUBBLOCKS 1024

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory themselves or let a library do it: code that runs inside another
 * framework's fixed memory pool or budget, or a real-time loop in which an
 * allocation (and the device-wide synchronisation cudaMalloc/cudaFree can
 * bring) is not allowed.  It advances such a caller-owned network by one time
 * step, exactly as dtb_block_run(..., DTB_MODE_PULL, ...) advances a handle
 * (bit-identical results), and calls no cudaMalloc, cudaFree or allocating
 * library routine.
 *
 * Its scratch memory (spike bitmasks, subblock accumulators, control block;
 * about 1.05 MB) is one fixed static device array inside libdtb.so, which
 * every GPU that loads the library holds until the process exits; hence the
 * limits DTB_PREALLOC_MAX_NEURONS and DTB_PREALLOC_MAX_SUBBLOCKS, beyond which
 * the call returns DTB_ERR_LIMIT (bad pointers or dt: DTB_ERR_ARG; a failed
 * launch: DTB_ERR_CUDA; this call reports by status code only; a CUDA error left
 * pending on the calling thread by earlier, unrelated work is reported through
 * this call as DTB_ERR_CUDA too).  The first call on a device is the warm-up:
 * it looks up the array's device address (with that device current) and, under
 * CUDA's lazy module loading (the default), that lookup loads the kernels and
 * the array, which can allocate and synchronise once.  Make that first call
 * before entering a loop that must not allocate and before any stream capture,
 * or set CUDA_MODULE_LOADING=EAGER.  All calls share the array and every call
 * re-initialises what it uses, but calls whose work overlaps on the GPU (two
 * streams, two host threads) race on it: serialise them.
 *
 * Preconditions the call does not check (the kernels index with these values;
 * an array that breaks them makes the kernels read outside the arrays): every
 * (index[e] & 0x7fffffff) < n_neurons; rowptr non-decreasing with rowptr[0] = 0
 * and rowptr[n_neurons] = the number of synapses; every cls[n] below the number
 * of rows of `classes`; every class's subblock below n_subblocks or -1.
 *
 * t is block.t before the step and step the number of steps already taken
 * (the noise counter); after the call block.t is float32(t + dt).  sum_out /
 * mean_out (device, [n_subblocks], nullable) receive the step's spike count
 * and mean V per subblock.  Work is issued on `stream` (a cudaStream_t,
 * NULL = legacy default stream); the call does not synchronise. */
int dtb_step_preallocated(const dtb_prealloc_net* net, float t, uint64_t step, float noise_rate, int isolated,
                          float* sum_out, float* mean_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DTB_H */
