/*
 * CPU ORACLE — test infrastructure only.
 *
 * This file is the checker for the CUDA product in digital_twin_brain_b200/.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load it. It is never linked into, or called by, the product path.
 *
 * It restates, in plain C with the same float32 operation order, the
 * reference's CPU time step and BOLD model:
 *
 *   - models/block.py:89-111   block.update_Vi   (leak + synaptic + external
 *                               current, refractory test, threshold, clamp)
 *   - models/block.py:133-142  block.run         (t += dt, Poisson noise OR,
 *                               J update, I_syn, t_ik_last)
 *   - models/block.py:68-81    block.update_J_ui + bmm (J*exp(-dt/tau) + W.active;
 *                               torch.sparse.mm accumulates every postsynaptic
 *                               row in COO nnz order, which the pull CSR keeps)
 *   - models/block.py:83-87    block.update_I_syn (I_ui = g (V_ui - V) J;
 *                               I_syn summed AMPA, NMDA, GABAa, GABAb in order)
 *   - models/bold_model_pytorch.py:43-78  BOLD.run (Euler step of s, q, v, f_in;
 *                               q before v before f_in before s)
 *
 * Pinning: tests/golden/make_golden.py runs the reference's own models/block.py
 * and models/bold_model_pytorch.py (torch 2.11 CPU) with torch.rand replaced by
 * the Philox stream below, and tests/test_oracle_golden.py checks this oracle
 * against those fixtures bit for bit (block step) and to 1e-6 relative (BOLD,
 * where torch's pow and libm's powf may differ by an ulp).
 *
 * Philox4x32-10 is written from Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3" (SC'11), and checked against that paper's
 * published known-answer vectors in tests/test_oracle_golden.py.
 *
 * The synthetic network generator (oracle_gen_rows) restates the product's
 * counter-based generator so that networks of any size can be checked row by
 * row without running the GPU.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ Philox */

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4])
{
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += PHILOX_W0; k1 += PHILOX_W1; }
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float u01_from_bits(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

/*
 * Noise uniform of neuron n at step `step`, stream `stream`, seed `seed`.
 * Counter index q = (n / 128) * 32 + n % 32, output word (n / 32) % 4,
 * counter = {q, stream, step_lo, step_hi}, key = {seed_lo, seed_hi}.
 */
void oracle_noise_uniforms(uint64_t seed, uint32_t stream, uint64_t step, int64_t n, float* out)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    #pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < (n + 127) / 128; ++g) {
        for (int lane = 0; lane < 32; ++lane) {
            uint64_t q = (uint64_t)g * 32 + lane;
            uint32_t ctr[4] = {(uint32_t)q, stream, (uint32_t)step, (uint32_t)(step >> 32)};
            uint32_t o[4];
            oracle_philox4x32_10(ctr, key, o);
            for (int w = 0; w < 4; ++w) {
                int64_t i = g * 128 + w * 32 + lane;
                if (i < n) out[i] = u01_from_bits(o[w]);
            }
        }
    }
}

/* ------------------------------------------------------------- block step */

/*
 * One call == one block.run(noise_rate, isolated) (models/block.py:116-150),
 * excluding the per-subblock statistics, which the caller computes.
 *
 * Per-neuron parameters are channel-major where they have 4 channels
 * (g, Vu, decay: [4][N]), as block.update_property splits them
 * (models/block.py:152-170). decay = exp(-dt / tau_ui) is passed in
 * because the reference evaluates it with torch.exp.
 *
 * Synapses are a pull CSR: rowptr[N+1] over postsynaptic neurons, each entry
 * (pre, kind in {0,2}, w[2]) adds w[0] to channel kind and w[1] to kind+1
 * (generation/read_block.py:68-74). Entries of a row are accumulated in
 * array order starting from +0, which is torch.sparse.mm's order.
 *
 * State in/out: V[N], J[4][N], tlast[N], Isyn[N], *t.
 * noise_rate >= 0: scalar rate (block.py:136); < 0: per-neuron rates.
 * forced_* (nullable): teacher forcing of this step's active / new_active;
 * a forced_active value of 2 keeps the computed spike of that neuron (input
 * neurons replay their raster, the others run free: models/block.py:104-106).
 */
int oracle_block_step(int64_t N,
                      const float* Iext, const float* C, const float* Tref,
                      const float* gL, const float* VL, const float* Vth, const float* Vreset,
                      const float* g, const float* Vu, const float* decay,
                      const int64_t* rowptr, const uint32_t* pre, const uint8_t* kind, const float* w,
                      float* V, float* J, float* tlast, float* Isyn, float* t_io, float dt,
                      float noise_rate, const float* noise_per_neuron,
                      uint64_t seed, uint32_t stream, uint64_t step, int isolated,
                      const uint8_t* forced_active, const uint8_t* forced_new_active,
                      uint8_t* active_out, uint8_t* new_active_out, float* Iui_out,
                      int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    const float t = *t_io + dt;  /* block.py:133, float32 accumulation */
    *t_io = t;
    float* u = (float*)malloc(sizeof(float) * (size_t)(N > 0 ? N : 1));
    if (!u) return -1;
    oracle_noise_uniforms(seed, stream, step, N, u);

    /* update_Vi (block.py:89-111) + noise (block.py:135-138) */
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        float v = V[i];
        float main_part = (-gL[i]) * (v - VL[i]);
        float cdiff = (main_part + Isyn[i]) + Iext[i];
        float rcdt = (1.0f / C[i]) * dt;           /* torch: C.reciprocal() * dt */
        float vn = v + rcdt * cdiff;
        int not_sat = (t >= tlast[i] + Tref[i]);
        float vsel = not_sat ? vn : Vreset[i];
        int act = (vsel >= Vth[i]);
        float vth = Vth[i];
        float vmin = isnan(vsel) ? vsel : (isnan(vth) ? vth : (vsel < vth ? vsel : vth));
        V[i] = vmin;
        if (forced_active && forced_active[i] != 2) act = forced_active[i] != 0;
        float rate = noise_rate >= 0.0f ? noise_rate : noise_per_neuron[i];
        int noise = u[i] < rate;
        int na = isolated ? noise : (noise | act);
        if (forced_new_active) na = forced_new_active[i] != 0;
        active_out[i] = (uint8_t)act;
        new_active_out[i] = (uint8_t)na;
    }
    free(u);

    /* update_J_ui (block.py:68-74) with bmm in nnz order (block.py:77-79),
       update_I_syn (block.py:83-87), update_t_ik_last (block.py:113-114) */
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < N; ++i) {
        float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int64_t e = rowptr[i]; e < rowptr[i + 1]; ++e) {
            if (new_active_out[pre[e]]) {
                int c = kind[e];
                s[c] = s[c] + w[2 * e];
                s[c + 1] = s[c + 1] + w[2 * e + 1];
            }
        }
        float v = V[i];
        float isum = 0.0f;
        for (int c = 0; c < 4; ++c) {
            int64_t k = (int64_t)c * N + i;
            float jd = J[k] * decay[k];
            float jn = jd + s[c];
            J[k] = jn;
            float iu = (g[k] * (Vu[k] - v)) * jn;
            if (Iui_out) Iui_out[k] = iu;
            isum = (c == 0) ? iu : (isum + iu);
        }
        Isyn[i] = isum;
        if (active_out[i]) tlast[i] = t;
    }
    return 0;
}

/* ------------------------------------------------------------------- BOLD */

/*
 * One BOLD.run(u) (models/bold_model_pytorch.py:43-78) on R regions, float32.
 * State arrays s, q, v, f are in/out and must be initialised by the caller
 * (s=0, q=0, v=1, f=1 for a fresh model, bold_model_pytorch.py:60-67).
 */
void oracle_bold_step_f32(int64_t R, const float* u, float* s, float* q, float* v, float* f,
                          float* out, double epsilon, double tao_s, double tao_f, double tao_0,
                          double alpha, double E0, double V0, double delta_t)
{
    /* Python scalars meet float32 tensors: each is rounded to float32 where
       the tensor op consumes it (bold_model_pytorch.py:21,69-77). */
    const double div_alpha = 1.0 / alpha;
    const float eps_f = (float)epsilon, ts_f = (float)tao_s, tf_f = (float)tao_f, t0_f = (float)tao_0;
    const float E0_f = (float)E0, V0_f = (float)V0, dt_f = (float)delta_t;
    const float base = (float)(1.0 - E0);
    const float ex_q = (float)(div_alpha - 1.0), ex_v = (float)div_alpha;
    const float k7 = (float)(7.0 * E0);
    const float k2 = (float)(2.0 * E0 - 0.2);
    for (int64_t i = 0; i < R; ++i) {
        float fi = f[i], si = s[i], qi = q[i], vi = v[i];
        float ds = ((u[i] * eps_f) - si / ts_f) - (fi - 1.0f) / tf_f;
        float qpart = fi > 0.0f ? (1.0f - powf(base, (1.0f / fi) * 1.0f)) : 1.0f;
        float dq = (((fi * qpart) / E0_f) - qi * powf(vi, ex_q)) / t0_f;
        qi = qi + dq * dt_f;
        float dv = (fi - powf(vi, ex_v)) / t0_f;
        vi = vi + dv * dt_f;
        fi = fi + si * dt_f;
        fi = fi > 0.0f ? fi : 0.0f;
        si = si + ds * dt_f;
        s[i] = si; q[i] = qi; v[i] = vi; f[i] = fi;
        out[i] = ((k7 * (1.0f - qi) + (1.0f - qi / vi) * 2.0f) + k2 * (1.0f - vi)) * V0_f;
    }
}

void oracle_bold_step_f64(int64_t R, const double* u, double* s, double* q, double* v, double* f,
                          double* out, double epsilon, double tao_s, double tao_f, double tao_0,
                          double alpha, double E0, double V0, double delta_t)
{
    const double div_alpha = 1.0 / alpha;
    const double base = 1.0 - E0;
    for (int64_t i = 0; i < R; ++i) {
        double fi = f[i], si = s[i], qi = q[i], vi = v[i];
        double ds = ((epsilon * u[i]) - si / tao_s) - (fi - 1.0) / tao_f;
        double qpart = fi > 0.0 ? (1.0 - pow(base, 1.0 / fi)) : 1.0;
        double dq = (((fi * qpart) / E0) - qi * pow(vi, div_alpha - 1.0)) / tao_0;
        qi = qi + dq * delta_t;
        double dv = (fi - pow(vi, div_alpha)) / tao_0;
        vi = vi + dv * delta_t;
        fi = fi + si * delta_t;
        fi = fi > 0.0 ? fi : 0.0;
        si = si + ds * delta_t;
        s[i] = si; q[i] = qi; v[i] = vi; f[i] = fi;
        out[i] = V0 * ((7.0 * E0 * (1.0 - qi) + 2.0 * (1.0 - qi / vi)) + (2.0 * E0 - 0.2) * (1.0 - vi));
    }
}

/* ------------------------------------------------------ synthetic network */

/*
 * Counter-based synthetic network (the product's generator, restated).
 * Regions r = 0..R-1 own neuron ranges [region_start[r], region_start[r+1]);
 * the first region_n_exc[r] neurons of a region are excitatory.
 * Every postsynaptic neuron i (region ri) draws K distinct presynaptic
 * neurons, never itself: a source region by its cumulative row (region =
 * number of cum entries <= u among all but the last, as
 * numpy.searchsorted(cum[:-1], u, 'right') in generation/make_block.py:290),
 * then a neuron uniformly inside it.  Candidates come two per Philox call:
 * counter {l_lo, TAG_SRC, attempt, l_hi} (l = row index within its member),
 * words (0,1) and (2,3).  The row is
 * then sorted by presynaptic index; entry j gets the weight pair from counter
 * {l_lo, TAG_W, j/2, l_hi} (words 0,1 for even j, 2,3 for odd j), each
 * U[0,1) * w_scale, and kind 0 (source excitatory -> AMPA/NMDA) or 2
 * (source inhibitory -> GABAa/GABAb), as generation/make_block.py:290-291.
 */
#define TAG_SRC 0xF0000001u
#define TAG_W   0xF0000002u

static int cmp_u64(const void* a, const void* b)
{
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static int region_of(int64_t n, int R, const int64_t* region_start)
{
    int lo = 0, hi = R - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) / 2;
        if (region_start[mid] <= n) lo = mid; else hi = mid - 1;
    }
    return lo;
}

/* rows [row_begin, row_end): writes K entries per row into pre/kind/w (row-local offsets).
 * General form: a row of region r draws its source region from the cumulative
 * row cum_flat[cum_off[r] .. + src_count[r]) as region src_base[r] + #{k <
 * src_count[r]-1 : cum <= u}; rows of member m = region_member[r] use the
 * member-local index l = i - member_start[m] in the Philox counters and the
 * key member_seed[m], so a member generated inside an ensemble equals the
 * same member generated alone. */
int oracle_gen_rows(int R, const int64_t* region_start, const int64_t* region_n_exc,
                    const int32_t* src_base, const int32_t* src_count, const int64_t* cum_off, const float* cum_flat,
                    const int32_t* region_member, const int64_t* member_start, const uint64_t* member_seed,
                    int K, float w_scale, int64_t row_begin, int64_t row_end,
                    uint32_t* pre, uint8_t* kind, float* w)
{
    int bad = 0;
    #pragma omp parallel for schedule(dynamic, 64) reduction(+:bad)
    for (int64_t i = row_begin; i < row_end; ++i) {
        uint64_t* chosen = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)K);
        int ri = region_of(i, R, region_start);
        const float* c = cum_flat + cum_off[ri];
        const int cnt = src_count[ri], sbase = src_base[ri];
        const int m = region_member[ri];
        const uint64_t l = (uint64_t)(i - member_start[m]);
        uint32_t key[2] = {(uint32_t)member_seed[m], (uint32_t)(member_seed[m] >> 32)};
        int have = 0;
        uint32_t attempt = 0;
        while (have < K) {
            if (attempt > (uint32_t)(64 * K + 1024)) { bad += 1; break; }
            uint32_t ctr[4] = {(uint32_t)l, TAG_SRC, attempt, (uint32_t)(l >> 32)};
            uint32_t o[4];
            oracle_philox4x32_10(ctr, key, o);
            attempt++;
            for (int h = 0; h < 2 && have < K; ++h) {
                float ur = u01_from_bits(o[2 * h]);
                int r = sbase;
                for (int j = 0; j < cnt - 1; ++j) r += (c[j] <= ur);
                int64_t size = region_start[r + 1] - region_start[r];
                if (size <= 0) continue;
                uint64_t off = ((uint64_t)o[2 * h + 1] * (uint64_t)size) >> 32;
                int64_t src = region_start[r] + (int64_t)off;
                if (src == i) continue;
                int dup = 0;
                for (int k = 0; k < have; ++k) if ((int64_t)chosen[k] == src) { dup = 1; break; }
                if (dup) continue;
                chosen[have++] = (uint64_t)src;
            }
        }
        qsort(chosen, (size_t)have, sizeof(uint64_t), cmp_u64);
        int64_t base = (i - row_begin) * (int64_t)K;
        for (int j = 0; j < K; ++j) {
            if (j >= have) { pre[base + j] = 0; kind[base + j] = 0; w[2 * (base + j)] = 0; w[2 * (base + j) + 1] = 0; continue; }
            int64_t src = (int64_t)chosen[j];
            int rs = region_of(src, R, region_start);
            pre[base + j] = (uint32_t)src;
            kind[base + j] = (src - region_start[rs] >= region_n_exc[rs]) ? 2 : 0;
            uint32_t ctr[4] = {(uint32_t)l, TAG_W, (uint32_t)(j >> 1), (uint32_t)(l >> 32)};
            uint32_t o[4];
            oracle_philox4x32_10(ctr, key, o);
            int h = j & 1;
            w[2 * (base + j)] = u01_from_bits(o[2 * h]) * w_scale;
            w[2 * (base + j) + 1] = u01_from_bits(o[2 * h + 1]) * w_scale;
        }
        free(chosen);
    }
    return bad;
}

/* --------------------------------------------------------- gamma properties */
/* Per-neuron Gamma(alpha, 1) / beta draws of gamma-distributed properties
 * (cuda/src/stage/property.cpp:313-344 sample_gamma uses the same method):
 * Marsaglia & Tsang, ACM TOMS 26(3) 2000, with the alpha < 1 boost
 * G(alpha) = G(alpha + 1) U^(1/alpha) and Box-Muller normals, in double, on
 * Philox4x32-10 with counter {n_lo, n_hi, attempt, tag} and key
 * {seed_lo, seed_hi ^ 0x47414D4D}; tag = 0x80000000 | receptor << 24 | call;
 * at most 64 attempts, then the mode d. */
static double gamma_u24(uint32_t x, int open_zero)
{
    return ((double)(x >> 8) + (open_zero ? 1.0 : 0.0)) * (1.0 / 16777216.0);
}

double oracle_gamma_unit(double alpha, uint64_t seed, uint64_t n, uint32_t tag)
{
    if (!(alpha > 0.0)) return 0.0;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x47414D4Du};
    uint32_t o[4];
    double scale = 1.0;
    if (alpha < 1.0) {
        const uint32_t ctr[4] = {(uint32_t)n, (uint32_t)(n >> 32), 0xffffffffu, tag};
        oracle_philox4x32_10(ctr, key, o);
        scale = pow(gamma_u24(o[0], 1), 1.0 / alpha);
        alpha += 1.0;
    }
    const double d = alpha - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    for (uint32_t it = 0; it < 64u; ++it) {
        const uint32_t ctr[4] = {(uint32_t)n, (uint32_t)(n >> 32), it, tag};
        oracle_philox4x32_10(ctr, key, o);
        const double u1 = gamma_u24(o[0], 1), u2 = gamma_u24(o[1], 0);
        const double x = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        const double y = 1.0 + c * x;
        if (y <= 0.0) continue;
        const double v = y * y * y;
        const double u = gamma_u24(o[2], 1);
        const double xx = x * x;
        if (u < 1.0 - 0.0331 * xx * xx) return scale * d * v;
        if (log(u) < 0.5 * xx + d * (1.0 - v + log(v))) return scale * d * v;
    }
    return scale * d;
}

void oracle_gamma(int64_t count, const int64_t* neuron, double alpha, double beta, int receptor, uint32_t call,
                  uint64_t seed, float* out)
{
    const uint32_t tag = 0x80000000u | ((uint32_t)receptor << 24) | (call & 0x00ffffffu);
    for (int64_t i = 0; i < count; ++i)
        out[i] = (float)(oracle_gamma_unit(alpha, seed, (uint64_t)neuron[i], tag) / beta);
}
