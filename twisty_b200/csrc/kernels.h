// kernels.h -- launch interface between the host runtime (runtime.cpp) and the CUDA
// translation units. Plain structs and host functions only; each launcher enqueues on the
// given stream and returns the launch error.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace twisty {

// One Monte Carlo pass over one experiment.
struct ChainSpec {
    uint32_t n_segments;     // N
    float arclength;         // S
    float ds;                // S/N (float, as the reference: FullExperimentRunnerOptimalPerturb.cpp:57)
    float inv_ds;            // (float)N / S (CurvePerturbUtils.cpp:160)
    uint64_t seed;
    uint32_t experiment;     // Philox stream id
    uint32_t chain0;         // global id of chain 0
    uint32_t n_chains;
    uint32_t steps;          // weighted steps of every chain but the last
    uint32_t last_steps;     // weighted steps of the last chain
    uint32_t burn_in;        // unweighted steps at the start of every chain
    uint32_t k_eff;          // min(k_max, N-2)
    float max_angle;
    double absorption_factor;// exp(-mu_a * ds) as the reference computes it (float exp, promoted)
    float eval_shift[3];     // receiver shift applied only when weighting
    int has_eval_shift;
    uint32_t incr_resync;    // compensated form: > 1 selects incremental weight updates with a
                             // full recompute every incr_resync-th weighted step (fixed-point,
                             // unclamped tables, forward passes); 0 or 1: full recompute every step
};

// Float table metadata (BaseWeightLookupTable accessors).
struct LutMetaF {
    float min_k, max_k, step;
    int32_t bins;
};

// Per-chain outcome, identical for every form.
struct ChainOut {
    double log10_sum;        // log10 of the chain's summed path weights (-inf if none)
    uint32_t valid;          // weighted paths with a finite weight
    uint32_t failed;         // NaN weights
    uint32_t clamped;        // curvatures outside the table, clamped
    uint32_t pad;
};

// Result of the FP64 global reduction.
struct ReduceOut {
    double log10_sum;        // log10 sum over chains
    double rel_se;           // standard error of the sum / the sum (spread over chains)
    double max_chain_log10;
    uint64_t valid, failed, clamped;
};

// ---------------------------------------------------------------- tables (lut.cu)
// Simpson quadrature of the reference's table (PathWeightUtils.cpp:281-433) in FP64:
// faithful=1 reproduces the reference's float phase function and float-pi constants,
// faithful=0 is double throughout. Writes out64[bins] (nullable) and out32[bins] (nullable).
struct LutBuildSpec {
    float mu, eps, scatter, min_bound, max_bound, bias;
    uint32_t num_steps_int;
    uint32_t bins;
    float ds;
    float min_k, step;       // the float grid (faithful) ...
    double step64;           // ... and its double twin
    int faithful;
    int derivatives;         // also d/d(mu_s) and d/d(eps) tables (adjoint)
};
cudaError_t launch_lut_build(const LutBuildSpec &s, double *out64, double *d_mus, double *d_eps,
                             cudaStream_t st);
// Non-positive entries replaced by the smallest non-negative one (PathWeightUtils.cpp:
// 327-344); min/max returned through minmax[2]; float copy written to out32.
cudaError_t launch_lut_finalize(uint32_t bins, double *lut64, float *out32, double *minmax, cudaStream_t st);
// Batches of n tables of `bins` entries, table x at offset x*bins: build (specs in device
// memory, derivatives off), finalize (minmax + 3x), and the compensated-form tables (struct
// LogFixed below; steps[x] = bin width, nsegs[x] = N of the paths the fixed point is scaled
// for, ok[x] = 1 when the fixed-point form is usable).
cudaError_t launch_lut_build_batch(const LutBuildSpec *d_specs, uint32_t n, uint32_t bins, double *out64,
                                   cudaStream_t st);
cudaError_t launch_lut_finalize_batch(uint32_t n, uint32_t bins, double *lut64, float *out32, double *minmax,
                                      cudaStream_t st);
struct LogFixed;
cudaError_t launch_comp_tables_batch(uint32_t n, uint32_t bins, const float *lut32, const float *steps,
                                     const uint32_t *nsegs, float2 *fix, float2 *lin, LogFixed *lf, int *ok,
                                     cudaStream_t st);

// ------------------------------------------------------------- chains (chain_*.cu)
cudaError_t launch_plain_chains(const ChainSpec &c, const float *init_pos, float *state,
                                const float *lut, LutMetaF m, ChainOut *out, cudaStream_t st,
                                float *exp_pos = nullptr, double *exp_w = nullptr);
// Plain-form state of one chain: positions (N+1)*3, tangents N*3, curvatures N-1,
// padded to a multiple of 4 floats.
__host__ __device__ inline size_t plain_state_floats_per_chain(uint32_t n)
{
    const size_t f = 3 * (size_t)(n + 1) + 3 * (size_t)n + (n - 1);
    return (f + 3) & ~(size_t)3;
}

cudaError_t launch_fp64_chains(const ChainSpec &c, const float *init_pos, double *state,
                               const double *lut, double min_k, double max_k, double step,
                               int32_t bins, ChainOut *out, cudaStream_t st);

// Compensated form. init_seg holds the N initial segment vectors (float3, x_{i+1}-x_i).
//
// Fixed-point form of the compensated log table: entry i of the float2 table holds
// round((log10 L_i - c0) * 2^s) as uint32 bits in .x (every entry at least 64) and the change
// of log10 of the blend across the bin in .y; a path's log10 weight is (N-1) c0 + (its integer
// total) * 2^-s, the total being the sum of its entries plus its rounded interpolation
// corrections. Narrow tables (wide = 0) keep (N+1) * max entry < 2^31: path totals and their
// differences are exact in 32 bits. Wide tables (wide = 1, long paths or wide-ranging tables)
// keep 32 * max entry < 2^32: a lane's sum of at most 32 entries is exact in 32 bits, path
// totals and differences are 64-bit. inv_scale = 0 selects the exact (L_i, L_{i+1}-L_i) table.
struct LogFixed {
    double c0;
    double inv_scale;
    int32_t wide;
    int32_t steep;           // bins whose secant slope is NaN (paths crossing them are re-weighed exactly)
};
struct CompTuning {
    int group;               // lanes per chain (1, 4, 8, 16, 32)
    int spl;                 // segments per lane
    int warps_per_block;
    int exact_blend;         // 1: interpolate the linear table and take log2 (MUFU)
    int lut_global = 0;      // 1: gather the table through L1 instead of staging it in shared memory
                             // (forward passes only; the chain state keeps the shared memory)
};
// The default shape of N segments for a pass of `paths` weighted paths with `burn_in` steps per
// chain (the defaults: a long pass); batched: among the shapes the batched kernels have.
CompTuning comp_default_tuning(uint32_t n_segments, bool batched = false, uint64_t paths = ~0ull,
                               uint64_t burn_in = 0);
int comp_stage_min_warps(const CompTuning &t);
bool comp_tuning_supported(const CompTuning &t, uint32_t n_segments, uint32_t k_eff);
size_t comp_smem_bytes(const CompTuning &t, uint32_t bins);
// Shared memory a CTA may use (B200: 227 KB).
constexpr size_t kCompSmemCap = 227 * 1024;
// Table placement of a forward pass of the full recompute: true when the table is gathered
// through L1 at the shape's warps, because staging it would leave fewer than
// comp_stage_min_warps(t) warps (or does not fit at all). may_shrink false: the warps were set
// by the caller and stay.
bool comp_table_through_l1(const CompTuning &t, uint32_t bins, bool may_shrink);
// Fewer warps per CTA (steps of 4, down to 4) until the chain state, and the table when it is
// staged (t.lut_global = 0), fit in shared memory; false when they do not fit even then.
bool comp_fit_smem(CompTuning &t, uint32_t bins, bool may_shrink);
cudaError_t launch_comp_chains(const ChainSpec &c, const CompTuning &t, const float *init_seg,
                               const float2 *fixtab, const float2 *lintab, LutMetaF m,
                               ChainOut *out, double2 *block_partials, cudaStream_t st,
                               LogFixed lf = LogFixed{0.0, 0.0});
uint32_t comp_blocks(const ChainSpec &c, const CompTuning &t);
// Replay of chains that also writes every weighted path: positions x_0 + prefix sums of the
// segment vectors (exp_pos[chain][step][N+1][3]) and log10 weights (exp_w[chain][step]).
cudaError_t launch_comp_export(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *fixtab,
                               const float2 *lintab, LutMetaF m, const float x0[3], float *exp_pos, double *exp_w,
                               ChainOut *out, cudaStream_t st, LogFixed lf = LogFixed{0.0, 0.0});
// Adjoint replay: per chain the weight-averaged gradients of log10 w with respect to
// (mu_s, eps, receiver x, y, z) and the sum of the weights w/10^ref_log10, reduced over
// chains into grad_out[6]. dtab: the derivative tables as launch_deriv_tables lays them out.
cudaError_t launch_comp_adjoint(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *lintab,
                                LutMetaF m, const float4 *dtab, float ref_log10, double *grad_chains, double *grad_out,
                                cudaStream_t st);

// Batched persistent form: one launch runs the chains of many experiments that share a
// kernel shape. Work items (experiment, first chain) are taken from *d_counter (zeroed by
// the caller) by persistent CTAs; each experiment's chains write out[out_offset + chain].
struct BatchShape {
    int group, spl, warps;
    int exact;               // tables are (L_i, L_{i+1}-L_i) with a log2 per segment
    int lut_smem;            // stage each item's table in shared memory (else read through L1)
    int clamp;               // some table's curvature range can be left (else no clamping code)
    int steep;               // fixed-point kernel with the steep-bin fallback (paths crossing a
                             // NaN-slope bin re-weighed through the linear table); fixed-point
                             // kernels have it exactly when lut_smem is set
};
// Whether curvatures of paths with this N/S can leave the table (it does not cover
// [0, 2 N/S] from 0): such tables need the clamping kernel variants.
bool comp_table_needs_clamp(float inv_ds, const LutMetaF &m);
struct BatchExpHost {
    ChainSpec spec;
    LutMetaF meta;
    LogFixed lf;
    const float2 *tab;       // device table of meta.bins entries in the shape's form
    const float2 *lin;       // device linear table of the same curve (steep-bin fallback)
    const float *init_seg;   // device initial segment vectors
    uint32_t out_offset;
};
size_t batch_exp_bytes();
void batch_pack_experiments(const BatchExpHost *in, uint32_t n, void *dst);
bool batch_shape_supported(const BatchShape &s, uint32_t n_max, uint32_t k_eff);
// Threads per CTA the batched kernel of a shape is compiled for (8-lane and narrower shapes
// with few segments per lane keep 512: the work-item loop costs them registers).
constexpr int batch_max_threads(int G, int SPL) { return SPL >= 12 ? 768 : (G <= 8 ? 768 : 1024); }
size_t batch_smem_bytes(const BatchShape &s, uint32_t bins);
int batch_chains_per_block(const BatchShape &s);
// Resident CTAs per SM of the shape's kernel (0 when it cannot launch).
int batch_blocks_per_sm(const BatchShape &s, int bins);
cudaError_t launch_batch(const BatchShape &s, const void *d_exps, const uint2 *d_items, uint32_t n_items,
                         uint32_t *d_counter, ChainOut *out, int bins, int grid, cudaStream_t st);

// Batched adjoint replay: the experiments packed as for launch_batch (their table being the
// linear one, staged in shared memory by every shape), plus per experiment its derivative
// tables (device, launch_deriv_tables layout) and the log10 reference the path weights are
// scaled by (the experiment's forward log10 sum without absorption).
// grad[(out_offset + chain) * 6 + k]: the chain's sums of 10^(w - ref) d log10 w / d (mu_s,
// eps, receiver x, y, z) and of 10^(w - ref).
struct BatchAdjHost {
    const float4 *dtab;
    float ref_log10;
};
size_t batch_adj_bytes();
void batch_pack_adjoint(const BatchAdjHost *in, uint32_t n, void *dst);
int batch_adjoint_blocks_per_sm(const BatchShape &s, int bins);
cudaError_t launch_batch_adjoint(const BatchShape &s, const void *d_exps, const void *d_adj, const uint2 *d_items,
                                 uint32_t n_items, uint32_t *d_counter, double *grad, int bins, int grid,
                                 cudaStream_t st);
// Per range ranges[x] = (first chain, count): the sums over its chains of the 6 gradient entries.
cudaError_t launch_grad_reduce_segments(const double *grad_chains, const uint2 *ranges, uint32_t n, double *out,
                                        cudaStream_t st);
// Derivative tables d/d(mu_s), d/d(eps) (double, n_tables x bins) in the form the adjoint reads:
// per bin float4 (dmu_i, dmu_{i+1} - dmu_i, deps_i, deps_{i+1} - deps_i).
cudaError_t launch_deriv_tables(const double *dmu, const double *deps, uint32_t bins, uint32_t n_tables, float4 *out,
                                cudaStream_t st);

// Path-weight histogram (chain_plain.cu): w[n] log10 path weights (NaN: not counted), counted as
// 10^(w + log10_norm) into nbins <= 12288 equal buckets over [lo, hi] (outside: the end buckets).
cudaError_t launch_weight_histogram(const double *w, uint64_t n, double log10_norm, double lo, double hi, uint32_t nbins,
                                    unsigned long long *counts, cudaStream_t st);

// ----------------------------------------------------------- reduction (chain_plain.cu)
cudaError_t launch_reduce(const ChainOut *chains, uint32_t n, ReduceOut *out, cudaStream_t st);
// One reduction per range: ranges[x] = (first chain, count) -> out[x].
cudaError_t launch_reduce_segments(const ChainOut *chains, const uint2 *ranges, uint32_t n_segments, ReduceOut *out,
                                   cudaStream_t st);

// ------------------------------------------------------------- weighting of given paths
cudaError_t launch_weigh_plain(const float *pos, uint64_t n_paths, uint32_t n_segments, float inv_ds,
                               const float *lut, LutMetaF m, double absorption_factor,
                               double *log10w, uint8_t *valid, int32_t *bins, cudaStream_t st);
cudaError_t launch_weigh_comp(const float *pos, uint64_t n_paths, uint32_t n_segments, float inv_ds,
                              const float2 *fixtab, const float2 *lintab, int exact_blend, LutMetaF m,
                              double log10_absorption, double *log10w, uint8_t *valid, int32_t *bins,
                              cudaStream_t st, LogFixed lf = LogFixed{0.0, 0.0});

// --------------------------------------------- independent-sample paths (msegment.cu)
// n_paths fresh random curves (the reference's recursive bootstrapper, Philox draws keyed by
// seed and path0 + i) into pos[n_paths][N+1][3]; N - 2 must be resolvable (4, 6, 8, 12, ...).
cudaError_t launch_msegment_paths(uint32_t n_segments, float ds, const float p0[3], const float p1[3],
                                  const float pm1[3], const float pm[3], uint64_t seed, uint32_t experiment,
                                  uint64_t path0, uint64_t n_paths, float *pos, cudaStream_t st);
// Per-path weights as one ChainOut each (invalid paths: -inf, failed = 1).
cudaError_t launch_pack_paths(const double *w, const uint8_t *valid, uint64_t n, ChainOut *out, cudaStream_t st);

// ------------------------------------------------------------ normaliser (norm.cu)
uint32_t norm_partial_blocks();
cudaError_t launch_norm_k56(float z, float ds, double *partials, double *out, cudaStream_t st);

}  // namespace twisty
