/*
 * twisty_oracle.h -- CPU oracle for the path-integral Monte Carlo hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference legs may load this library, and only as the
 * checker; the product (twisty_b200/) never links or calls it.
 *
 * A plain-C restatement of the reference's algorithm, function by function, with the
 * reference file:line each one follows. Two arithmetic flavours:
 *   *_f32  the reference's own FP32/FP64 mix, operation for operation (IEEE, no FMA
 *          contraction), so the CUDA drop-in path can be compared bit for bit;
 *   *_f64  the FP64 twin: the same algorithm in double everywhere (LUT built in double,
 *          double pi), the yardstick every result states its error against.
 * The Markov chains are driven by counter-based Philox-4x32-10 proposals whose mapping
 * to (k, left, angle) is shared with the CUDA kernels (tor_draw_step), so a chain here
 * and on the GPU see the same proposal sequence.
 *
 * Pinned against the reference itself (compiled from its sources into oracle/_ref by
 * oracle/Makefile) through the golden vectors under tests/golden/.
 */
#ifndef TWISTY_ORACLE_H
#define TWISTY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* WeightingParameters (Twisty/PathWeightUtils.h:35-48). */
typedef struct {
    float mu;          /* config "mu": the regulariser (arguments swapped at PathWeightUtils.cpp:401) */
    float eps;         /* config "eps": the Gaussian phase-function parameter */
    float scatter;     /* mu_s */
    float absorption;  /* mu_a */
    float min_bound;   /* 0 */
    float max_bound;   /* 10/eps (ExperimentRunner.cpp:169-171) */
    float bias;        /* 1 */
    uint32_t num_steps_int;
    uint32_t num_curvature_steps;
} tor_wparams;

typedef struct {
    float min_k, max_k, step, min_w, max_w, ds;
    uint32_t bins, pad;
} tor_lut_meta;

typedef struct {
    double min_k, max_k, step, min_w, max_w, ds;
    uint32_t bins, pad;
} tor_lut_meta64;

/* Base-10 scaled running sum (Twisty/CombinedWeightUtils.h:28-33). */
typedef struct {
    double max_log10, total, offset;
    uint32_t n, pad;
} tor_cw;

/* ---- RNG and proposal mapping (shared definition with the CUDA kernels) ---- */
void tor_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void tor_draw_step(uint64_t seed, uint32_t experiment, uint32_t chain, uint32_t step,
                   uint32_t n_segments, uint32_t k_max, float max_angle,
                   uint32_t *k, uint32_t *left, float *angle);
void tor_sincos_half(float angle, float *s, float *c);

/* ---- LUT construction ---- */
void tor_wparams_default(tor_wparams *wp, float mu, float eps, float scatter, float absorption,
                         uint32_t num_steps_int, uint32_t bins);
int tor_lut_build_f32(const tor_wparams *wp, float ds, float *lut, tor_lut_meta *meta, int n_threads);
int tor_lut_build_f64(const tor_wparams *wp, double ds, double *lut, tor_lut_meta64 *meta, int n_threads);
float tor_gaussian_phase_f32(float p, float m);
double tor_integrand_rt(double p, double kds, double bds, double eps, double mu);

/* ---- curve operations and weighting ---- */
void tor_rotate_by_quat_f32(const float q[4], float v[3]);
void tor_tangents_f32(const float *pos, uint32_t n_segments, float *tan);
void tor_curvatures_f32(const float *tan, uint32_t n_segments, float arclength, float *curv);
int tor_weight_curvatures_f32(const float *curv, uint32_t n, const float *lut, const tor_lut_meta *m,
                              float absorption, double *log10w, int32_t *bins, uint32_t *n_clamped);
int tor_weigh_paths_f32(const float *pos, uint64_t n_paths, uint32_t n_segments, float arclength,
                        const float *lut, const tor_lut_meta *m, float absorption,
                        double *log10w, uint8_t *valid, int32_t *bins, float *curv);
int tor_weigh_paths_f64(const double *pos, uint64_t n_paths, uint32_t n_segments, double arclength,
                        const double *lut, const tor_lut_meta64 *m, double absorption,
                        double *log10w, uint8_t *valid, int32_t *bins, double *curv);

/* ---- per-experiment accumulation ---- */
void tor_cw_reset(tor_cw *c);
void tor_cw_add(tor_cw *c, double value_log10);
void tor_cw_combine(const tor_cw *a, const tor_cw *b, tor_cw *out);
double tor_cw_extract_log10(const tor_cw *c);
double tor_log10_sum(const double *log10v, uint64_t n);

/* ---- normaliser ---- */
double tor_norm_log10(int n_segments, float ds, const float bc[12]);

/* ---- Markov chains ----
 * init_pos: (N+1)*3 floats. Each chain c (global id chain0 + c) runs burn_in unweighted
 * steps then `steps` weighted steps. Outputs (each nullable):
 *   path_log10[c*steps + s], path_valid[...]  per weighted path
 *   chain_log10[c]  log10 of the chain's sum of valid path weights (-inf if none)
 *   chain_valid[c]  number of valid paths
 *   final_pos[c*(N+1)*3 ...]  chain state after the last step
 */
int tor_run_chains_f32(const float *init_pos, uint32_t n_segments, float arclength,
                       const float *lut, const tor_lut_meta *m, float absorption,
                       uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                       uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                       double *path_log10, uint8_t *path_valid, double *chain_log10,
                       uint64_t *chain_valid, float *final_pos, int n_threads);
int tor_run_chains_f64(const float *init_pos, uint32_t n_segments, double arclength,
                       const double *lut, const tor_lut_meta64 *m, double absorption,
                       uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                       uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                       double *path_log10, uint8_t *path_valid, double *chain_log10,
                       uint64_t *chain_valid, double *final_pos, int n_threads);

/* The FP64 twin chains with the options of a gradient check:
 *   has_shift, eval_shift  weights evaluated with the receiver (points N-1 and N) moved by
 *                          eval_shift, the chain itself unchanged (finite differences of the
 *                          estimate with respect to the receiver, common random numbers);
 *   grad_chains            nullable, [n_chains][4]: per chain, the sum over its valid paths of
 *                          10^(w - ref_log10) d log10 w / d receiver (x, y, z) and of
 *                          10^(w - ref_log10) -- the pathwise receiver gradient in FP64, with
 *                          the table slope taken as the slope of the expected segment weight
 *                          (see dlog10_dkappa_f64). */
typedef struct {
    int has_shift;
    double eval_shift[3];
    double ref_log10;
    double *grad_chains;
} tor_chain_opts;

int tor_run_chains_f64_opts(const float *init_pos, uint32_t n_segments, double arclength,
                            const double *lut, const tor_lut_meta64 *m, double absorption,
                            uint64_t seed, uint32_t experiment, uint32_t chain0, uint32_t n_chains,
                            uint32_t steps, uint32_t burn_in, uint32_t k_max, float max_angle,
                            double *chain_log10, uint64_t *chain_valid, const tor_chain_opts *opts,
                            int n_threads);

#ifdef __cplusplus
}
#endif
#endif
