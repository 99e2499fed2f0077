/*
 * twisty_b200.h -- C ABI of the B200-native path-integral Monte Carlo runner.
 *
 * Drop-in for the reference's experiment-runner API (Twisty/ExperimentRunner.h:29-131)
 * and its two runners, FullExperimentRunnerOptimalPerturb (CPU,
 * Twisty/FullExperimentRunnerOptimalPerturb.h:26-74) and
 * FullExperimentRunnerOptimalPerturbOptimized_GPU
 * (Twisty/FullExperimentRunnerOptimalPerturbOptimized_GPU.h:36-47).
 *
 * All types are plain C structs; no exception, exit() or C++ type crosses this
 * boundary. Every call returns a twisty_status; twisty_last_error() gives the message.
 * Weights cross the ABI as log10 values (the reference's weights overflow double:
 * Twisty/ExperimentRunner.h:75 keeps them in a 100-digit decimal type).
 *
 * A context is not re-entrant: one thread at a time may call into a given context
 * (the reference's RunExperiment is not re-entrant either). Distinct contexts may be
 * used concurrently from distinct threads.
 */
#ifndef TWISTY_B200_H
#define TWISTY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TWISTY_B200_ABI_VERSION 2

/* Status codes. The reference reports failures by std::nullopt
 * (FullExperimentRunnerOptimalPerturbOptimized_GPU.cu:153-157), std::runtime_error
 * (PathGeneration.cpp:51-57,75-77,240-247), exit(1)
 * (FullExperimentRunnerOptimalPerturb.cpp:320-325) or printf-and-continue (.cu:50-56). */
typedef enum twisty_status {
    TWISTY_OK = 0,
    TWISTY_ERR_INVALID_ARGUMENT = 1,   /* null pointer, size out of range */
    TWISTY_ERR_INVALID_CONFIG = 2,     /* config text/params rejected (N < 4, odd numStepsInt, ...) */
    TWISTY_ERR_INFEASIBLE_GEOMETRY = 3,/* no polyline of N segments of length S/N joins the ends */
    TWISTY_ERR_LUT_INVALID = 4,        /* weight table has NaN/negative entries or < 2 bins */
    TWISTY_ERR_CUDA = 5,               /* a CUDA runtime call failed */
    TWISTY_ERR_DEVICE_TIMEOUT = 6,     /* a device-side wait ran past its deadline */
    TWISTY_ERR_IO = 7,                 /* export/config file could not be written/read */
    TWISTY_ERR_UNSUPPORTED = 8,        /* combination not implemented (e.g. perturbMethod != 0) */
    TWISTY_ERR_NO_DEVICE = 9,          /* no CUDA device, or the library was built without one */
    TWISTY_ERR_OUT_OF_MEMORY = 10
} twisty_status;

/* Arithmetic form of the Markov-chain kernel. */
typedef enum twisty_form {
    /* The reference GPU kernel's design (FullExperimentRunnerOptimalPerturbOptimized_GPU.cu:
     * 689-918): one chain per thread, chain state in global memory, FP32 IEEE
     * rotate/tangent/curvature, FP64 log10 per segment, CombinedWeightValues_C partials. */
    TWISTY_FORM_PLAIN_FP32 = 0,
    /* The B200 form: warp-cooperative chains held in shared memory as segment vectors,
     * FP32 tables staged in shared memory, Kahan-compensated FP32 log-weights, log-sum-exp
     * reductions rescaled by the running maximum, FP64 only across chains. */
    TWISTY_FORM_COMPENSATED = 1,
    /* FP64 everywhere (positions, rotation, table, weights): the error yardstick. */
    TWISTY_FORM_FP64 = 2
} twisty_form;

typedef enum twisty_lut_mode {
    TWISTY_LUT_FAITHFUL = 0, /* the reference's mixed precision: float phase function, double
                                Simpson, float table (PathWeightUtils.cpp:19-33,371-433) */
    TWISTY_LUT_FP64 = 1,     /* the same quadrature entirely in double */
    TWISTY_LUT_EXTERNAL = 2, /* the caller's table, set with twisty_set_lut */
    TWISTY_LUT_MULTI_DS = 3  /* the table of the multi-arclength set (twisty_multi_ds_tables)
                                whose ds is closest to the run's */
} twisty_lut_mode;

typedef struct twisty_vec3 {
    float x, y, z;
} twisty_vec3;

/* PerturbUtils::BoundaryConditions (Twisty/CurvePerturbUtils.h:62-68). */
typedef struct twisty_bc {
    twisty_vec3 start_pos;
    twisty_vec3 start_dir; /* unit */
    twisty_vec3 end_pos;
    twisty_vec3 end_dir;   /* unit */
    float arclength;
} twisty_bc;

/* ExperimentRunner::ExperimentParameters (Twisty/ExperimentRunner.h:42-68) with its
 * WeightingParameters (Twisty/PathWeightUtils.h:35-48), plus the B200 knobs.
 * Fill with twisty_params_init() first. */
typedef struct twisty_params {
    uint32_t struct_size;        /* sizeof(twisty_params) */
    uint64_t paths_to_generate;  /* pathsToGenerate: accepted paths in the estimate */
    uint64_t paths_to_skip;      /* pathsToSkip: unweighted burn-in steps of every chain */
    uint32_t num_segments;       /* numSegments (N >= 4) */
    uint32_t bootstrap_seed;     /* random.bootstrapSeed */
    uint32_t perturb_seed;       /* random.perturbSeed */
    int32_t weight_function;     /* weighting.weightFunction: 0 radiative transfer */
    int32_t perturb_method;      /* perturbMethod: 0 GeometricRandom (the only one the reference runs) */
    float mu;                    /* weighting.mu  (regulariser; see F5 swap in the docs) */
    float eps;                   /* weighting.eps (phase-function parameter) */
    float scatter;               /* weighting.scatter  (mu_s) */
    float absorption;            /* weighting.absorption (mu_a) */
    uint32_t num_steps_int;      /* weighting.numStepsInt (even) */
    uint32_t num_curvature_steps;/* weighting.numCurvatureSteps (table bins) */
    float min_bound;             /* 0 */
    float max_bound;             /* 10/eps */
    float bias;                  /* 1 */
    /* ---- B200 knobs ---- */
    int32_t form;                /* twisty_form */
    int32_t lut_mode;            /* twisty_lut_mode */
    uint32_t max_sub_chain;      /* k_max of the rotated sub-chain (reference: 25) */
    float max_angle;             /* rotation angle ~ U(-max_angle, max_angle) (reference: pi) */
    uint32_t num_chains;         /* independent Markov chains; 0 = form default */
    int32_t device;              /* CUDA device ordinal */
    uint32_t chain_offset;       /* first global chain id (shards one experiment over GPUs) */
    uint32_t experiment_id;      /* Philox stream id of this experiment */
    int32_t bootstrap_kind;      /* initial curve: 0 the reference's recursive bootstrapper
                                    (PathGeneration.cpp:47-414, the reference's curve for the
                                    same bootstrap_seed) where it resolves N (N-2 in {4, 6, 8,
                                    12, 16, 24, 32, 48, ...}), else the arc; 1 the reference's
                                    only; 2 the arc (any N >= 4) */
    twisty_vec3 eval_end_shift;  /* weights evaluated with the receiver moved by this vector,
                                    the chain itself unchanged (finite-difference checks) */
    /* compensated-form kernel shape; 0 = chosen from N. comp_group lanes per chain (1, 4, 8, 16,
       32) x comp_spl segments per lane (>= N in total), comp_warps warps per CTA. Shapes:
       1 x {8, 12, 16, 24}; 4 x {2, 3, 4, 5, 8, 9, 12, 16, 17, 20, 24, 28, 32}; 8 x {2, 4, 8, 9, 12,
       16, 17, 20, 24, 32}; 16 x {4, 8, 12, 16, 17, 20, 24, 28, 32}; 32 x {4, 8, 12, 16, 17, 20, 24,
       28, 32} (batched runs: all but 8 x 32, 1 x 16, 1 x 24 and 4 x 12). */
    uint32_t comp_group;
    uint32_t comp_spl;
    uint32_t comp_warps;
    /* compensated form, single runs: 0 recomputes every curvature of every weighted path (the
       reference's definition); R > 1 updates a path's weight incrementally from the two
       curvatures a rotation changes and recomputes it in full every R-th weighted step
       (an algorithmic shortcut, reported separately; fixed-point tables without clamping) */
    uint32_t incremental_resync;
    /* where the compensated form keeps the weight table (no reference counterpart): 0 = chosen
       from its size (shared memory when it fits beside a full CTA of chain state, or beside
       20 of the 24 warps of the 20- and 24-segment shapes, else read through L1), 1 = shared
       memory (fewer warps per CTA for large tables), 2 = through L1.
       Path export, the adjoint, receiver-shifted and incremental runs always stage it. */
    uint32_t comp_table_memory;
    /* error against FP64, measured (no reference counterpart): K > 0 replays the pass's first K
       chains (the same proposals) in the FP64 form after the pass and reports the relative
       difference of their summed weights in twisty_result.fp64_rel_error. The FP64 form runs a
       chain per thread, so the check costs about K / (all chains) of a pass of that form; 0 = off. */
    uint32_t fp64_check_chains;
} twisty_params;

/* ExperimentRunner::ExperimentResults (Twisty/ExperimentRunner.h:73-82). */
typedef struct twisty_result {
    double log10_weight;         /* log10 experimentWeight = log10(sum of path weights * normaliser) */
    double log10_normalizer;     /* log10 Norm(N, ds, bc) (PathWeightUtils.cpp:721-752) */
    double log10_mean_weight;    /* log10(experimentWeight / totalPathsGenerated) */
    double rel_std_error;        /* standard error of experimentWeight / experimentWeight,
                                    from the spread of the independent chains' sums */
    uint64_t total_paths;        /* totalPathsGenerated (valid, weighted paths) */
    uint64_t failed_paths;       /* numFailedPaths (NaN weights) */
    uint64_t clamped_curvatures; /* curvatures outside the table range, clamped */
    uint32_t num_chains;
    uint32_t steps_per_chain;
    double total_ms;             /* totalExperimentMs */
    double setup_ms;             /* setupExperimentMs: table, normaliser, initial curve */
    double perturb_ms;           /* perturbExperimentMs: the chain kernel, device time */
    double weighting_ms;         /* weightingExperimentMs: final reduction */
    /* Compensated form only (no reference counterpart): which table the pass weighed with,
       TWISTY_TABLE_FIXED_NARROW / _FIXED_WIDE (fixed-point log tables, 32- or 64-bit path
       totals) or TWISTY_TABLE_EXACT_BLEND (linear table, a log per segment); other forms
       report TWISTY_TABLE_NONE. steep_bins counts the fixed-point table's bins whose secant
       would err by more than 1e-7 per segment: paths crossing one are re-weighed through the
       linear table. */
    uint32_t table_form;
    uint32_t steep_bins;
    /* The result's error against FP64 (no reference counterpart). weight_error_bound: bound on
       |log10 w - log10 w_FP64| of every path's weight for the path's own curvatures and table,
       from the form's arithmetic -- fixed-point tables (N-1)(2^-s + secant error), exact-blend
       tables (N-1) 4e-7, the plain form's float blend (N-1) 2.6e-8, 0 for the FP64 form; it does
       not cover the FP32 trajectory's drift from the FP64 one, which fp64_rel_error measures:
       |W_K / W_K,FP64 - 1| over the first fp64_check_chains chains replayed in the FP64 form
       (NaN when the check is off). */
    double weight_error_bound;
    double fp64_rel_error;
    uint32_t fp64_check_chains;
    /* The compensated form's kernel shape that ran: lanes per chain << 8 | segments per lane
       (0x0110 = 1 x 16); 0 for the other forms. No reference counterpart. */
    uint32_t kernel_shape;
} twisty_result;

enum {
    TWISTY_TABLE_FIXED_NARROW = 0,
    TWISTY_TABLE_FIXED_WIDE = 1,
    TWISTY_TABLE_EXACT_BLEND = 2,
    TWISTY_TABLE_NONE = 3
};

/* Table metadata (BaseWeightLookupTable accessors, Twisty/PathWeightUtils.h:129-141). */
typedef struct twisty_lut_info {
    float min_curvature, max_curvature, curvature_step;
    float min_segment_weight, max_segment_weight, ds;
    uint32_t bins;
} twisty_lut_info;

/* One experiment of a batch (the receiver/pixel loops of the reference's drivers,
 * e.g. Experiments/BeamSpreadExperiment.cpp:240-269, NoisyCircleExperiment.cpp:259-361). */
typedef struct twisty_experiment {
    twisty_bc bc;
    uint32_t num_segments;
    float scatter;               /* per-experiment mu_s */
    float eps;                   /* per-experiment phase parameter (sigma^2) */
    uint64_t paths;              /* paths_to_generate of this experiment */
} twisty_experiment;

typedef struct twisty_ctx twisty_ctx;

/* ---------------------------------------------------------------- basics */
int twisty_abi_version(void);
const char *twisty_status_string(twisty_status s);
/* Reference defaults: ExperimentParameters/WeightingParameters member initialisers. */
void twisty_params_init(twisty_params *p);

/* ExperimentRunner::ParseExperimentParamsFromConfig (Twisty/ExperimentRunner.cpp:48-177)
 * plus the basicExperiment block read by Experiments/FullExperiment.cpp:162-191.
 * `text` is the reference's JSON config schema, or the same keys in YAML block syntax
 * (is_yaml != 0). bc may be NULL. */
twisty_status twisty_params_from_config(const char *text, int is_yaml, twisty_params *out, twisty_bc *bc);

/* --------------------------------------------------------------- context */
/* ExperimentRunner(ExperimentParameters&) ctor (Twisty/ExperimentRunner.cpp:180-192);
 * the params are copied. Selects and initialises the CUDA device. */
twisty_status twisty_create(const twisty_params *p, twisty_ctx **out);
void twisty_destroy(twisty_ctx *ctx);
const char *twisty_last_error(const twisty_ctx *ctx);
/* New parameters for the context's next runs; the next run builds its weight tables again
 * (as every RunExperiment of the reference builds its table). */
twisty_status twisty_update_params(twisty_ctx *ctx, const twisty_params *p);

/* ----------------------------------------------------------- experiments */
/* ExperimentRunner::RunExperiment (Twisty/ExperimentRunner.cpp:196-301) ->
 * RunnerSpecificRunExperiment (FullExperimentRunnerOptimalPerturb.cpp:48-435). Host in,
 * host out: builds the table, the normaliser and the initial curve, runs the chains,
 * reduces, and fills *res. */
twisty_status twisty_run(twisty_ctx *ctx, const twisty_bc *bc, twisty_result *res);

/* Split form of twisty_run for callers that keep inputs resident and time the device:
 * twisty_prepare does the setup (table, normaliser, curve, device state) once;
 * twisty_launch enqueues one full Monte Carlo pass on `stream` (a cudaStream_t, NULL for
 * the context's own stream) without synchronising; twisty_collect waits and reduces. */
twisty_status twisty_prepare(twisty_ctx *ctx, const twisty_bc *bc);
twisty_status twisty_launch(twisty_ctx *ctx, void *stream);
twisty_status twisty_collect(twisty_ctx *ctx, twisty_result *res);
/* Number of kernels twisty_launch enqueues (for launch accounting). */
uint32_t twisty_launch_kernel_count(const twisty_ctx *ctx);

/* Per-chain outcomes of the context's last pass (twisty_run, twisty_launch): log10 of each
 * chain's summed path weights (normaliser applied) and its count of valid paths; valid may be
 * NULL, n_chains must be the pass's chain count (twisty_result.num_chains). The reference's
 * runner keeps per-thread running sums for its convergence records
 * (FullExperimentRunnerOptimalPerturb.cpp:96-109,358-365); a chain here is a thread there. */
twisty_status twisty_chain_results(twisty_ctx *ctx, double *log10_sum, uint64_t *valid, uint32_t n_chains);

/* Histogram of the experiment's path weights, the reference's histogram.txt
 * (FullExperimentRunnerOptimalPerturb.cpp:26-37,394-422,562-575): every weighted path's linear
 * weight 10^(log10 w + log10 normaliser) counted into n_buckets equal buckets over
 * [min_weight, max_weight] (the reference: 500 over [4.69653e-16, 1.17517e-13], the range of
 * five-segment paths); weights below the range count in the first bucket, above it in the last.
 * Replays the chains of twisty_run with the same parameters (plain or compensated form), keeping
 * each weight: about the cost of one more pass. counts[n_buckets], n_buckets <= 12288. */
twisty_status twisty_weight_histogram(twisty_ctx *ctx, const twisty_bc *bc, double min_weight, double max_weight,
                                      uint32_t n_buckets, uint64_t *counts);

/* Many experiments (uneven N, S, mu_s, eps) in one persistent launch fed by a device
 * work queue; the pass is captured once as a CUDA graph and replayed `iterations` times
 * (results of the last replay). res has n entries. */
twisty_status twisty_run_batch(twisty_ctx *ctx, const twisty_experiment *ex, uint32_t n,
                               uint32_t iterations, twisty_result *res);

/* Independent-sample M-segment Monte Carlo: MSegmentPathGenerationMC
 * (Experiments/ExperimentBase.cpp:1246-1386). params.paths_to_generate fresh random curves from
 * the recursive bootstrapper (N-2 in {4, 6, 8, 12, 16, 24, 32, 48, ...}) between the fixed points
 * of bc, drawn on the device from Philox (seed perturb_seed, stream experiment_id, paths
 * numbered from chain_offset * paths_to_generate), weighed in the plain (reference FP32) or
 * compensated form. The estimate is the MEAN weight times the normaliser: res->log10_weight =
 * res->log10_mean_weight; rel_std_error from the spread of the independent paths. */
twisty_status twisty_run_msegment(twisty_ctx *ctx, const twisty_bc *bc, twisty_result *res);

/* ------------------------------------------------------------- weighting */
/* Weigh exported paths: UpdateTangentsFromPos + UpdateCurvaturesFromTangents_RadiativeTransfer
 * + WeightCurveViaCurvatureLog10_CudaSafe (CurvePerturbUtils.cpp:147-166,
 * PathWeighters.cpp:27-104) on pos[n_paths][N+1][3]. Uses the context's table for
 * ds = bc->arclength / N. Outputs log10 weights (without the normaliser), validity, and
 * optionally the left bin index of every curvature (bins[n_paths][N-1], may be NULL).
 * form selects the reference FP32 semantics (PLAIN_FP32) or the compensated path. */
twisty_status twisty_weight_paths(twisty_ctx *ctx, const twisty_bc *bc, const float *pos,
                                  uint64_t n_paths, int32_t form, double *log10w,
                                  uint8_t *valid, int32_t *bins);

/* WeightLookupTableIntegral(params, ds) + Initialize (PathWeightUtils.cpp:281-348), on
 * the device in FP64. lut may be NULL (info only). */
twisty_status twisty_build_lut(twisty_ctx *ctx, float ds, float *lut, twisty_lut_info *info);
/* Use the caller's table (e.g. one exported by the reference) for subsequent runs. */
twisty_status twisty_set_lut(twisty_ctx *ctx, const float *lut, const twisty_lut_info *info);

/* NormalizerStuff::Norm (PathWeightUtils.cpp:721-752) as log10; N = 5, 6 run their
 * 1e10-term quadrature on the device in FP64. */
twisty_status twisty_normalizer_log10(twisty_ctx *ctx, uint32_t n_segments, float ds,
                                      const twisty_bc *bc, double *out);

/* Initial curve (Curve::SetBoundaryConditions + PathGeneration::ResolveEvenNumberOfSegments,
 * Twisty/Curve.cpp:20-30, Twisty/PathGeneration.cpp:236-414) for any N >= 4:
 * pos[N+1][3]. Fails with TWISTY_ERR_INFEASIBLE_GEOMETRY when no curve exists. */
twisty_status twisty_bootstrap_curve(const twisty_params *p, const twisty_bc *bc, float *pos);
/* CalculateMinimumArclength (Twisty/PathGeneration.cpp:12-43). */
float twisty_min_arclength(const twisty_bc *bc, uint32_t n_segments);
/* Use pos[n_points][3] (n_points = N+1) as the initial curve of the context's next runs
 * instead of the bootstrapper; the reference replicates one initial curve into every
 * chain (FullExperimentRunnerOptimalPerturb.cpp:122-179). NULL reverts to the bootstrapper. */
twisty_status twisty_set_initial_curve(twisty_ctx *ctx, const float *pos, uint32_t n_points);

/* --------------------------------------------------------------- exports */
/* Path-batch export of GeometryRandom_ExportPaths / BeginPathBatchOutput
 * (FullExperimentRunnerOptimalPerturb.cpp:599-858, ExperimentRunner.cpp:303-396): runs the
 * experiment and writes, under dir/GeneratedCurves/, Paths_Binary.pbd (f32 [P][N+1][3]),
 * Log10PathWeights_Binary.bdt (f64 linear weights incl. normaliser, as the reference),
 * Paths_Metadata.pmd ("chain batch count" lines), BoundaryConditions.bcf (56 bytes) and
 * index.json, for the first max_paths accepted paths. Also returns them in memory when
 * pos/log10w are not NULL (pos[max_paths][N+1][3], log10w[max_paths], without the normaliser). */
twisty_status twisty_export_paths(twisty_ctx *ctx, const twisty_bc *bc, const char *dir,
                                  uint64_t max_paths, float *pos, double *log10w,
                                  uint64_t *n_written, twisty_result *res);

/* ---------------------------------------------------------------- adjoint */
/* Gradient of log10 experimentWeight with respect to (mu_s, sigma, receiver x, y, z),
 * sigma = sqrt(eps), by a hand-written adjoint pass that replays the chains of the
 * forward run in `fwd` (same params, same bc) and recomputes curvatures instead of storing
 * them. The receiver gradient moves the two fixed end points with the interior held
 * (pathwise estimator). grad has 5 entries. */
twisty_status twisty_adjoint(twisty_ctx *ctx, const twisty_bc *bc, const twisty_result *fwd,
                             double grad[5]);

/* The adjoint of a batch: the receiver/pixel loops of the reference's image drivers
 * (Experiments/BeamSpreadExperiment.cpp:240-269, NoisyCircleExperiment.cpp:259-361) call
 * RunExperiment per pixel; differentiating the image takes one forward pass of the batch
 * (twisty_run_batch, results in res[n]) and one persistent adjoint replay of every experiment's
 * chains (curvatures recomputed, derivative tables d/d(mu_s), d/d(eps) built in FP64 on the
 * device). grad[n][5]: d log10 W_e / d (mu_s, sigma, receiver x, y, z) of each experiment, for
 * its own mu_s, sigma = sqrt(eps) and receiver, as twisty_adjoint defines them. total (nullable):
 * {log10 sum_e W_e, d / d mu_s, d / d sigma} of the batch's total -- the image's total
 * log-energy -- for a mu_s and sigma shared by all experiments (each experiment's derivative
 * weighted by its share of the total). timing_ms (nullable): device time of the derivative
 * tables and of the replay. Needs lut_mode FP64 or MULTI_DS. */
twisty_status twisty_adjoint_batch(twisty_ctx *ctx, const twisty_experiment *ex, uint32_t n, twisty_result *res,
                                   double *grad, double total[3], double timing_ms[2]);

/* CachedMultiArclengthWeightLookupTable (Twisty/PathWeightUtils.cpp:123-278): n_ds tables for
 * ds_i = min_ds + i (max_ds - min_ds) / (n_ds - 1) (float arithmetic, :170-173) with the
 * context's weighting parameters, built in one batched FP64 quadrature on the device, or read
 * from cache_path when that file holds the same set (written there otherwise; NULL: no file).
 * Runs and batches with lut_mode TWISTY_LUT_MULTI_DS then take the table whose ds is closest to
 * their own (GetWeightLookupTable, :230-243: the first of equally close ones), as the
 * reference's image drivers do; their weighting parameters must be the set's. */
twisty_status twisty_multi_ds_tables(twisty_ctx *ctx, float min_ds, float max_ds, uint32_t n_ds, const char *cache_path);

/* ---------------------------------------------------------------- autotuner */
/* No counterpart in the reference. Times every supported compensated-form kernel shape
 * (lanes per chain x segments per lane x warps per CTA) for the context's N and table on a
 * short pass of trial_paths paths (0: 2^22) with the context's other parameters, records
 * the fastest in the process-wide tuning cache and returns it. Every later pass (twisty_run,
 * twisty_run_batch) on a device of the same name, with the same N and table size and the
 * shape knobs (comp_group, comp_spl, comp_warps) left at zero, uses the recorded shape. */
typedef struct twisty_tuning {
    uint32_t num_segments;
    uint32_t bins;
    uint32_t group;              /* lanes per chain */
    uint32_t spl;                /* segments per lane */
    uint32_t warps;              /* warps per CTA */
    double path_segments_per_s;  /* measured rate of that shape */
} twisty_tuning;

twisty_status twisty_autotune(twisty_ctx *ctx, const twisty_bc *bc, uint64_t trial_paths, twisty_tuning *best);
/* The tuning cache as JSON: {"entries": [{"device", "n", "bins", "group", "spl", "warps",
 * "path_segments_per_s"}, ...]}. Loading merges into the cache (an entry replaces one with
 * the same device, n and bins); a malformed file or unsupported shape is rejected whole. */
twisty_status twisty_tuning_cache_save(const char *path);
twisty_status twisty_tuning_cache_load(const char *path);

/* No counterpart in the reference. The kernel shape and table placement that a compensated
 * forward pass of num_segments segments with a bins-bin weight table takes when the shape
 * knobs are zero, comp_table_memory is 0 and the tuning cache has no entry for them
 * (comp_default_tuning and the placement rule of twisty_run). Host-only: needs no device.
 * For N = 13..24 the shape also depends on the pass: a pass takes the one-lane 1 x 16 (N <= 16)
 * or 1 x 24 only when its paths_to_generate reaches 60000 or 130000 times its paths_to_skip
 * (shorter passes take 4 x 4, 4 x 5 or 4 x 8), and 1 x 16 runs 24 warps instead of 16 from
 * 210000 times; this reports the longest pass's shape.
 * TWISTY_ERR_INVALID_ARGUMENT for a null out, N < 4 or bins < 2; TWISTY_ERR_UNSUPPORTED
 * when no shape covers N (N > 1024). */
typedef struct twisty_shape {
    uint32_t group;         /* lanes per chain */
    uint32_t spl;           /* segments per lane */
    uint32_t warps;         /* warps per CTA */
    uint32_t table_in_l1;   /* 1: the table is gathered through L1; 0: staged in shared memory */
    uint32_t smem_bytes;    /* dynamic shared memory per CTA */
    uint32_t batched;       /* 1: twisty_run_batch has a kernel of this shape (0 for the one-lane
                               1 x 16 and 1 x 24 of N = 13..24 and for 4 x 12 of N = 37..48:
                               batched runs of such N take 4 x 4, 4 x 5, 4 x 8 or 4 x 16) */
} twisty_shape;
twisty_status twisty_default_shape(uint32_t num_segments, uint32_t bins, twisty_shape *out);

/* No counterpart in the reference. The FP32 issue rate of the device (lane-level FMA
 * instructions per second, independent FMA chains in every lane of every SM), measured in
 * about 100 ms: the denominator of the chain kernels' roofline. */
twisty_status twisty_measure_fp32_peak(int device, double *lane_instr_per_s);

/* ------------------------------------------------------- allocation-free pass */
/* No counterpart in the reference. For callers that cannot allocate device memory when
 * they run a pass: an application whose own caching allocator holds nearly all of the
 * GPU (a library cudaMalloc behind its back can fail or upset its accounting), or a
 * pipeline that must not stall (cudaMalloc and cudaFree may synchronize the device).
 * twisty_run_noalloc runs one compensated-form Monte Carlo pass over the caller's device
 * inputs and writes a twisty_noalloc_result to the caller's device memory; it calls no
 * cudaMalloc, cudaFree or other allocating routine. Its per-chain scratch is a fixed array
 * compiled into the library (TWISTY_NOALLOC_MAX_CHAINS chains, 24 bytes each: 384 KiB held
 * on every GPU that loads the library, until the process exits); more chains are rejected
 * with TWISTY_ERR_INVALID_ARGUMENT.
 *
 * It runs on the calling thread's current device, enqueued on `stream` (NULL: the legacy
 * default stream). The first call on each device looks up that device's address of the
 * scratch array; make that first call before any stream capture on the device. Every
 * call writes each scratch entry it later reads, so nothing carries over between calls,
 * but all calls share the one array: calls that overlap on the GPU (concurrent streams,
 * threads) race on it and must be ordered by the caller. The looked-up address lives as long
 * as the device's context: do not call this entry point again after cudaDeviceReset in the
 * same process.
 *
 * The kernel shape and table placement are twisty_run's defaults for N, bins and the pass
 * (twisty_default_shape): the table is staged in shared memory when it fits beside the
 * chain state, else gathered through L1. bins is at most TWISTY_NOALLOC_MAX_BINS. */
#define TWISTY_NOALLOC_MAX_CHAINS 16384u
#define TWISTY_NOALLOC_MAX_BINS (1u << 24)

typedef struct twisty_noalloc_args {
    const void *table;           /* device float2[bins]: (L_i, L_{i+1} - L_i); last (L_{bins-1}, 0) */
    uint32_t bins;
    float min_curvature, max_curvature, curvature_step;
    const float *init_segments;  /* device float[3 * N]: x_{i+1} - x_i of the initial curve */
    uint32_t num_segments;       /* 4 <= N <= 1024 */
    float arclength;
    float absorption;            /* mu_a */
    uint64_t seed;
    uint32_t experiment_id;
    uint32_t chain_offset;
    uint32_t num_chains;         /* 1 .. TWISTY_NOALLOC_MAX_CHAINS */
    uint64_t paths;              /* weighted paths of the pass */
    uint32_t burn_in;            /* unweighted steps per chain */
    uint32_t max_sub_chain;      /* 2 .. 64 */
    float max_angle;             /* [0, pi] */
    void *result;                /* device twisty_noalloc_result */
} twisty_noalloc_args;

typedef struct twisty_noalloc_result {
    double log10_weight;         /* log10 of the summed path weights (normaliser not applied) */
    double rel_std_error;
    double max_chain_log10;
    uint64_t valid_paths, failed_paths, clamped_curvatures;
} twisty_noalloc_result;

twisty_status twisty_run_noalloc(const twisty_noalloc_args *args, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TWISTY_B200_H */
