// runtime.cu -- implementation of the C ABI in include/twisty_b200.h.
//
// Owns the device state of one context: the weight tables for the current ds (cached by
// their parameters), the initial curve, the per-chain state and outputs, and the events
// that time each phase. Host code only; the kernels live in lut.cu, chain_*.cu, norm.cu.
// No exception leaves an entry point: every body runs under guard().
#include "kernels.h"
#include "host_util.h"
#include "../../include/twisty_b200.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <algorithm>
#include <functional>
#include <limits>
#include <mutex>
#include <new>
#include <sstream>
#include <thread>
#include <atomic>
#include <string>
#include <vector>

using namespace twisty;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n)
    {
        if (n <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n ? n : 16;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

struct Failure {
    twisty_status s;
    std::string msg;
};

[[noreturn]] void fail(twisty_status s, const std::string &m) { throw Failure{s, m}; }

void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(e == cudaErrorMemoryAllocation ? TWISTY_ERR_OUT_OF_MEMORY : TWISTY_ERR_CUDA,
             std::string(what) + ": " + cudaGetErrorString(e));
    }
}

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t seed_of(uint32_t s)
{
    // ProcessRandomSeed (Twisty/ExperimentRunner.cpp:40-46): seed 0 means the wall clock.
    return s ? (uint64_t)s : (uint64_t)time(nullptr);
}

}  // namespace

// Device buffers of batched runs, kept by the context so that repeated batches of the same
// size allocate nothing (DevBuf::ensure only grows). The last row serves the batched adjoint.
struct BatchBufs {
    DevBuf specs, lut64, lut32, fix, lin, steps, nsegs, lf, ok, init_seg, exps, items, counters, chain_out, ranges, red;
    DevBuf dtab, d64mu, d64eps, d64scratch, adj_exps, adj_aux, adj_items, adj_counters, grad, grad_sum;
    void release()
    {
        DevBuf *all[] = {&specs, &lut64, &lut32, &fix, &lin, &steps, &nsegs, &lf, &ok, &init_seg, &exps, &items,
                         &counters, &chain_out, &ranges, &red, &dtab, &d64mu, &d64eps, &d64scratch,
                         &adj_exps, &adj_aux, &adj_items, &adj_counters, &grad, &grad_sum};
        for (DevBuf *b : all) b->release();
    }
};

// Outputs of the batched adjoint (twisty_adjoint_batch); every pointer nullable but grad.
struct BatchAdjointOut {
    double *grad;     // [n][5]
    double *total;    // [3]
    double *timing;   // [2]
};

// Streams, events and the graph of one batched pass, kept by the context: a batch whose buckets,
// grids and device buffers are those of the previous call replays the same graph (the
// experiments' tables, curves and work items are uploaded afresh; the graph reads them from the
// same buffers), so that a loop over the same grid (new mu_s or sigma per iteration, say) pays
// no capture and no instantiation.
struct BatchGraph {
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key;   // what the graph was captured for
    void release()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (cudaStream_t st : streams) cudaStreamDestroy(st);
        exec = nullptr;
        graph = nullptr;
        events.clear();
        streams.clear();
        key.clear();
    }
};

struct twisty_ctx {
    twisty_params p{};
    int device = 0;
    int sm_count = 148;
    std::string device_name;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::string err;

    // tables for the current key
    bool lut_ready = false;
    uint64_t lut_key[4] = {0, 0, 0, 0};
    DevBuf lut64, lut32, fixtab, lintab, dmus, deps, lutaux;
    LutMetaF meta{};
    double min_w = 0, max_w = 0, secant_err = 0;
    int exact_blend = 0;
    LogFixed lf{0.0, 0.0, 0, 0};   // fixed-point form of fixtab; inv_scale 0 when exact_blend
    std::vector<float> ext_lut;
    twisty_lut_info ext_info{};
    // multi-arclength table set (twisty_multi_ds_tables)
    struct MultiDs {
        bool ready = false;
        uint32_t gen = 0;          // bumped on every rebuild: part of the table cache key
        uint32_t n = 0, bins = 0;
        float min_ds = 0, max_ds = 0;
        float wp[9] = {};          // the weighting parameters the set was built for
        std::vector<float> ds;     // per table
        std::vector<LutMetaF> meta;
        std::vector<double> min_w, max_w;
        std::vector<float> host;   // [n][bins]
        DevBuf dev;                // [n][bins] float
    } multi;

    // the prepared experiment
    bool prepared = false;
    twisty_bc bc{};
    ChainSpec spec{};
    CompTuning tuning{};
    double log10_norm = 0.0;
    double setup_ms = 0.0;
    double prepare_start = 0.0;
    std::vector<float> user_curve;
    std::vector<float> init_pos_host;
    DevBuf init_pos, init_seg, state, chain_out, partials, reduce_out, norm_scratch;
    DevBuf check_state, check_out;   // the FP64 replay of the first chains (fp64_check_chains)
    uint32_t check_chains = 0;
    double check_meta[3] = {0.0, 0.0, 0.0};   // min_k, max_k, step of the FP64 replay's table
    uint32_t kernels_per_launch = 0;
    bool launched = false;
    BatchBufs batch;
    BatchGraph batch_graph;
};

namespace {

twisty_status guard(twisty_ctx *ctx, const std::function<void()> &f);

void validate(const twisty_params &p)
{
    if (p.struct_size != sizeof(twisty_params)) fail(TWISTY_ERR_INVALID_ARGUMENT, "twisty_params.struct_size mismatch (call twisty_params_init)");
    if (p.num_segments < 4) fail(TWISTY_ERR_INVALID_CONFIG, "numSegments must be at least 4");
    if (p.num_segments > 1024 && p.form == TWISTY_FORM_COMPENSATED) fail(TWISTY_ERR_INVALID_CONFIG, "the compensated form supports numSegments <= 1024");
    if (p.num_curvature_steps < 2) fail(TWISTY_ERR_INVALID_CONFIG, "numCurvatureSteps must be at least 2");
    if (p.lut_mode != TWISTY_LUT_EXTERNAL && (p.num_steps_int < 4 || (p.num_steps_int & 1u)))
        fail(TWISTY_ERR_INVALID_CONFIG, "numStepsInt must be even and at least 4");
    if (p.lut_mode != TWISTY_LUT_EXTERNAL && !(p.eps > 0.0f)) fail(TWISTY_ERR_INVALID_CONFIG, "weighting.eps must be positive");
    if (p.form < 0 || p.form > 2) fail(TWISTY_ERR_INVALID_CONFIG, "unknown form");
    if (p.lut_mode < 0 || p.lut_mode > 3) fail(TWISTY_ERR_INVALID_CONFIG, "unknown lut_mode");
    if (p.perturb_method != 0) fail(TWISTY_ERR_UNSUPPORTED, "only perturbMethod 0 (GeometricRandom) runs; the reference exits on the others");
    if (p.weight_function != 0) fail(TWISTY_ERR_UNSUPPORTED, "only weightFunction 0 (radiative transfer) is implemented on the device");
    if (p.max_sub_chain < 2) fail(TWISTY_ERR_INVALID_CONFIG, "max_sub_chain must be at least 2");
    if (!(p.max_angle >= 0.0f) || p.max_angle > 3.1415927f) fail(TWISTY_ERR_INVALID_CONFIG, "max_angle must be in [0, pi]");
    if (p.bootstrap_kind < 0 || p.bootstrap_kind > 2) fail(TWISTY_ERR_INVALID_CONFIG, "bootstrap_kind must be 0, 1 or 2");
    if (p.comp_table_memory > 2) fail(TWISTY_ERR_INVALID_CONFIG, "comp_table_memory must be 0, 1 or 2");
}

void validate_bc(const twisty_bc *bc)
{
    if (!bc) fail(TWISTY_ERR_INVALID_ARGUMENT, "bc is NULL");
    if (!(bc->arclength > 0.0f) || !std::isfinite(bc->arclength)) fail(TWISTY_ERR_INVALID_CONFIG, "arclength must be positive");
    auto unit = [](const twisty_vec3 &v) {
        const double l = std::sqrt((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        return std::fabs(l - 1.0) < 1e-3;
    };
    if (!unit(bc->start_dir) || !unit(bc->end_dir)) fail(TWISTY_ERR_INVALID_CONFIG, "start_dir and end_dir must be unit vectors");
}

void set_device(twisty_ctx *ctx) { ck(cudaSetDevice(ctx->device), "cudaSetDevice"); }

// ------------------------------------------------------------ tuning cache
// Compensated-form kernel shapes measured by twisty_autotune (or loaded from a cache file),
// keyed by device name, N and table size; consulted whenever the shape knobs are zero.
struct TuneEntry {
    std::string device;
    uint32_t n, bins, group, spl, warps;
    double rate;
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune;

void tune_record(const TuneEntry &e)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (TuneEntry &x : g_tune)
        if (x.device == e.device && x.n == e.n && x.bins == e.bins) {
            x = e;
            return;
        }
    g_tune.push_back(e);
}

bool tune_lookup(const std::string &device, uint32_t n, uint32_t bins, CompTuning &t)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneEntry &x : g_tune)
        if (x.device == device && x.n == n && x.bins == bins) {
            CompTuning c = t;
            c.group = (int)x.group;
            c.spl = (int)x.spl;
            c.warps_per_block = (int)x.warps;
            if (!comp_tuning_supported(c, n, 2)) return false;
            t = c;
            return true;
        }
    return false;
}

// ------------------------------------------------------------------ tables
void weighting_fingerprint(const twisty_params &p, float wp[9])
{
    wp[0] = p.mu;
    wp[1] = p.eps;
    wp[2] = p.scatter;
    wp[3] = p.absorption;
    wp[4] = (float)p.num_steps_int;
    wp[5] = (float)p.num_curvature_steps;
    wp[6] = p.min_bound;
    wp[7] = p.max_bound;
    wp[8] = p.bias;
}

// GetWeightLookupTable (Twisty/PathWeightUtils.cpp:230-243): the first table with the smallest
// |ds_i - ds| (float).
uint32_t multi_closest(const twisty_ctx *ctx, float ds)
{
    float best = std::numeric_limits<float>::max();
    uint32_t arg = 0;
    for (uint32_t i = 0; i < ctx->multi.n; ++i) {
        const float d = std::abs(ctx->multi.ds[i] - ds);
        if (d < best) {
            best = d;
            arg = i;
        }
    }
    return arg;
}

void check_multi(const twisty_ctx *ctx, const twisty_params &p)
{
    if (!ctx->multi.ready) fail(TWISTY_ERR_LUT_INVALID, "lut_mode MULTI_DS needs twisty_multi_ds_tables first");
    float wp[9];
    weighting_fingerprint(p, wp);
    if (std::memcmp(wp, ctx->multi.wp, sizeof(wp)) != 0)
        fail(TWISTY_ERR_LUT_INVALID, "the multi-ds tables were built for other weighting parameters");
}

void build_tables(twisty_ctx *ctx, float ds, bool derivatives)
{
    const twisty_params &p = ctx->p;
    const uint32_t bins = p.num_curvature_steps;
    uint64_t key[4];
    uint32_t dsb;
    std::memcpy(&dsb, &ds, 4);
    uint32_t f[6];
    std::memcpy(&f[0], &p.mu, 4);
    std::memcpy(&f[1], &p.eps, 4);
    std::memcpy(&f[2], &p.scatter, 4);
    std::memcpy(&f[3], &p.bias, 4);
    std::memcpy(&f[4], &p.max_bound, 4);
    std::memcpy(&f[5], &p.min_bound, 4);
    key[0] = ((uint64_t)dsb << 32) | ((uint64_t)(p.num_segments & 0xFFFFFFu) << 8) | (uint64_t)(uint32_t)(p.lut_mode & 0xFF);
    key[1] = ((uint64_t)f[0] << 32) | f[1];
    key[2] = ((uint64_t)f[2] << 32) | f[3];
    key[3] = ((uint64_t)f[4] << 32) ^ ((uint64_t)f[5]) ^ ((uint64_t)bins << 8) ^ ((uint64_t)p.num_steps_int << 40) ^
             (derivatives ? 1ull : 0ull) ^ (p.lut_mode == TWISTY_LUT_MULTI_DS ? ((uint64_t)ctx->multi.gen << 1) : 0ull);
    if (ctx->lut_ready && std::memcmp(key, ctx->lut_key, sizeof(key)) == 0) return;
    ctx->lut_ready = false;
    cudaStream_t st = ctx->stream;
    ck(ctx->lut32.ensure(sizeof(float) * bins), "alloc table");
    ck(ctx->fixtab.ensure(sizeof(float2) * bins), "alloc fixed-point table");
    ck(ctx->lintab.ensure(sizeof(float2) * bins), "alloc linear table");
    ck(ctx->lutaux.ensure(sizeof(double) * 4), "alloc table scratch");
    std::vector<float> host32(bins);
    if (p.lut_mode == TWISTY_LUT_MULTI_DS) {
        if (derivatives) fail(TWISTY_ERR_UNSUPPORTED, "derivative tables need lut_mode FP64");
        check_multi(ctx, p);
        const uint32_t i = multi_closest(ctx, ds);
        std::memcpy(host32.data(), ctx->multi.host.data() + (size_t)i * bins, sizeof(float) * bins);
        ctx->meta = ctx->multi.meta[i];
        ctx->min_w = ctx->multi.min_w[i];
        ctx->max_w = ctx->multi.max_w[i];
        ck(ctx->lut64.ensure(sizeof(double) * bins), "alloc table");
        std::vector<double> h64(host32.begin(), host32.end());
        ck(cudaMemcpyAsync(ctx->lut32.p, host32.data(), sizeof(float) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(cudaMemcpyAsync(ctx->lut64.p, h64.data(), sizeof(double) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(cudaStreamSynchronize(st), "sync");
    } else if (p.lut_mode == TWISTY_LUT_EXTERNAL) {
        if (ctx->ext_lut.size() != bins) fail(TWISTY_ERR_LUT_INVALID, "no external table of numCurvatureSteps entries was set (twisty_set_lut)");
        host32 = ctx->ext_lut;
        ctx->meta = LutMetaF{ctx->ext_info.min_curvature, ctx->ext_info.max_curvature, ctx->ext_info.curvature_step, (int32_t)bins};
        ctx->min_w = ctx->ext_info.min_segment_weight;
        ctx->max_w = ctx->ext_info.max_segment_weight;
        ck(cudaMemcpyAsync(ctx->lut32.p, host32.data(), sizeof(float) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(ctx->lut64.ensure(sizeof(double) * bins), "alloc table");
        std::vector<double> h64(host32.begin(), host32.end());
        ck(cudaMemcpyAsync(ctx->lut64.p, h64.data(), sizeof(double) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(cudaStreamSynchronize(st), "sync");
    } else if (p.lut_mode == TWISTY_LUT_FAITHFUL) {
        if (derivatives) fail(TWISTY_ERR_UNSUPPORTED, "derivative tables need lut_mode FP64");
        float mm[2];
        if (!lut_faithful_host(p.mu, p.eps, p.scatter, p.min_bound, p.max_bound, p.bias, p.num_steps_int, bins, ds,
                               host32.data(), mm))
            fail(TWISTY_ERR_INVALID_CONFIG, "invalid table parameters");
        const float max_k = (float)((2.0 / (double)ds) * (double)1.01f);
        ctx->meta = LutMetaF{0.0f, max_k, (max_k - 0.0f) / (float)(bins - 1), (int32_t)bins};
        ctx->min_w = mm[0];
        ctx->max_w = mm[1];
        ck(ctx->lut64.ensure(sizeof(double) * bins), "alloc table");
        std::vector<double> h64(host32.begin(), host32.end());
        ck(cudaMemcpyAsync(ctx->lut32.p, host32.data(), sizeof(float) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(cudaMemcpyAsync(ctx->lut64.p, h64.data(), sizeof(double) * bins, cudaMemcpyHostToDevice, st), "upload table");
        ck(cudaStreamSynchronize(st), "sync");
    } else {
        // WeightLookupTableIntegral ctor (PathWeightUtils.cpp:281-289), float grid
        const float min_k = 0.0f;
        const float max_k = (float)((2.0 / (double)ds) * (double)1.01f);
        const float step = (max_k - min_k) / (float)(bins - 1);
        LutBuildSpec s{};
        s.mu = p.mu;
        s.eps = p.eps;
        s.scatter = p.scatter;
        s.min_bound = p.min_bound;
        s.max_bound = p.max_bound;
        s.bias = p.bias;
        s.num_steps_int = p.num_steps_int;
        s.bins = bins;
        s.ds = ds;
        s.min_k = min_k;
        s.step = step;
        s.step64 = ((2.0 / (double)ds) * 1.01) / (double)(bins - 1);
        s.faithful = 0;
        s.derivatives = derivatives ? 1 : 0;
        ck(ctx->lut64.ensure(sizeof(double) * bins), "alloc table");
        if (derivatives) {
            ck(ctx->dmus.ensure(sizeof(double) * bins), "alloc derivative table");
            ck(ctx->deps.ensure(sizeof(double) * bins), "alloc derivative table");
        }
        ck(launch_lut_build(s, ctx->lut64.as<double>(), ctx->dmus.as<double>(), ctx->deps.as<double>(), st), "table build");
        ck(launch_lut_finalize(bins, ctx->lut64.as<double>(), ctx->lut32.as<float>(), ctx->lutaux.as<double>(), st),
           "table finalize");
        double mm[3];
        ck(cudaMemcpyAsync(mm, ctx->lutaux.p, sizeof(double) * 3, cudaMemcpyDeviceToHost, st), "read table range");
        ck(cudaMemcpyAsync(host32.data(), ctx->lut32.p, sizeof(float) * bins, cudaMemcpyDeviceToHost, st), "read table");
        ck(cudaStreamSynchronize(st), "table build");
        ctx->min_w = mm[0];
        ctx->max_w = mm[1];
        ctx->meta = LutMetaF{min_k, max_k, step, (int32_t)bins};
    }
    for (uint32_t i = 0; i < bins; ++i)
        if (!std::isfinite(host32[i])) fail(TWISTY_ERR_LUT_INVALID, "weight table has non-finite entries");
    // compensated-form tables, the fixed-point one scaled for paths of this N. Bins where the
    // fixed-point secant would err by more than 1e-7 per segment carry a NaN slope (paths
    // crossing them are re-weighed through the linear table); a table with too many of
    // them, or too wide a range, takes the exact blend.
    std::vector<float> lin, fix;
    double c0 = 0.0, inv_scale = 0.0, err = 0.0;
    int wide = 0;
    uint32_t steep = 0;
    const bool fixed_ok = compensated_tables(host32.data(), bins, ctx->meta.step, p.num_segments, lin, fix, c0,
                                             inv_scale, wide, err, steep);
    ck(cudaMemcpyAsync(ctx->lintab.p, lin.data(), sizeof(float) * lin.size(), cudaMemcpyHostToDevice, st), "upload linear table");
    if (fixed_ok)
        ck(cudaMemcpyAsync(ctx->fixtab.p, fix.data(), sizeof(float) * fix.size(), cudaMemcpyHostToDevice, st),
           "upload fixed-point table");
    ck(cudaStreamSynchronize(st), "tables");
    ctx->secant_err = err;
    ctx->exact_blend = fixed_ok ? 0 : 1;
    ctx->lf = fixed_ok ? LogFixed{c0, inv_scale, wide, (int32_t)steep} : LogFixed{0.0, 0.0, 0, (int32_t)steep};
    std::memcpy(ctx->lut_key, key, sizeof(key));
    ctx->lut_ready = true;
}

// -------------------------------------------------------------- normaliser
double normalizer_log10(twisty_ctx *ctx, uint32_t n, float ds, const twisty_bc &bc)
{
    if (n == 4) return norm_k4_log10(norm_z(bc, ds), ds);
    if (n == 5 || n == 6) {
        const uint32_t blocks = norm_partial_blocks();
        ck(ctx->norm_scratch.ensure(sizeof(double) * (blocks + 1)), "alloc normaliser scratch");
        double *d = ctx->norm_scratch.as<double>();
        ck(launch_norm_k56(norm_z(bc, ds), ds, d + 1, d, ctx->stream), "normaliser");
        double v = 0.0;
        ck(cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "read normaliser");
        ck(cudaStreamSynchronize(ctx->stream), "normaliser");
        return std::log10(v);
    }
    return 0.0;  // Norm returns 1.0 for any other N (PathWeightUtils.cpp:745-750)
}

// ------------------------------------------------------------ chain layout
void layout(twisty_ctx *ctx, uint64_t paths, uint32_t requested, uint32_t max_steps)
{
    ChainSpec &c = ctx->spec;
    if (paths == 0) {
        c.n_chains = 0;
        c.steps = 0;
        c.last_steps = 0;
        return;
    }
    uint64_t C = requested ? requested : 1;
    if (C > paths) C = paths;
    uint64_t L = (paths + C - 1) / C;
    if (L > max_steps) {
        L = max_steps;
    }
    C = (paths + L - 1) / L;
    if (C > 0xFFFFFFFFull) fail(TWISTY_ERR_INVALID_CONFIG, "too many chains");
    c.n_chains = (uint32_t)C;
    c.steps = (uint32_t)L;
    c.last_steps = (uint32_t)(paths - (C - 1) * L);
}

constexpr size_t kSmemCap = kCompSmemCap;

// Fewer warps per CTA until the table (when staged) and the chain state fit in shared memory;
// fails when even 4 warps do not fit.
void fit_table_smem(CompTuning &t, uint32_t bins, bool may_shrink)
{
    if (!comp_fit_smem(t, bins, may_shrink)) fail(TWISTY_ERR_UNSUPPORTED, "weight table too large to stage in shared memory");
}

// Forward passes of the full recompute: whether the table goes through L1. A table too large
// to stage beside the chain state costs warps per CTA; when staging it would leave fewer than
// comp_stage_min_warps (normally all of the shape's warps), it is gathered through L1 at the
// shape's warps instead. may_shrink false: the warps were set by the caller.
bool table_through_l1(const CompTuning &t, uint32_t bins, bool may_shrink)
{
    return comp_table_through_l1(t, bins, may_shrink);
}

// The context's shape for the passes that stage the table (export, adjoint).
CompTuning staged_tuning(const twisty_ctx *ctx)
{
    CompTuning t = ctx->tuning;
    t.lut_global = 0;
    fit_table_smem(t, ctx->p.num_curvature_steps, true);
    return t;
}

void prepare(twisty_ctx *ctx, const twisty_bc *bcp)
{
    const double t0 = now_ms();
    validate(ctx->p);
    validate_bc(bcp);
    set_device(ctx);
    const twisty_params &p = ctx->p;
    const twisty_bc bc = *bcp;
    const uint32_t N = p.num_segments;
    const float ds = bc.arclength / (float)N;
    build_tables(ctx, ds, false);
    ctx->log10_norm = normalizer_log10(ctx, N, ds, bc);
    // initial curve
    std::vector<float> pos;
    if (!ctx->user_curve.empty()) {
        if (ctx->user_curve.size() != 3 * (size_t)(N + 1)) fail(TWISTY_ERR_INVALID_ARGUMENT, "initial curve has the wrong number of points");
        pos = ctx->user_curve;
    } else {
        std::string e;
        if (!bootstrap_curve(bc, N, p.bootstrap_seed, p.bootstrap_kind, pos, e)) fail(TWISTY_ERR_INFEASIBLE_GEOMETRY, e);
    }
    ctx->init_pos_host = pos;
    std::vector<float> seg(3 * (size_t)N);
    for (uint32_t i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) seg[3 * i + k] = pos[3 * (i + 1) + k] - pos[3 * i + k];

    ChainSpec &c = ctx->spec;
    c = ChainSpec{};
    c.n_segments = N;
    c.arclength = bc.arclength;
    c.ds = ds;
    c.inv_ds = (float)N / bc.arclength;
    c.seed = seed_of(p.perturb_seed);
    c.experiment = p.experiment_id;
    c.chain0 = p.chain_offset;
    c.burn_in = (uint32_t)std::min<uint64_t>(p.paths_to_skip, 0xFFFFFFFFull);
    c.k_eff = std::min<uint32_t>(p.max_sub_chain, N - 2);
    c.max_angle = p.max_angle;
    c.absorption_factor = (double)std::exp(-p.absorption * ds);
    c.eval_shift[0] = p.eval_end_shift.x;
    c.eval_shift[1] = p.eval_end_shift.y;
    c.eval_shift[2] = p.eval_end_shift.z;
    c.has_eval_shift = (p.eval_end_shift.x != 0.f || p.eval_end_shift.y != 0.f || p.eval_end_shift.z != 0.f) ? 1 : 0;
    c.incr_resync = p.form == TWISTY_FORM_COMPENSATED ? p.incremental_resync : 0;

    uint32_t requested = p.num_chains;
    uint32_t max_steps = 0xFFFFFFFFu - c.burn_in;
    if (p.form == TWISTY_FORM_PLAIN_FP32) {
        if (!requested) requested = (uint32_t)ctx->sm_count * 256;
        // one CombinedWeightValues_C per chain holds at most 1e6 paths (CombinedWeightUtils.h:22-24)
        max_steps = std::min<uint32_t>(max_steps, 1000000u);
    } else if (p.form == TWISTY_FORM_COMPENSATED) {
        ctx->tuning = comp_default_tuning(N, false, p.paths_to_generate, p.paths_to_skip);
        bool default_shape = !p.comp_group && !p.comp_spl && !p.comp_warps;
        if (default_shape && tune_lookup(ctx->device_name, N, p.num_curvature_steps, ctx->tuning)) default_shape = false;
        if (p.comp_group || p.comp_spl) {
            if (!p.comp_group || !p.comp_spl) fail(TWISTY_ERR_INVALID_CONFIG, "comp_group and comp_spl are set together");
            ctx->tuning.group = (int)p.comp_group;
            ctx->tuning.spl = (int)p.comp_spl;
            if (!p.comp_warps) ctx->tuning.warps_per_block = (p.comp_spl >= 12) ? 24 : 32;
        }
        if (p.comp_warps) ctx->tuning.warps_per_block = (int)p.comp_warps;
        // A pass of fewer chains than a full grid of the shape holds (num_chains set by the
        // caller) takes fewer warps per CTA, so that its chains spread over every SM: 4096
        // chains of the 8 x 16 shape would fill 43 CTAs of 24 warps on 43 of 148 SMs, and fill
        // 147 CTAs of 7 warps instead. Chain ids and proposals do not depend on the layout.
        // When that leaves fewer than 12 warps per CTA, a default shape of 8 or more lanes per
        // chain doubles its lanes per chain and halves its segments per lane (the same slots)
        // while the kernels have such a shape: more warps to hide latency with (shapes of 1 and
        // 4 lanes pack chains into warps on purpose, and keep their shorter-side moves). The
        // differentiation configuration (N = 128, 4096 chains) takes 16 x 8 at 14 warps over
        // 8 x 16 at 7: forward 2.61 -> 2.20 ms, adjoint call 6.19 -> 4.57 ms.
        if (requested && !p.comp_warps) {
            const uint64_t chains = std::min<uint64_t>(requested, std::max<uint64_t>(p.paths_to_generate, 1));
            auto need_warps = [&](const CompTuning &t) {
                const uint64_t per_warp_grid = (uint64_t)ctx->sm_count * (32u / (uint32_t)t.group);
                return std::max<uint64_t>((chains + per_warp_grid - 1) / per_warp_grid, 1);
            };
            uint64_t need = need_warps(ctx->tuning);
            if (need < (uint64_t)ctx->tuning.warps_per_block) {
                ctx->tuning.warps_per_block = (int)need;
                while (default_shape && need < 12 && ctx->tuning.group >= 8 && ctx->tuning.group < 32 &&
                       ctx->tuning.spl % 2 == 0) {
                    CompTuning w = ctx->tuning;
                    w.group *= 2;
                    w.spl /= 2;
                    if (!comp_tuning_supported(w, N, c.k_eff)) break;
                    need = std::min<uint64_t>(need_warps(w), 24);   // 24 warps: within every shape's thread limit
                    w.warps_per_block = (int)need;
                    ctx->tuning = w;
                }
            }
        }
        ctx->tuning.exact_blend = ctx->exact_blend;
        if (!comp_tuning_supported(ctx->tuning, N, c.k_eff)) fail(TWISTY_ERR_UNSUPPORTED, "no compensated kernel shape for this N / max_sub_chain");
        // the table's placement (table_through_l1); comp_table_memory 1 / 2 force the choice
        ctx->tuning.lut_global = 0;
        const bool can_global = c.incr_resync <= 1 && !c.has_eval_shift;
        const bool few_warps = p.comp_table_memory == 0 && can_global &&
                               table_through_l1(ctx->tuning, p.num_curvature_steps, p.comp_warps == 0);
        if (p.comp_table_memory == 2 || few_warps) {
            if (!can_global)
                fail(TWISTY_ERR_UNSUPPORTED, "comp_table_memory 2 serves plain forward passes (no incremental or shifted runs)");
            ctx->tuning.lut_global = 1;
        }
        fit_table_smem(ctx->tuning, p.num_curvature_steps, p.comp_warps == 0);
        if (!requested)
            requested = (uint32_t)ctx->sm_count * (uint32_t)ctx->tuning.warps_per_block * (32u / (uint32_t)ctx->tuning.group);
    } else {
        if (!requested) requested = (uint32_t)ctx->sm_count * 256;
    }
    layout(ctx, p.paths_to_generate, requested, max_steps);

    cudaStream_t st = ctx->stream;
    ck(ctx->init_pos.ensure(sizeof(float) * pos.size()), "alloc curve");
    ck(ctx->init_seg.ensure(sizeof(float) * seg.size()), "alloc curve");
    ck(cudaMemcpyAsync(ctx->init_pos.p, pos.data(), sizeof(float) * pos.size(), cudaMemcpyHostToDevice, st), "upload curve");
    ck(cudaMemcpyAsync(ctx->init_seg.p, seg.data(), sizeof(float) * seg.size(), cudaMemcpyHostToDevice, st), "upload curve");
    const uint32_t C = std::max<uint32_t>(c.n_chains, 1);
    ck(ctx->chain_out.ensure(sizeof(ChainOut) * C), "alloc chain results");
    ck(ctx->reduce_out.ensure(sizeof(ReduceOut)), "alloc result");
    if (p.form == TWISTY_FORM_PLAIN_FP32) {
        ck(ctx->state.ensure(sizeof(float) * plain_state_floats_per_chain(N) * C), "alloc chain state");
    } else if (p.form == TWISTY_FORM_FP64) {
        ck(ctx->state.ensure(sizeof(double) * 3 * (size_t)(N + 1) * C), "alloc chain state");
        if (p.lut_mode == TWISTY_LUT_FAITHFUL) {
            // the FP64 form weighs with a double table; rebuild it in double
            ctx->lut_ready = false;
            twisty_params saved = ctx->p;
            ctx->p.lut_mode = TWISTY_LUT_FP64;
            build_tables(ctx, ds, false);
            ctx->p = saved;
        }
    } else {
        ck(ctx->partials.ensure(sizeof(double2) * comp_blocks(c, ctx->tuning)), "alloc block partials");
    }
    // the FP64 replay of the first chains, on the double copy of the run's table
    ctx->check_chains = (p.form != TWISTY_FORM_FP64) ? std::min<uint32_t>(p.fp64_check_chains, c.n_chains) : 0u;
    if (ctx->check_chains) {
        ck(ctx->check_state.ensure(sizeof(double) * 3 * (size_t)(N + 1) * ctx->check_chains), "alloc FP64 check");
        ck(ctx->check_out.ensure(sizeof(ChainOut) * ctx->check_chains), "alloc FP64 check");
        if (p.lut_mode == TWISTY_LUT_FP64) {
            const double max_k = (2.0 / (double)ds) * 1.01;
            ctx->check_meta[0] = 0.0;
            ctx->check_meta[1] = max_k;
            ctx->check_meta[2] = max_k / (double)(p.num_curvature_steps - 1);
        } else {
            ctx->check_meta[0] = ctx->meta.min_k;
            ctx->check_meta[1] = ctx->meta.max_k;
            ctx->check_meta[2] = ctx->meta.step;
        }
    }
    ck(cudaStreamSynchronize(st), "prepare");
    ctx->kernels_per_launch = c.n_chains ? 2 + (ctx->check_chains ? 1 : 0) : 0;
    ctx->bc = bc;
    ctx->prepared = true;
    ctx->launched = false;
    ctx->setup_ms = now_ms() - t0;
}

void launch(twisty_ctx *ctx, cudaStream_t st)
{
    if (!ctx->prepared) fail(TWISTY_ERR_INVALID_ARGUMENT, "twisty_launch before twisty_prepare");
    set_device(ctx);
    const ChainSpec &c = ctx->spec;
    ck(cudaEventRecord(ctx->ev[0], st), "event");
    if (c.n_chains) {
        const twisty_params &p = ctx->p;
        if (p.form == TWISTY_FORM_PLAIN_FP32) {
            ck(launch_plain_chains(c, ctx->init_pos.as<float>(), ctx->state.as<float>(), ctx->lut32.as<float>(), ctx->meta,
                                   ctx->chain_out.as<ChainOut>(), st),
               "plain chain kernel");
        } else if (p.form == TWISTY_FORM_FP64) {
            const double max_k = (2.0 / (double)c.ds) * 1.01;
            const double step = max_k / (double)(p.num_curvature_steps - 1);
            ck(launch_fp64_chains(c, ctx->init_pos.as<float>(), ctx->state.as<double>(), ctx->lut64.as<double>(), 0.0, max_k,
                                  step, (int32_t)p.num_curvature_steps, ctx->chain_out.as<ChainOut>(), st),
               "fp64 chain kernel");
        } else {
            ck(launch_comp_chains(c, ctx->tuning, ctx->init_seg.as<float>(), ctx->fixtab.as<float2>(), ctx->lintab.as<float2>(),
                                  ctx->meta, ctx->chain_out.as<ChainOut>(), ctx->partials.as<double2>(), st, ctx->lf),
               "compensated chain kernel");
        }
    }
    ck(cudaEventRecord(ctx->ev[1], st), "event");
    if (c.n_chains) ck(launch_reduce(ctx->chain_out.as<ChainOut>(), c.n_chains, ctx->reduce_out.as<ReduceOut>(), st), "reduction");
    ck(cudaEventRecord(ctx->ev[2], st), "event");
    if (ctx->check_chains) {
        // after the timed pass: the first chains again, in FP64, on the same proposals
        ChainSpec ck64 = c;
        ck64.n_chains = ctx->check_chains;
        ck64.last_steps = (ctx->check_chains == c.n_chains) ? c.last_steps : c.steps;
        ck64.incr_resync = 0;
        ck(launch_fp64_chains(ck64, ctx->init_pos.as<float>(), ctx->check_state.as<double>(), ctx->lut64.as<double>(),
                              ctx->check_meta[0], ctx->check_meta[1], ctx->check_meta[2],
                              (int32_t)ctx->p.num_curvature_steps, ctx->check_out.as<ChainOut>(), st),
           "FP64 check");
    }
    ck(cudaEventRecord(ctx->ev[3], st), "event");
    ctx->launched = true;
}

void collect(twisty_ctx *ctx, twisty_result *res)
{
    if (!ctx->launched) fail(TWISTY_ERR_INVALID_ARGUMENT, "twisty_collect before twisty_launch");
    if (!res) fail(TWISTY_ERR_INVALID_ARGUMENT, "result is NULL");
    set_device(ctx);
    ReduceOut r{};
    r.log10_sum = -std::numeric_limits<double>::infinity();
    // The pass may have been enqueued on any stream; its last event orders the copy.
    ck(cudaEventSynchronize(ctx->ev[2]), "sync");
    if (ctx->spec.n_chains) {
        ck(cudaMemcpyAsync(&r, ctx->reduce_out.p, sizeof(r), cudaMemcpyDeviceToHost, ctx->stream), "read result");
        ck(cudaStreamSynchronize(ctx->stream), "read result");
    }
    float a = 0, b = 0;
    ck(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]), "event time");
    ck(cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]), "event time");
    std::memset(res, 0, sizeof(*res));
    res->log10_normalizer = ctx->log10_norm;
    res->log10_weight = r.log10_sum + ctx->log10_norm;
    res->total_paths = r.valid;
    res->failed_paths = r.failed;
    res->clamped_curvatures = r.clamped;
    res->log10_mean_weight = r.valid ? res->log10_weight - std::log10((double)r.valid) : -std::numeric_limits<double>::infinity();
    res->rel_std_error = r.rel_se;
    res->num_chains = ctx->spec.n_chains;
    res->steps_per_chain = ctx->spec.steps;
    res->setup_ms = ctx->setup_ms;
    res->perturb_ms = a;
    res->weighting_ms = b;
    res->table_form = TWISTY_TABLE_NONE;
    const double segs = (double)(ctx->spec.n_segments - 1);
    if (ctx->p.form == TWISTY_FORM_COMPENSATED) {
        const bool exact = ctx->tuning.exact_blend || ctx->lf.inv_scale == 0.0 || ctx->spec.has_eval_shift;
        res->table_form = exact ? TWISTY_TABLE_EXACT_BLEND : ctx->lf.wide ? TWISTY_TABLE_FIXED_WIDE : TWISTY_TABLE_FIXED_NARROW;
        res->steep_bins = exact ? 0u : (uint32_t)ctx->lf.steep;
        res->kernel_shape = ((uint32_t)ctx->tuning.group << 8) | (uint32_t)ctx->tuning.spl;
        // per segment: entry and correction each rounded to 2^-(s+1), plus the secant's error;
        // exact blend: the float blend and the hardware log2 (under 4e-7 in log10 together)
        res->weight_error_bound = exact ? segs * 4e-7 : segs * (ctx->lf.inv_scale + ctx->secant_err);
    } else if (ctx->p.form == TWISTY_FORM_PLAIN_FP32) {
        res->weight_error_bound = segs * 2.6e-8;   // the blend rounded to float: 2^-24 relative
    }
    res->fp64_rel_error = std::numeric_limits<double>::quiet_NaN();
    res->fp64_check_chains = ctx->check_chains;
    if (ctx->check_chains) {
        const uint32_t K = ctx->check_chains;
        std::vector<ChainOut> a(K), b(K);
        ck(cudaEventSynchronize(ctx->ev[3]), "sync");
        ck(cudaMemcpyAsync(a.data(), ctx->chain_out.p, sizeof(ChainOut) * K, cudaMemcpyDeviceToHost, ctx->stream), "read");
        ck(cudaMemcpyAsync(b.data(), ctx->check_out.p, sizeof(ChainOut) * K, cudaMemcpyDeviceToHost, ctx->stream), "read");
        ck(cudaStreamSynchronize(ctx->stream), "read FP64 check");
        auto lse = [](const std::vector<ChainOut> &v) {
            double m = -std::numeric_limits<double>::infinity();
            for (const ChainOut &o : v) m = std::max(m, o.log10_sum);
            if (!std::isfinite(m)) return m;
            double sum = 0.0;
            for (const ChainOut &o : v)
                if (std::isfinite(o.log10_sum)) sum += std::pow(10.0, o.log10_sum - m);
            return m + std::log10(sum);
        };
        const double la = lse(a), lb = lse(b);
        if (std::isfinite(la) && std::isfinite(lb)) res->fp64_rel_error = std::fabs(std::pow(10.0, la - lb) - 1.0);
    }
}

twisty_status guard(twisty_ctx *ctx, const std::function<void()> &f)
{
    try {
        f();
        if (ctx) ctx->err.clear();
        return TWISTY_OK;
    } catch (const Failure &e) {
        if (ctx) ctx->err = e.msg;
        return e.s;
    } catch (const std::bad_alloc &) {
        if (ctx) ctx->err = "host out of memory";
        return TWISTY_ERR_OUT_OF_MEMORY;
    } catch (const std::exception &e) {
        if (ctx) ctx->err = e.what();
        return TWISTY_ERR_INVALID_ARGUMENT;
    } catch (...) {
        if (ctx) ctx->err = "unknown error";
        return TWISTY_ERR_INVALID_ARGUMENT;
    }
}

thread_local std::string g_free_err;

// The angles GeometryRandom_ExportPaths records for five-segment paths
// (FullExperimentRunnerOptimalPerturb.cpp:318-357), in float.
void five_segment_angles(const float *p, float out[3])
{
    auto sub = [&](int a, int b, float v[3]) {
        for (int k = 0; k < 3; ++k) v[k] = p[3 * a + k] - p[3 * b + k];
    };
    auto norm = [](float v[3]) {
        const float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int k = 0; k < 3; ++k) v[k] *= inv;
    };
    auto cross = [](const float a[3], const float b[3], float r[3]) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
    };
    float s1[3], z[3], x[3], y[3], v[3];
    sub(2, 1, s1);
    norm(s1);
    out[0] = std::acos(s1[2]);
    out[1] = std::atan2(s1[1], s1[0]);
    sub(4, 2, z);
    norm(z);
    float other[3] = {1.0f, 0.0f, 0.0f};
    if (std::fabs(z[0]) >= 0.99f) { other[0] = 0.0f; other[1] = 1.0f; }
    cross(z, other, x);
    norm(x);
    cross(z, x, y);
    sub(3, 2, v);
    norm(v);
    out[2] = std::atan2(v[0] * y[0] + v[1] * y[1] + v[2] * y[2], v[0] * x[0] + v[1] * x[1] + v[2] * x[2]);
}

// BeginPathBatchOutput / GeometryRandom_ExportPaths / EndPathBatchOutput file set
// (ExperimentRunner.cpp:210-262,303-345,383-396; FullExperimentRunnerOptimalPerturb.cpp:746-856)
// under dir/GeneratedCurves/. One batch per exported chain, recorded in the .pmd as
// "chain 0 count".
void write_path_batch(const char *dir, const twisty_bc &bc, uint32_t N, double log10_norm, const std::vector<float> &pos,
                      const std::vector<double> &w, const std::vector<uint32_t> &chain_of)
{
    namespace fs = std::filesystem;
    std::error_code ec;
    const fs::path out = fs::path(dir) / "GeneratedCurves";
    fs::create_directories(out, ec);
    if (ec) fail(TWISTY_ERR_IO, "cannot create " + out.string());
    auto open = [&](const char *name, std::ios::openmode m) {
        std::ofstream f(out / name, m);
        if (!f.is_open()) fail(TWISTY_ERR_IO, std::string("cannot open ") + (out / name).string());
        return f;
    };
    {
        std::ofstream f = open("BoundaryConditions.bcf", std::ios::binary);
        const float v[13] = {bc.start_pos.x, bc.start_pos.y, bc.start_pos.z, bc.start_dir.x, bc.start_dir.y, bc.start_dir.z,
                             bc.end_pos.x, bc.end_pos.y, bc.end_pos.z, bc.end_dir.x, bc.end_dir.y, bc.end_dir.z, bc.arclength};
        f.write(reinterpret_cast<const char *>(v), sizeof(v));
        f.write(reinterpret_cast<const char *>(&N), sizeof(N));
    }
    {
        std::string name = fs::path(dir).filename().string();
        if (name.empty()) name = fs::path(dir).parent_path().filename().string();
        std::ofstream f = open("index.json", std::ios::out);
        f << "{\n    \"experiment_name\": \"" << name << "\",\n    \"path_batch_links\": []\n}" << std::endl;
    }
    std::ofstream pmd = open("Paths_Metadata.pmd", std::ios::out);
    std::ofstream pbd = open("Paths_Binary.pbd", std::ios::binary);
    std::ofstream bdt = open("Log10PathWeights_Binary.bdt", std::ios::binary);
    std::ofstream pwt = open("Log10PathWeights_Text.pwt", std::ios::out);
    std::ofstream fsb = open("FiveSegment_Binary.bdt", std::ios::binary);
    const size_t stride = 3 * (size_t)(N + 1);
    size_t i = 0;
    while (i < w.size()) {
        size_t j = i;
        while (j < w.size() && chain_of[j] == chain_of[i]) ++j;
        const uint32_t ch = chain_of[i];
        pmd << ch << " " << 0 << " " << (j - i) << std::endl;
        pbd.write(reinterpret_cast<const char *>(pos.data() + i * stride), sizeof(float) * stride * (j - i));
        for (size_t k = i; k < j; ++k) {
            // the ".bdt" holds linear weights including the normaliser (:751-752)
            const double lin = std::pow(10.0, w[k] + log10_norm);
            bdt.write(reinterpret_cast<const char *>(&lin), sizeof(lin));
            if ((static_cast<uint32_t>((double)(k - i) + ch * (10000.0 / 12.0)) % 10000) == 0) pwt << lin << std::endl;
            float ang[3] = {0.0f, 0.0f, 0.0f};
            if (N == 5) five_segment_angles(pos.data() + k * stride, ang);
            fsb.write(reinterpret_cast<const char *>(ang), sizeof(ang));
        }
        i = j;
    }
}

}  // namespace

namespace twisty {
// Message returned by twisty_last_error(NULL) for entry points without a context.
void set_free_error(const std::string &msg) { g_free_err = msg; }
}  // namespace twisty

extern "C" {

int twisty_abi_version(void) { return TWISTY_B200_ABI_VERSION; }

const char *twisty_status_string(twisty_status s)
{
    switch (s) {
        case TWISTY_OK: return "ok";
        case TWISTY_ERR_INVALID_ARGUMENT: return "invalid argument";
        case TWISTY_ERR_INVALID_CONFIG: return "invalid config";
        case TWISTY_ERR_INFEASIBLE_GEOMETRY: return "infeasible geometry";
        case TWISTY_ERR_LUT_INVALID: return "invalid weight table";
        case TWISTY_ERR_CUDA: return "CUDA error";
        case TWISTY_ERR_DEVICE_TIMEOUT: return "device timeout";
        case TWISTY_ERR_IO: return "I/O error";
        case TWISTY_ERR_UNSUPPORTED: return "unsupported";
        case TWISTY_ERR_NO_DEVICE: return "no CUDA device";
        case TWISTY_ERR_OUT_OF_MEMORY: return "out of memory";
    }
    return "unknown status";
}

void twisty_params_init(twisty_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->struct_size = sizeof(twisty_params);
    // ExperimentParameters / WeightingParameters member initialisers
    // (Twisty/ExperimentRunner.h:42-68, Twisty/PathWeightUtils.h:35-48)
    p->paths_to_generate = 0;
    p->paths_to_skip = 0;
    p->num_segments = 4;
    p->mu = 0.1f;
    p->num_steps_int = 2000;
    p->min_bound = 0.0f;
    p->max_bound = 100.0f;
    p->eps = 0.01f;
    p->bias = 1.0f;
    p->scatter = 0.0f;
    p->absorption = 0.0f;
    p->num_curvature_steps = 10000;
    p->form = TWISTY_FORM_COMPENSATED;
    p->lut_mode = TWISTY_LUT_FP64;
    p->max_sub_chain = 25;                 // FullExperimentRunnerOptimalPerturb.cpp:483-484
    p->max_angle = 3.141592653589793f;     // :501-502
    p->device = 0;
}

twisty_status twisty_params_from_config(const char *text, int is_yaml, twisty_params *out, twisty_bc *bc)
{
    if (!text || !out) return TWISTY_ERR_INVALID_ARGUMENT;
    twisty::Node root;
    std::string err;
    const bool ok = is_yaml ? twisty::parse_yaml(text, root, err) : twisty::parse_json(text, root, err);
    if (!ok) {
        g_free_err = err;
        return TWISTY_ERR_INVALID_CONFIG;
    }
    twisty_params p;
    twisty_params_init(&p);
    if (!twisty::params_from_node(root, p, bc, err)) {
        g_free_err = err;
        return TWISTY_ERR_INVALID_CONFIG;
    }
    *out = p;
    return TWISTY_OK;
}

twisty_status twisty_create(const twisty_params *p, twisty_ctx **out)
{
    if (!p || !out) return TWISTY_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (p->struct_size != sizeof(twisty_params)) return TWISTY_ERR_INVALID_ARGUMENT;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        g_free_err = "no CUDA device";
        return TWISTY_ERR_NO_DEVICE;
    }
    if (p->device < 0 || p->device >= n) {
        g_free_err = "device ordinal out of range";
        return TWISTY_ERR_INVALID_ARGUMENT;
    }
    twisty_ctx *ctx = new (std::nothrow) twisty_ctx();
    if (!ctx) return TWISTY_ERR_OUT_OF_MEMORY;
    ctx->p = *p;
    ctx->device = p->device;
    const twisty_status s = guard(ctx, [&] {
        set_device(ctx);
        int sms = 0;
        ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "device query");
        ctx->sm_count = sms;
        cudaDeviceProp prop{};
        ck(cudaGetDeviceProperties(&prop, ctx->device), "device query");
        ctx->device_name = prop.name;
        ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
        for (auto &e : ctx->ev) ck(cudaEventCreate(&e), "event");
    });
    if (s != TWISTY_OK) {
        g_free_err = ctx->err;
        twisty_destroy(ctx);
        return s;
    }
    *out = ctx;
    return TWISTY_OK;
}

void twisty_destroy(twisty_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    DevBuf *bufs[] = {&ctx->lut64, &ctx->lut32, &ctx->fixtab, &ctx->lintab, &ctx->dmus, &ctx->deps, &ctx->lutaux,
                      &ctx->init_pos, &ctx->init_seg, &ctx->state, &ctx->chain_out, &ctx->partials, &ctx->reduce_out,
                      &ctx->norm_scratch, &ctx->multi.dev, &ctx->check_state, &ctx->check_out};
    for (DevBuf *b : bufs) b->release();
    ctx->batch_graph.release();
    ctx->batch.release();
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *twisty_last_error(const twisty_ctx *ctx) { return ctx ? ctx->err.c_str() : g_free_err.c_str(); }

twisty_status twisty_update_params(twisty_ctx *ctx, const twisty_params *p)
{
    if (!ctx || !p) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (p->struct_size != sizeof(twisty_params)) fail(TWISTY_ERR_INVALID_ARGUMENT, "struct_size mismatch");
        if (p->device != ctx->device) fail(TWISTY_ERR_INVALID_ARGUMENT, "the device of a context cannot change");
        ctx->p = *p;
        ctx->prepared = false;
        ctx->launched = false;
        ctx->lut_ready = false;   // the next run builds its tables again
    });
}

twisty_status twisty_prepare(twisty_ctx *ctx, const twisty_bc *bc)
{
    if (!ctx) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] { prepare(ctx, bc); });
}

twisty_status twisty_launch(twisty_ctx *ctx, void *stream)
{
    if (!ctx) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] { launch(ctx, stream ? (cudaStream_t)stream : ctx->stream); });
}

twisty_status twisty_collect(twisty_ctx *ctx, twisty_result *res)
{
    if (!ctx) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] { collect(ctx, res); });
}

uint32_t twisty_launch_kernel_count(const twisty_ctx *ctx) { return ctx ? ctx->kernels_per_launch : 0; }

twisty_status twisty_run(twisty_ctx *ctx, const twisty_bc *bc, twisty_result *res)
{
    if (!ctx || !res) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        const double t0 = now_ms();
        prepare(ctx, bc);
        launch(ctx, ctx->stream);
        collect(ctx, res);
        res->total_ms = now_ms() - t0;
    });
}

// Independent-sample M-segment Monte Carlo (MSegmentPathGenerationMC,
// Experiments/ExperimentBase.cpp:1246-1386): fresh random curves from the recursive
// bootstrapper, weighed with the context's table (plain form: the reference's FP32 semantics;
// compensated: the fixed-point weigher), the estimate being their mean weight. Paths are built
// and weighed in chunks of at most 1 GB of positions; each chunk's FP64 reduction treats its
// paths as independent samples, and the chunks combine by log-sum-exp, errors in quadrature.
twisty_status twisty_run_msegment(twisty_ctx *ctx, const twisty_bc *bc, twisty_result *res)
{
    if (!ctx || !bc || !res) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        const double t0 = now_ms();
        const twisty_params p = ctx->p;
        validate(p);
        validate_bc(bc);
        if (p.form == TWISTY_FORM_FP64) fail(TWISTY_ERR_UNSUPPORTED, "M-segment runs weigh in the plain or compensated form");
        const uint32_t N = p.num_segments;
        if (!bootstrap_resolvable(N))
            fail(TWISTY_ERR_UNSUPPORTED, "M-segment paths come from the recursive bootstrapper: N-2 in {4, 6, 8, 12, 16, 24, 32, 48, ...}");
        set_device(ctx);
        const float ds = bc->arclength / (float)N;
        build_tables(ctx, ds, false);
        const double log10_norm = normalizer_log10(ctx, N, ds, *bc);
        // the fixed points (ExperimentBase.cpp:1253-1260)
        const float sp[3] = {bc->start_pos.x, bc->start_pos.y, bc->start_pos.z};
        const float sd[3] = {bc->start_dir.x, bc->start_dir.y, bc->start_dir.z};
        const float ep[3] = {bc->end_pos.x, bc->end_pos.y, bc->end_pos.z};
        const float ed[3] = {bc->end_dir.x, bc->end_dir.y, bc->end_dir.z};
        float p1[3], pm1[3];
        for (int k = 0; k < 3; ++k) {
            p1[k] = sp[k] + ds * sd[k];
            pm1[k] = ep[k] - ds * ed[k];
        }
        const uint64_t total = p.paths_to_generate;
        const uint64_t per_path = 3 * sizeof(float) * (uint64_t)(N + 1);
        const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(total, (1ull << 30) / per_path));
        cudaStream_t st = ctx->stream;
        DevBuf dpos, dw, dv, dch, dred, drg;
        struct Release {
            DevBuf *b[6];
            ~Release()
            {
                for (DevBuf *x : b) x->release();
            }
        } rel{{&dpos, &dw, &dv, &dch, &dred, &drg}};
        // the samples of a chunk reduce in slices of kSlice, one CTA each, combined on the host
        constexpr uint64_t kSlice = 16384;
        const uint64_t max_slices = (chunk + kSlice - 1) / kSlice;
        ck(dpos.ensure(per_path * chunk), "alloc paths");
        ck(dw.ensure(sizeof(double) * chunk), "alloc weights");
        ck(dv.ensure(chunk), "alloc validity");
        ck(dch.ensure(sizeof(ChainOut) * chunk), "alloc samples");
        ck(dred.ensure(sizeof(ReduceOut) * max_slices), "alloc result");
        ck(drg.ensure(sizeof(uint2) * max_slices), "alloc slices");
        std::vector<uint2> slices(max_slices);
        for (uint64_t k = 0; k < max_slices; ++k) slices[k] = make_uint2((uint32_t)(k * kSlice), (uint32_t)kSlice);
        std::vector<ReduceOut> parts(max_slices);
        const double af = (double)std::exp(-p.absorption * ds);
        const float inv_ds = (float)N / bc->arclength;
        const uint64_t seed = seed_of(p.perturb_seed);
        double m = -std::numeric_limits<double>::infinity(), sum = 0.0, var = 0.0;
        uint64_t valid = 0, failed = 0;
        float gpu_ms = 0.f;
        for (uint64_t done = 0; done < total; done += chunk) {
            const uint64_t n = std::min(chunk, total - done);
            ck(cudaEventRecord(ctx->ev[0], st), "event");
            ck(launch_msegment_paths(N, ds, sp, p1, pm1, ep, seed, p.experiment_id, p.chain_offset * total + done, n,
                                     dpos.as<float>(), st),
               "path generation");
            if (p.form == TWISTY_FORM_PLAIN_FP32)
                ck(launch_weigh_plain(dpos.as<float>(), n, N, inv_ds, ctx->lut32.as<float>(), ctx->meta, af,
                                      dw.as<double>(), dv.as<uint8_t>(), nullptr, st),
                   "weigh kernel");
            else
                ck(launch_weigh_comp(dpos.as<float>(), n, N, inv_ds, ctx->fixtab.as<float2>(), ctx->lintab.as<float2>(),
                                     ctx->exact_blend, ctx->meta, std::log10(af), dw.as<double>(), dv.as<uint8_t>(),
                                     nullptr, st, ctx->lf),
                   "weigh kernel");
            ck(launch_pack_paths(dw.as<double>(), dv.as<uint8_t>(), n, dch.as<ChainOut>(), st), "pack");
            const uint64_t ns = (n + kSlice - 1) / kSlice;
            slices[ns - 1].y = (uint32_t)(n - (ns - 1) * kSlice);
            ck(cudaMemcpyAsync(drg.p, slices.data(), sizeof(uint2) * ns, cudaMemcpyHostToDevice, st), "upload slices");
            slices[ns - 1].y = (uint32_t)kSlice;
            ck(launch_reduce_segments(dch.as<ChainOut>(), drg.as<uint2>(), (uint32_t)ns, dred.as<ReduceOut>(), st),
               "reduction");
            ck(cudaEventRecord(ctx->ev[1], st), "event");
            ck(cudaMemcpyAsync(parts.data(), dred.p, sizeof(ReduceOut) * ns, cudaMemcpyDeviceToHost, st), "read result");
            ck(cudaStreamSynchronize(st), "M-segment chunk");
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]), "event time");
            gpu_ms += ms;
            for (uint64_t k = 0; k < ns; ++k) {
                const ReduceOut &r = parts[k];
                valid += r.valid;
                failed += r.failed;
                if (r.valid && r.log10_sum > -std::numeric_limits<double>::infinity()) {
                    // running log-sum-exp of the chunk sums, absolute standard errors in quadrature
                    const double se = std::isnan(r.rel_se) ? 0.0 : r.rel_se;
                    if (r.log10_sum > m) {
                        const double f = std::pow(10.0, m - r.log10_sum);
                        sum *= f;
                        var *= f * f;
                        m = r.log10_sum;
                    }
                    const double x = std::pow(10.0, r.log10_sum - m);
                    sum += x;
                    var += (se * x) * (se * x);
                }
            }
        }
        std::memset(res, 0, sizeof(*res));
        res->log10_normalizer = log10_norm;
        const double log10_sum = sum > 0 ? m + std::log10(sum) : -std::numeric_limits<double>::infinity();
        res->log10_mean_weight = valid ? log10_sum - std::log10((double)valid) + log10_norm : -std::numeric_limits<double>::infinity();
        res->log10_weight = res->log10_mean_weight;   // the estimator is the mean (ExperimentBase.cpp:1378-1381)
        res->fp64_rel_error = std::numeric_limits<double>::quiet_NaN();
        res->weight_error_bound = (double)(N - 1) * (p.form == TWISTY_FORM_PLAIN_FP32 ? 2.6e-8
                                                     : ctx->exact_blend ? 4e-7 : ctx->lf.inv_scale + ctx->secant_err);
        res->rel_std_error = sum > 0 ? std::sqrt(var) / sum : NAN;
        res->total_paths = valid;
        res->failed_paths = failed;
        res->num_chains = 0;
        res->steps_per_chain = 0;
        res->perturb_ms = gpu_ms;
        res->total_ms = now_ms() - t0;
    });
}

twisty_status twisty_weight_paths(twisty_ctx *ctx, const twisty_bc *bc, const float *pos, uint64_t n_paths, int32_t form,
                                  double *log10w, uint8_t *valid, int32_t *bins)
{
    if (!ctx || !bc || (!pos && n_paths) || (!log10w && n_paths)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        validate(ctx->p);
        validate_bc(bc);
        set_device(ctx);
        const uint32_t N = ctx->p.num_segments;
        const float ds = bc->arclength / (float)N;
        build_tables(ctx, ds, false);
        if (n_paths == 0) return;
        cudaStream_t st = ctx->stream;
        DevBuf dpos, dw, dv, db;
        const size_t np = 3 * (size_t)(N + 1) * n_paths;
        try {
            ck(dpos.ensure(sizeof(float) * np), "alloc paths");
            ck(dw.ensure(sizeof(double) * n_paths), "alloc weights");
            ck(dv.ensure(n_paths), "alloc validity");
            if (bins) ck(db.ensure(sizeof(int32_t) * (N - 1) * n_paths), "alloc bins");
            ck(cudaMemcpyAsync(dpos.p, pos, sizeof(float) * np, cudaMemcpyHostToDevice, st), "upload paths");
            const float inv_ds = (float)N / bc->arclength;
            const double af = (double)std::exp(-ctx->p.absorption * ds);
            if (form == TWISTY_FORM_COMPENSATED) {
                ck(launch_weigh_comp(dpos.as<float>(), n_paths, N, inv_ds, ctx->fixtab.as<float2>(), ctx->lintab.as<float2>(),
                                     ctx->exact_blend, ctx->meta, std::log10(af), dw.as<double>(), dv.as<uint8_t>(),
                                     bins ? db.as<int32_t>() : nullptr, st, ctx->lf),
                   "weigh kernel");
            } else if (form == TWISTY_FORM_PLAIN_FP32) {
                ck(launch_weigh_plain(dpos.as<float>(), n_paths, N, inv_ds, ctx->lut32.as<float>(), ctx->meta, af,
                                      dw.as<double>(), dv.as<uint8_t>(), bins ? db.as<int32_t>() : nullptr, st),
                   "weigh kernel");
            } else {
                fail(TWISTY_ERR_UNSUPPORTED, "weight_paths supports the plain and compensated forms");
            }
            ck(cudaMemcpyAsync(log10w, dw.p, sizeof(double) * n_paths, cudaMemcpyDeviceToHost, st), "read weights");
            if (valid) ck(cudaMemcpyAsync(valid, dv.p, n_paths, cudaMemcpyDeviceToHost, st), "read validity");
            if (bins) ck(cudaMemcpyAsync(bins, db.p, sizeof(int32_t) * (N - 1) * n_paths, cudaMemcpyDeviceToHost, st), "read bins");
            ck(cudaStreamSynchronize(st), "weigh");
        } catch (...) {
            cudaStreamSynchronize(st);
            dpos.release(); dw.release(); dv.release(); db.release();
            throw;
        }
        dpos.release(); dw.release(); dv.release(); db.release();
    });
}

twisty_status twisty_build_lut(twisty_ctx *ctx, float ds, float *lut, twisty_lut_info *info)
{
    if (!ctx || !(ds > 0.0f)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        validate(ctx->p);
        set_device(ctx);
        build_tables(ctx, ds, false);
        if (lut) {
            ck(cudaMemcpyAsync(lut, ctx->lut32.p, sizeof(float) * ctx->p.num_curvature_steps, cudaMemcpyDeviceToHost,
                               ctx->stream), "read table");
            ck(cudaStreamSynchronize(ctx->stream), "read table");
        }
        if (info) {
            info->min_curvature = ctx->meta.min_k;
            info->max_curvature = ctx->meta.max_k;
            info->curvature_step = ctx->meta.step;
            info->min_segment_weight = (float)ctx->min_w;
            info->max_segment_weight = (float)ctx->max_w;
            info->ds = ds;
            info->bins = ctx->p.num_curvature_steps;
        }
    });
}

twisty_status twisty_set_lut(twisty_ctx *ctx, const float *lut, const twisty_lut_info *info)
{
    if (!ctx || !lut || !info || info->bins < 2) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        for (uint32_t i = 0; i < info->bins; ++i)
            if (!std::isfinite(lut[i])) fail(TWISTY_ERR_LUT_INVALID, "table has non-finite entries");
        if (!(info->curvature_step > 0.0f) || !(info->max_curvature > info->min_curvature))
            fail(TWISTY_ERR_LUT_INVALID, "table range is empty");
        ctx->ext_lut.assign(lut, lut + info->bins);
        ctx->ext_info = *info;
        ctx->p.lut_mode = TWISTY_LUT_EXTERNAL;
        ctx->p.num_curvature_steps = info->bins;
        ctx->lut_ready = false;
        ctx->prepared = false;
    });
}

twisty_status twisty_normalizer_log10(twisty_ctx *ctx, uint32_t n, float ds, const twisty_bc *bc, double *out)
{
    if (!ctx || !bc || !out || n < 4 || !(ds > 0.0f)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        set_device(ctx);
        *out = normalizer_log10(ctx, n, ds, *bc);
    });
}

twisty_status twisty_bootstrap_curve(const twisty_params *p, const twisty_bc *bc, float *pos)
{
    if (!p || !bc || !pos) return TWISTY_ERR_INVALID_ARGUMENT;
    std::vector<float> v;
    std::string e;
    if (p->num_segments < 4) return TWISTY_ERR_INVALID_CONFIG;
    if (!(bc->arclength > 0.0f)) return TWISTY_ERR_INVALID_CONFIG;
    if (!twisty::bootstrap_curve(*bc, p->num_segments, p->bootstrap_seed, p->bootstrap_kind, v, e)) {
        g_free_err = e;
        return TWISTY_ERR_INFEASIBLE_GEOMETRY;
    }
    std::memcpy(pos, v.data(), sizeof(float) * v.size());
    return TWISTY_OK;
}

float twisty_min_arclength(const twisty_bc *bc, uint32_t n) { return bc ? twisty::min_arclength(*bc, n) : 0.0f; }

namespace {


std::string exp_msg(uint32_t e, const std::string &m)
{
    std::ostringstream o;
    o << "experiment " << e << ": " << m;
    return o.str();
}

// Many experiments in one pass (the receiver / pixel loops of the reference's drivers, e.g.
// Experiments/NoisyCircleExperiment.cpp:259-361, each a RunExperiment call there):
//  1. per experiment on the host: validation, initial curve, normaliser, chain layout;
//  2. on the device, all tables at once: FP64 quadrature (one CTA per bin per experiment),
//     finalisation and the compensated-form tables (one CTA per experiment);
//  3. experiments bucketed by kernel shape (lanes per chain x segments per lane, exact or
//     fixed-point table); work items = (experiment, first chain of a CTA), sorted by cost
//     (steps x N) so the longest start first; each bucket is one persistent launch on its
//     own stream taking items from a device counter, so one bucket's tail overlaps the next;
//  4. one segmented FP64 reduction (a CTA per experiment).
// Steps 3-4 are captured once as a CUDA graph and replayed `iters` times; results are those
// of the last replay, perturb_ms the mean replay time.
void run_batch(twisty_ctx *ctx, const twisty_experiment *ex, uint32_t n, uint32_t iters, twisty_result *res,
               const BatchAdjointOut *adj = nullptr)
{
    const double t0 = now_ms();
    const twisty_params p = ctx->p;
    {
        twisty_params pv = p;  // num_segments comes from each experiment
        pv.num_segments = 4;
        validate(pv);
    }
    if (p.form != TWISTY_FORM_COMPENSATED) fail(TWISTY_ERR_UNSUPPORTED, "batched runs use the compensated form");
    if (p.lut_mode != TWISTY_LUT_FP64 && p.lut_mode != TWISTY_LUT_MULTI_DS)
        fail(TWISTY_ERR_UNSUPPORTED, "batched runs build their tables on the device (lut_mode FP64) or take them "
                                     "from the multi-ds set (lut_mode MULTI_DS)");
    const bool multi = p.lut_mode == TWISTY_LUT_MULTI_DS;
    if (multi) check_multi(ctx, p);
    if (n > 65535u) fail(TWISTY_ERR_INVALID_ARGUMENT, "at most 65535 experiments per batch");
    set_device(ctx);
    for (uint32_t e = 0; e < n; ++e) std::memset(&res[e], 0, sizeof(twisty_result));
    if (n == 0) {
        if (adj && adj->total) {
            adj->total[0] = -std::numeric_limits<double>::infinity();
            adj->total[1] = adj->total[2] = std::numeric_limits<double>::quiet_NaN();
        }
        return;
    }
    const uint32_t bins = p.num_curvature_steps;
    cudaStream_t st = ctx->stream;

    struct ExpHost {
        uint32_t N;
        float ds;
        CompTuning t;
        ChainSpec spec;
        uint32_t seg_off, chain_off;
        double log10_norm;
        LutMetaF meta;
        uint32_t multi_index;
    };
    std::vector<ExpHost> eh(n);
    std::vector<LutBuildSpec> specs(n);
    std::vector<float> steps(n);
    std::vector<uint32_t> nsegs(n);
    uint32_t total_chains = 0;
    uint32_t n_seg_floats = 0;
    for (uint32_t e = 0; e < n; ++e) {
        const twisty_experiment &x = ex[e];
        ExpHost &h = eh[e];
        const uint32_t N = x.num_segments;
        if (N < 4 || N > 1024) fail(TWISTY_ERR_INVALID_CONFIG, exp_msg(e, "numSegments must be in [4, 1024]"));
        try {
            validate_bc(&x.bc);
        } catch (const Failure &f) {
            fail(f.s, exp_msg(e, f.msg));
        }
        if (!(x.eps > 0.0f)) fail(TWISTY_ERR_INVALID_CONFIG, exp_msg(e, "eps must be positive"));
        if (!(x.scatter >= 0.0f)) fail(TWISTY_ERR_INVALID_CONFIG, exp_msg(e, "scatter must be non-negative"));
        h.N = N;
        h.ds = x.bc.arclength / (float)N;
        // the table of WeightLookupTableIntegral for this ds (PathWeightUtils.cpp:281-289),
        // maxBound = 10/eps per experiment (ExperimentRunner.cpp:169-171)
        const float max_k = (float)((2.0 / (double)h.ds) * (double)1.01f);
        h.meta = LutMetaF{0.0f, max_k, max_k / (float)(bins - 1), (int32_t)bins};
        if (multi) {
            if (x.eps != p.eps || x.scatter != p.scatter)
                fail(TWISTY_ERR_LUT_INVALID, exp_msg(e, "lut_mode MULTI_DS needs the set's eps and scatter"));
            h.multi_index = multi_closest(ctx, h.ds);
            h.meta = ctx->multi.meta[h.multi_index];
        }
        LutBuildSpec &ls = specs[e];
        ls = LutBuildSpec{};
        ls.mu = p.mu;
        ls.eps = x.eps;
        ls.scatter = x.scatter;
        ls.min_bound = p.min_bound;
        ls.max_bound = 10.0f / x.eps;
        ls.bias = p.bias;
        ls.num_steps_int = p.num_steps_int;
        ls.bins = bins;
        ls.ds = h.ds;
        ls.min_k = 0.0f;
        ls.step = h.meta.step;
        ls.step64 = ((2.0 / (double)h.ds) * 1.01) / (double)(bins - 1);
        steps[e] = h.meta.step;
        nsegs[e] = N;
        // the initial curve's segment vectors go to segs[seg_off .. seg_off + 3N) (below)
        h.seg_off = n_seg_floats;
        n_seg_floats += 3 * N;
        // kernel shape and chain layout: whole CTAs of chains, ~2048 steps per chain
        h.t = comp_default_tuning(N, true);
        {
            // a tuned shape the batched kernel does not have keeps the default
            CompTuning tuned = h.t;
            if (tune_lookup(ctx->device_name, N, bins, tuned)) {
                const int w = std::min(tuned.warps_per_block, batch_max_threads(tuned.group, tuned.spl) / 32);
                if (batch_shape_supported(BatchShape{tuned.group, tuned.spl, w, 0, 1, 0, 0}, N, 2)) h.t = tuned;
            }
        }
        ChainSpec &c = h.spec;
        c = ChainSpec{};
        c.n_segments = N;
        c.arclength = x.bc.arclength;
        c.ds = h.ds;
        c.inv_ds = (float)N / x.bc.arclength;
        c.seed = seed_of(p.perturb_seed);
        c.experiment = p.experiment_id + e;
        c.chain0 = p.chain_offset;
        c.burn_in = (uint32_t)std::min<uint64_t>(p.paths_to_skip, 0xFFFFFFFFull);
        c.k_eff = std::min<uint32_t>(p.max_sub_chain, N - 2);
        c.max_angle = p.max_angle;
        c.absorption_factor = (double)std::exp(-p.absorption * h.ds);
        if (!comp_tuning_supported(h.t, N, c.k_eff))
            fail(TWISTY_ERR_UNSUPPORTED, exp_msg(e, "no compensated kernel shape for this N / max_sub_chain"));
        const int maxt = batch_max_threads(h.t.group, h.t.spl);
        h.t.warps_per_block = std::min(h.t.warps_per_block, maxt / 32);
        {
            // a staged table may take the shape down to comp_stage_min_warps; below that the
            // table is gathered through L1 at the shape's full warps
            const int floor_w = comp_stage_min_warps(h.t);
            auto staged_fits = [&](int w) {
                return batch_smem_bytes(BatchShape{h.t.group, h.t.spl, w, 0, 1, 0, 1}, bins) <= kSmemCap;
            };
            int w = h.t.warps_per_block;
            while (w - 4 >= floor_w && !staged_fits(w)) w -= 4;
            if (staged_fits(w)) h.t.warps_per_block = w;
        }
        const uint64_t cpb = (uint64_t)h.t.warps_per_block * (32u / (uint32_t)h.t.group);
        uint64_t chains = p.num_chains;
        if (!chains) chains = cpb * std::max<uint64_t>(1, (x.paths + cpb * 1024) / (cpb * 2048));
        if (x.paths == 0) {
            c.n_chains = 0;
        } else {
            chains = std::min<uint64_t>(chains, x.paths);
            const uint64_t L = (x.paths + chains - 1) / chains;
            if (L > 0xFFFFFFFFull - c.burn_in) fail(TWISTY_ERR_INVALID_CONFIG, exp_msg(e, "too many paths per chain"));
            chains = (x.paths + L - 1) / L;
            c.n_chains = (uint32_t)chains;
            c.steps = (uint32_t)L;
            c.last_steps = (uint32_t)(x.paths - (chains - 1) * L);
        }
        h.chain_off = total_chains;
        if ((uint64_t)total_chains + c.n_chains > 0xFFFFFFFFull) fail(TWISTY_ERR_INVALID_CONFIG, "too many chains in the batch");
        total_chains += c.n_chains;
    }

    BatchBufs &B = ctx->batch;
    // ---- tables, all experiments at once (launched before the host builds the curves)
    ck(B.init_seg.ensure(sizeof(float) * std::max<uint32_t>(1, n_seg_floats)), "alloc batch curves");
    ck(B.specs.ensure(sizeof(LutBuildSpec) * n), "alloc batch");
    ck(B.lut64.ensure(sizeof(double) * (size_t)bins * n), "alloc batch tables");
    ck(B.lut32.ensure(sizeof(float) * (size_t)bins * n), "alloc batch tables");
    ck(B.fix.ensure(sizeof(float2) * (size_t)bins * n), "alloc batch tables");
    ck(B.lin.ensure(sizeof(float2) * (size_t)bins * n), "alloc batch tables");
    ck(B.steps.ensure(sizeof(float) * n), "alloc batch");
    ck(B.nsegs.ensure(sizeof(uint32_t) * n), "alloc batch");
    ck(B.lf.ensure(sizeof(LogFixed) * n), "alloc batch");
    ck(B.ok.ensure(sizeof(int) * n), "alloc batch");
    ck(cudaMemcpyAsync(B.specs.p, specs.data(), sizeof(LutBuildSpec) * n, cudaMemcpyHostToDevice, st), "upload specs");
    ck(cudaMemcpyAsync(B.steps.p, steps.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st), "upload");
    ck(cudaMemcpyAsync(B.nsegs.p, nsegs.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st), "upload");
    if (multi) {
        for (uint32_t e = 0; e < n; ++e)
            ck(cudaMemcpyAsync(B.lut32.as<float>() + (size_t)e * bins, ctx->multi.dev.as<float>() + (size_t)eh[e].multi_index * bins,
                               sizeof(float) * bins, cudaMemcpyDeviceToDevice, st),
               "multi-ds table");
    } else {
        ck(launch_lut_build_batch(B.specs.as<LutBuildSpec>(), n, bins, B.lut64.as<double>(), st), "batch table build");
        ck(launch_lut_finalize_batch(n, bins, B.lut64.as<double>(), B.lut32.as<float>(), nullptr, st),
           "batch table finalize");
    }
    ck(launch_comp_tables_batch(n, bins, B.lut32.as<float>(), B.steps.as<float>(), B.nsegs.as<uint32_t>(),
                                B.fix.as<float2>(), B.lin.as<float2>(), B.lf.as<LogFixed>(), B.ok.as<int>(), st),
       "batch compensated tables");
    // ---- initial curves on host threads while the device builds the tables
    std::vector<float> segs(n_seg_floats);
    {
        std::atomic<uint32_t> next{0};
        std::atomic<bool> failed{false};
        std::mutex err_mu;
        uint32_t err_exp = n;
        std::string err_msg;
        auto work = [&] {
            std::vector<float> pos;
            std::string err;
            for (;;) {
                const uint32_t e = next.fetch_add(1);
                if (e >= n || failed.load()) return;
                const uint32_t N = eh[e].N;
                if (!bootstrap_curve(ex[e].bc, N, p.bootstrap_seed + e, p.bootstrap_kind, pos, err)) {
                    std::lock_guard<std::mutex> lk(err_mu);
                    if (e < err_exp) { err_exp = e; err_msg = err; }
                    failed.store(true);
                    return;
                }
                float *dst = segs.data() + eh[e].seg_off;
                for (uint32_t i = 0; i < N; ++i)
                    for (int k = 0; k < 3; ++k) dst[3 * i + k] = pos[3 * (i + 1) + k] - pos[3 * i + k];
            }
        };
        const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
        const uint32_t nt = std::min<uint32_t>(std::min<uint32_t>(hw, 32u), std::max<uint32_t>(1, n / 16));
        std::vector<std::thread> pool;
        for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (std::thread &t : pool) t.join();
        if (failed.load()) fail(TWISTY_ERR_INFEASIBLE_GEOMETRY, exp_msg(err_exp, err_msg));
    }
    for (uint32_t e = 0; e < n; ++e) eh[e].log10_norm = normalizer_log10(ctx, eh[e].N, eh[e].ds, ex[e].bc);
    std::vector<LogFixed> lf(n);
    std::vector<int> okv(n);
    ck(cudaMemcpyAsync(B.init_seg.p, segs.data(), sizeof(float) * segs.size(), cudaMemcpyHostToDevice, st), "upload curves");
    ck(cudaMemcpyAsync(lf.data(), B.lf.p, sizeof(LogFixed) * n, cudaMemcpyDeviceToHost, st), "read tables");
    ck(cudaMemcpyAsync(okv.data(), B.ok.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st), "read tables");
    ck(cudaStreamSynchronize(st), "batch tables");

    // ---- experiments packed for the device, buckets by shape and table form
    std::vector<BatchExpHost> bh(n);
    struct Bucket {
        BatchShape shape;
        std::vector<uint32_t> exps;
        std::vector<uint2> items;
        int grid = 0;
        uint32_t item_off = 0;
    };
    std::vector<Bucket> buckets;
    auto bucket_of = [&](const BatchShape &sh) -> Bucket & {
        for (Bucket &b : buckets)
            if (b.shape.group == sh.group && b.shape.spl == sh.spl && b.shape.warps == sh.warps && b.shape.exact == sh.exact &&
                b.shape.clamp == sh.clamp && b.shape.lut_smem == sh.lut_smem && b.shape.steep == sh.steep)
                return b;
        buckets.push_back(Bucket{});
        buckets.back().shape = sh;
        return buckets.back();
    };
    for (uint32_t e = 0; e < n; ++e) {
        ExpHost &h = eh[e];
        // Fixed-point tables staged in shared memory all take the kernel with the steep-bin
        // fallback (whether or not this table has steep bins: one bucket per shape balances
        // better than two, measured 5 % faster on the batching workload); a table that does
        // not fit in shared memory takes the plain fixed-point kernel, or the exact blend
        // when it has steep bins.
        const bool smem_fits = batch_smem_bytes(BatchShape{h.t.group, h.t.spl, h.t.warps_per_block, 0, 1, 0, 1}, bins) <=
                               227 * 1024;
        const bool exact = okv[e] == 0 || (lf[e].steep > 0 && !smem_fits);
        const bool steep = !exact && smem_fits;
        BatchExpHost &b = bh[e];
        b.spec = h.spec;
        b.meta = h.meta;
        b.lf = exact ? LogFixed{0.0, 0.0, 0, 0} : lf[e];
        b.tab = (exact ? B.lin.as<float2>() : B.fix.as<float2>()) + (size_t)e * bins;
        b.lin = B.lin.as<float2>() + (size_t)e * bins;
        b.init_seg = B.init_seg.as<float>() + h.seg_off;
        b.out_offset = h.chain_off;
        BatchShape sh{h.t.group, h.t.spl, h.t.warps_per_block, exact ? 1 : 0, 1,
                      (exact || comp_table_needs_clamp(h.spec.inv_ds, h.meta)) ? 1 : 0, steep ? 1 : 0};
        if (batch_smem_bytes(sh, bins) > 227 * 1024) sh.lut_smem = 0;
        if (!batch_shape_supported(sh, h.N, h.spec.k_eff) || batch_smem_bytes(sh, bins) > 227 * 1024)
            fail(TWISTY_ERR_UNSUPPORTED, exp_msg(e, "no batched kernel shape fits"));
        Bucket &bk = bucket_of(sh);
        bk.exps.push_back(e);
        const uint32_t cpb = (uint32_t)batch_chains_per_block(sh);
        for (uint32_t c0 = 0; c0 < h.spec.n_chains; c0 += cpb) bk.items.push_back(make_uint2(e, c0));
    }
    std::vector<uint2> items;
    for (Bucket &bk : buckets) {
        // longest work first: cost of an item ~ (burn-in + steps) x N
        std::stable_sort(bk.items.begin(), bk.items.end(), [&](const uint2 &a, const uint2 &b) {
            const ExpHost &x = eh[a.x], &y = eh[b.x];
            return (double)(x.spec.burn_in + x.spec.steps) * x.N > (double)(y.spec.burn_in + y.spec.steps) * y.N;
        });
        bk.item_off = (uint32_t)items.size();
        items.insert(items.end(), bk.items.begin(), bk.items.end());
        const int occ = batch_blocks_per_sm(bk.shape, (int)bins);
        if (occ <= 0) fail(TWISTY_ERR_UNSUPPORTED, "batched kernel shape cannot launch");
        bk.grid = (int)std::min<uint64_t>((uint64_t)ctx->sm_count * occ, std::max<size_t>(1, bk.items.size()));
    }
    std::vector<unsigned char> packed(batch_exp_bytes() * n);
    batch_pack_experiments(bh.data(), n, packed.data());
    std::vector<uint2> ranges(n);
    for (uint32_t e = 0; e < n; ++e) ranges[e] = make_uint2(eh[e].chain_off, eh[e].spec.n_chains);
    ck(B.exps.ensure(packed.size()), "alloc batch");
    ck(B.items.ensure(sizeof(uint2) * std::max<size_t>(1, items.size())), "alloc batch");
    ck(B.counters.ensure(sizeof(uint32_t) * buckets.size()), "alloc batch");
    ck(B.chain_out.ensure(sizeof(ChainOut) * std::max<uint32_t>(1, total_chains)), "alloc batch results");
    ck(B.ranges.ensure(sizeof(uint2) * n), "alloc batch");
    ck(B.red.ensure(sizeof(ReduceOut) * n), "alloc batch results");
    ck(cudaMemcpyAsync(B.exps.p, packed.data(), packed.size(), cudaMemcpyHostToDevice, st), "upload batch");
    if (!items.empty())
        ck(cudaMemcpyAsync(B.items.p, items.data(), sizeof(uint2) * items.size(), cudaMemcpyHostToDevice, st), "upload batch");
    ck(cudaMemcpyAsync(B.ranges.p, ranges.data(), sizeof(uint2) * n, cudaMemcpyHostToDevice, st), "upload batch");
    ck(cudaStreamSynchronize(st), "batch upload");

    // ---- the pass as a graph: counters reset, one launch per bucket on forked streams, reduction;
    // captured again only when the buckets, grids or buffers differ from the previous call's
    std::vector<uint64_t> key = {(uint64_t)n, (uint64_t)bins, (uint64_t)(uintptr_t)B.exps.p, (uint64_t)(uintptr_t)B.items.p,
                                 (uint64_t)(uintptr_t)B.counters.p, (uint64_t)(uintptr_t)B.chain_out.p,
                                 (uint64_t)(uintptr_t)B.ranges.p, (uint64_t)(uintptr_t)B.red.p};
    for (const Bucket &bk : buckets) {
        key.push_back(((uint64_t)bk.shape.group << 48) | ((uint64_t)bk.shape.spl << 40) | ((uint64_t)bk.shape.warps << 32) |
                      ((uint64_t)bk.shape.exact << 4) | ((uint64_t)bk.shape.lut_smem << 3) |
                      ((uint64_t)bk.shape.clamp << 2) | ((uint64_t)bk.shape.steep << 1));
        key.push_back(((uint64_t)bk.grid << 32) | bk.item_off);
        key.push_back(bk.items.size());
    }
    BatchGraph &G = ctx->batch_graph;
    if (!G.exec || G.key != key) {
        G.release();
        G.streams.resize(buckets.size(), nullptr);
        G.events.resize(buckets.size() + 3, nullptr);
        for (auto &x : G.streams) ck(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking), "stream");
        for (auto &x : G.events) ck(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), "event");
        cudaEvent_t fork = G.events[buckets.size()];
        ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "capture");
        {
            cudaError_t ce = cudaMemsetAsync(B.counters.p, 0, sizeof(uint32_t) * buckets.size(), st);
            if (ce == cudaSuccess) ce = cudaEventRecord(fork, st);
            for (size_t b = 0; b < buckets.size() && ce == cudaSuccess; ++b) {
                const Bucket &bk = buckets[b];
                ce = cudaStreamWaitEvent(G.streams[b], fork, 0);
                if (ce == cudaSuccess)
                    ce = launch_batch(bk.shape, B.exps.p, B.items.as<uint2>() + bk.item_off, (uint32_t)bk.items.size(),
                                      B.counters.as<uint32_t>() + b, B.chain_out.as<ChainOut>(), (int)bins, bk.grid,
                                      G.streams[b]);
                if (ce == cudaSuccess) ce = cudaEventRecord(G.events[b], G.streams[b]);
                if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, G.events[b], 0);
            }
            if (ce == cudaSuccess) ce = launch_reduce_segments(B.chain_out.as<ChainOut>(), B.ranges.as<uint2>(), n,
                                                               B.red.as<ReduceOut>(), st);
            const cudaError_t ee = cudaStreamEndCapture(st, &G.graph);
            if (ce != cudaSuccess || ee != cudaSuccess) G.release();
            ck(ce, "batched pass capture");
            ck(ee, "end capture");
        }
        const cudaError_t ie = cudaGraphInstantiate(&G.exec, G.graph, 0);
        if (ie != cudaSuccess) G.release();
        ck(ie, "graph instantiate");
        G.key = key;
    }
    const double setup_ms = now_ms() - t0;
    ctx->kernels_per_launch = (uint32_t)buckets.size() + 1;   // one persistent launch per bucket + the reduction

    // ---- replays, each timed on the stream
    double sum_ms = 0.0;
    for (uint32_t it = 0; it < iters; ++it) {
        ck(cudaEventRecord(ctx->ev[0], st), "event");
        ck(cudaGraphLaunch(G.exec, st), "graph launch");
        ck(cudaEventRecord(ctx->ev[1], st), "event");
        ck(cudaEventSynchronize(ctx->ev[1]), "batched pass");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]), "event time");
        sum_ms += ms;
    }
    std::vector<ReduceOut> red(n);
    ck(cudaMemcpyAsync(red.data(), B.red.p, sizeof(ReduceOut) * n, cudaMemcpyDeviceToHost, st), "read batch results");
    ck(cudaStreamSynchronize(st), "read batch results");
    const double total_ms = now_ms() - t0;
    for (uint32_t e = 0; e < n; ++e) {
        twisty_result &r = res[e];
        const ReduceOut &o = red[e];
        r.log10_normalizer = eh[e].log10_norm;
        r.log10_weight = o.log10_sum + eh[e].log10_norm;
        r.total_paths = o.valid;
        r.failed_paths = o.failed;
        r.clamped_curvatures = o.clamped;
        r.log10_mean_weight = o.valid ? r.log10_weight - std::log10((double)o.valid) : -std::numeric_limits<double>::infinity();
        r.rel_std_error = o.rel_se;
        r.num_chains = eh[e].spec.n_chains;
        r.steps_per_chain = eh[e].spec.steps;
        r.setup_ms = setup_ms;
        const bool fixed = bh[e].lf.inv_scale != 0.0;
        r.table_form = fixed ? (lf[e].wide ? TWISTY_TABLE_FIXED_WIDE : TWISTY_TABLE_FIXED_NARROW) : TWISTY_TABLE_EXACT_BLEND;
        r.steep_bins = fixed ? (uint32_t)lf[e].steep : 0u;
        r.kernel_shape = ((uint32_t)eh[e].t.group << 8) | (uint32_t)eh[e].t.spl;
        // the device-built tables keep every secant within 1e-7 (steeper bins are re-weighed exactly)
        r.weight_error_bound = (double)(eh[e].N - 1) * (fixed ? bh[e].lf.inv_scale + 1e-7 : 4e-7);
        r.fp64_rel_error = std::numeric_limits<double>::quiet_NaN();
        r.perturb_ms = sum_ms / iters;
        r.weighting_ms = 0.0;
        r.total_ms = total_ms;
    }
    if (!adj) return;

    // ---- adjoint replay of the same chains (twisty_adjoint_batch)
    // derivative tables d/d(mu_s), d/d(eps) in FP64 on the device: one per experiment, or one per
    // table of the multi-ds set the experiments take theirs from
    const uint32_t ntab = multi ? ctx->multi.n : n;
    ck(B.dtab.ensure(sizeof(float4) * (size_t)bins * ntab), "alloc derivative tables");
    ck(B.d64mu.ensure(sizeof(double) * (size_t)bins * ntab), "alloc derivative tables");
    ck(B.d64eps.ensure(sizeof(double) * (size_t)bins * ntab), "alloc derivative tables");
    ck(B.d64scratch.ensure(sizeof(double) * (size_t)bins), "alloc derivative tables");
    std::vector<char> tab_used(ntab, multi ? 0 : 1);
    if (multi)
        for (uint32_t e = 0; e < n; ++e) tab_used[eh[e].multi_index] = 1;
    ck(cudaEventRecord(ctx->ev[0], st), "event");
    for (uint32_t t = 0; t < ntab; ++t) {
        if (!tab_used[t]) continue;
        LutBuildSpec s{};
        if (multi) {
            s.mu = p.mu;
            s.eps = p.eps;
            s.scatter = p.scatter;
            s.min_bound = p.min_bound;
            s.max_bound = p.max_bound;
            s.bias = p.bias;
            s.num_steps_int = p.num_steps_int;
            s.bins = bins;
            s.ds = ctx->multi.ds[t];
            s.min_k = 0.0f;
            s.step = ctx->multi.meta[t].step;
            s.step64 = ((2.0 / (double)s.ds) * 1.01) / (double)(bins - 1);
        } else {
            s = specs[t];
        }
        s.faithful = 0;
        s.derivatives = 1;
        ck(launch_lut_build(s, B.d64scratch.as<double>(), B.d64mu.as<double>() + (size_t)t * bins,
                            B.d64eps.as<double>() + (size_t)t * bins, st),
           "derivative tables");
    }
    ck(launch_deriv_tables(B.d64mu.as<double>(), B.d64eps.as<double>(), bins, ntab, B.dtab.as<float4>(), st),
       "derivative tables");
    ck(cudaEventRecord(ctx->ev[1], st), "event");

    // experiments for the replay: the linear table staged in shared memory, the exact blend
    std::vector<BatchExpHost> bx(n);
    std::vector<BatchAdjHost> ax(n);
    struct AdjBucket {
        BatchShape shape;
        std::vector<uint2> items;
        int grid = 0;
        uint32_t item_off = 0;
    };
    std::vector<AdjBucket> abk;
    for (uint32_t e = 0; e < n; ++e) {
        const ExpHost &h = eh[e];
        bx[e] = bh[e];
        bx[e].lf = LogFixed{0.0, 0.0, 0, 0};
        bx[e].tab = B.lin.as<float2>() + (size_t)e * bins;
        const uint32_t t = multi ? h.multi_index : e;
        const double log10_abs = std::log10(h.spec.absorption_factor);
        const bool ok = red[e].valid > 0 && std::isfinite(red[e].log10_sum);
        ax[e] = BatchAdjHost{B.dtab.as<float4>() + (size_t)t * bins,
                             ok ? (float)(red[e].log10_sum - (double)(h.N - 1) * log10_abs) : 0.0f};
        if (h.spec.n_chains == 0) continue;
        BatchShape sh{h.t.group, h.t.spl, std::min(h.t.warps_per_block, batch_max_threads(h.t.group, h.t.spl) / 32), 1, 1,
                      1, 0};
        while (sh.warps > 4 && batch_smem_bytes(sh, bins) > kSmemCap) sh.warps -= 4;
        if (batch_smem_bytes(sh, bins) > kSmemCap)
            fail(TWISTY_ERR_UNSUPPORTED, exp_msg(e, "weight table too large to stage for the adjoint"));
        AdjBucket *bk = nullptr;
        for (AdjBucket &b : abk)
            if (b.shape.group == sh.group && b.shape.spl == sh.spl && b.shape.warps == sh.warps) bk = &b;
        if (!bk) {
            abk.push_back(AdjBucket{});
            abk.back().shape = sh;
            bk = &abk.back();
        }
        const uint32_t cpb = (uint32_t)batch_chains_per_block(sh);
        for (uint32_t c0 = 0; c0 < h.spec.n_chains; c0 += cpb) bk->items.push_back(make_uint2(e, c0));
    }
    std::vector<uint2> aitems;
    for (AdjBucket &bk : abk) {
        std::stable_sort(bk.items.begin(), bk.items.end(), [&](const uint2 &a, const uint2 &b) {
            const ExpHost &x = eh[a.x], &y = eh[b.x];
            return (double)(x.spec.burn_in + x.spec.steps) * x.N > (double)(y.spec.burn_in + y.spec.steps) * y.N;
        });
        bk.item_off = (uint32_t)aitems.size();
        aitems.insert(aitems.end(), bk.items.begin(), bk.items.end());
        const int occ = batch_adjoint_blocks_per_sm(bk.shape, (int)bins);
        if (occ <= 0) fail(TWISTY_ERR_UNSUPPORTED, "batched adjoint shape cannot launch");
        bk.grid = (int)std::min<uint64_t>((uint64_t)ctx->sm_count * occ, std::max<size_t>(1, bk.items.size()));
    }
    std::vector<unsigned char> pexp(batch_exp_bytes() * n), padj(batch_adj_bytes() * n);
    batch_pack_experiments(bx.data(), n, pexp.data());
    batch_pack_adjoint(ax.data(), n, padj.data());
    ck(B.adj_exps.ensure(pexp.size()), "alloc adjoint");
    ck(B.adj_aux.ensure(padj.size()), "alloc adjoint");
    ck(B.adj_items.ensure(sizeof(uint2) * std::max<size_t>(1, aitems.size())), "alloc adjoint");
    ck(B.adj_counters.ensure(sizeof(uint32_t) * std::max<size_t>(1, abk.size())), "alloc adjoint");
    ck(B.grad.ensure(sizeof(double) * 6 * std::max<uint32_t>(1, total_chains)), "alloc adjoint");
    ck(B.grad_sum.ensure(sizeof(double) * 6 * n), "alloc adjoint");
    ck(cudaMemcpyAsync(B.adj_exps.p, pexp.data(), pexp.size(), cudaMemcpyHostToDevice, st), "upload adjoint");
    ck(cudaMemcpyAsync(B.adj_aux.p, padj.data(), padj.size(), cudaMemcpyHostToDevice, st), "upload adjoint");
    if (!aitems.empty())
        ck(cudaMemcpyAsync(B.adj_items.p, aitems.data(), sizeof(uint2) * aitems.size(), cudaMemcpyHostToDevice, st),
           "upload adjoint");
    ck(cudaMemsetAsync(B.adj_counters.p, 0, sizeof(uint32_t) * std::max<size_t>(1, abk.size()), st), "memset");
    ck(cudaMemsetAsync(B.grad.p, 0, sizeof(double) * 6 * std::max<uint32_t>(1, total_chains), st), "memset");
    ck(cudaEventRecord(ctx->ev[2], st), "event");
    for (size_t b = 0; b < abk.size(); ++b)
        ck(launch_batch_adjoint(abk[b].shape, B.adj_exps.p, B.adj_aux.p, B.adj_items.as<uint2>() + abk[b].item_off,
                                (uint32_t)abk[b].items.size(), B.adj_counters.as<uint32_t>() + b, B.grad.as<double>(),
                                (int)bins, abk[b].grid, st),
           "batched adjoint kernel");
    ck(launch_grad_reduce_segments(B.grad.as<double>(), B.ranges.as<uint2>(), n, B.grad_sum.as<double>(), st),
       "adjoint reduction");
    ck(cudaEventRecord(ctx->ev[3], st), "event");
    std::vector<double> gs(6 * (size_t)n);
    ck(cudaMemcpyAsync(gs.data(), B.grad_sum.p, sizeof(double) * gs.size(), cudaMemcpyDeviceToHost, st), "read gradients");
    ck(cudaStreamSynchronize(st), "batched adjoint");
    float t_tab = 0.f, t_rep = 0.f;
    ck(cudaEventElapsedTime(&t_tab, ctx->ev[0], ctx->ev[1]), "event time");
    ck(cudaEventElapsedTime(&t_rep, ctx->ev[2], ctx->ev[3]), "event time");
    ctx->kernels_per_launch = (uint32_t)abk.size() + 1;
    // per experiment: the weight-averaged path gradients; d/d(sigma) = d/d(eps) 2 sigma
    double m = -std::numeric_limits<double>::infinity();
    for (uint32_t e = 0; e < n; ++e)
        if (res[e].total_paths && std::isfinite(res[e].log10_weight)) m = std::max(m, res[e].log10_weight);
    double wsum = 0.0, tmu = 0.0, tsig = 0.0;
    for (uint32_t e = 0; e < n; ++e) {
        const double *g = gs.data() + 6 * (size_t)e;
        double *o = adj->grad + 5 * (size_t)e;
        if (!(g[5] > 0.0)) {
            for (int k = 0; k < 5; ++k) o[k] = std::numeric_limits<double>::quiet_NaN();
            continue;
        }
        const double sigma = std::sqrt((double)ex[e].eps);
        o[0] = g[0] / g[5];
        o[1] = g[1] / g[5] * 2.0 * sigma;
        o[2] = g[2] / g[5];
        o[3] = g[3] / g[5];
        o[4] = g[4] / g[5];
        const double w = std::pow(10.0, res[e].log10_weight - m);
        wsum += w;
        tmu += w * o[0];
        tsig += w * o[1];
    }
    if (adj->total) {
        adj->total[0] = wsum > 0.0 ? m + std::log10(wsum) : -std::numeric_limits<double>::infinity();
        adj->total[1] = wsum > 0.0 ? tmu / wsum : std::numeric_limits<double>::quiet_NaN();
        adj->total[2] = wsum > 0.0 ? tsig / wsum : std::numeric_limits<double>::quiet_NaN();
    }
    if (adj->timing) {
        adj->timing[0] = t_tab;
        adj->timing[1] = t_rep;
    }
}

}  // namespace

twisty_status twisty_run_batch(twisty_ctx *ctx, const twisty_experiment *ex, uint32_t n, uint32_t iterations,
                               twisty_result *res)
{
    if (!ctx || (!ex && n) || (!res && n)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] { run_batch(ctx, ex, n, iterations ? iterations : 1, res); });
}

twisty_status twisty_adjoint_batch(twisty_ctx *ctx, const twisty_experiment *ex, uint32_t n, twisty_result *res,
                                   double *grad, double total[3], double timing_ms[2])
{
    if (!ctx || (!ex && n) || (!res && n) || (!grad && n)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (ctx->p.lut_mode != TWISTY_LUT_FP64 && ctx->p.lut_mode != TWISTY_LUT_MULTI_DS)
            fail(TWISTY_ERR_UNSUPPORTED, "the batched adjoint builds its derivative tables in FP64 (lut_mode FP64 or MULTI_DS)");
        const BatchAdjointOut out{grad, total, timing_ms};
        run_batch(ctx, ex, n, 1, res, &out);
    });
}

twisty_status twisty_export_paths(twisty_ctx *ctx, const twisty_bc *bc, const char *dir, uint64_t max_paths, float *pos,
                                  double *log10w, uint64_t *n_written, twisty_result *res)
{
    if (!ctx || !bc) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        const double t0 = now_ms();
        prepare(ctx, bc);
        launch(ctx, ctx->stream);
        twisty_result r{};
        collect(ctx, &r);
        const ChainSpec &c = ctx->spec;
        const uint32_t N = c.n_segments;
        std::vector<float> hpos;
        std::vector<double> hw;
        std::vector<uint32_t> chain_of;
        if (max_paths > 0 && c.n_chains > 0) {
            // replay the first E chains with every weighted path written out
            const uint64_t E64 = std::min<uint64_t>(c.n_chains, (max_paths + c.steps - 1) / c.steps);
            const uint32_t E = (uint32_t)E64;
            ChainSpec ce = c;
            ce.n_chains = E;
            ce.last_steps = (E == c.n_chains) ? c.last_steps : c.steps;
            const size_t npaths = (size_t)E * c.steps;
            DevBuf dpos, dw, dout;
            try {
                ck(dpos.ensure(sizeof(float) * 3 * (size_t)(N + 1) * npaths), "alloc export buffer");
                ck(dw.ensure(sizeof(double) * npaths), "alloc export buffer");
                ck(dout.ensure(sizeof(ChainOut) * E), "alloc export buffer");
                ck(cudaMemsetAsync(dw.p, 0xff, sizeof(double) * npaths, ctx->stream), "memset");  // NaN: not written
                if (ctx->p.form == TWISTY_FORM_PLAIN_FP32) {
                    ck(launch_plain_chains(ce, ctx->init_pos.as<float>(), ctx->state.as<float>(), ctx->lut32.as<float>(),
                                           ctx->meta, dout.as<ChainOut>(), ctx->stream, dpos.as<float>(), dw.as<double>()),
                       "export replay");
                } else if (ctx->p.form == TWISTY_FORM_COMPENSATED) {
                    if (ce.has_eval_shift) fail(TWISTY_ERR_UNSUPPORTED, "eval_end_shift applies to forward passes of the compensated form only");
                    const float x0[3] = {bc->start_pos.x, bc->start_pos.y, bc->start_pos.z};
                    ck(launch_comp_export(ce, staged_tuning(ctx), ctx->init_seg.as<float>(), ctx->fixtab.as<float2>(),
                                          ctx->lintab.as<float2>(), ctx->meta, x0, dpos.as<float>(), dw.as<double>(),
                                          dout.as<ChainOut>(), ctx->stream, ctx->lf),
                       "export replay");
                } else {
                    fail(TWISTY_ERR_UNSUPPORTED, "path export runs the plain and compensated forms");
                }
                std::vector<float> apos(3 * (size_t)(N + 1) * npaths);
                std::vector<double> aw(npaths);
                ck(cudaMemcpyAsync(apos.data(), dpos.p, sizeof(float) * apos.size(), cudaMemcpyDeviceToHost, ctx->stream), "read export");
                ck(cudaMemcpyAsync(aw.data(), dw.p, sizeof(double) * npaths, cudaMemcpyDeviceToHost, ctx->stream), "read export");
                ck(cudaStreamSynchronize(ctx->stream), "export");
                // invalid paths are skipped, as the reference skips them before exporting
                for (uint32_t ch = 0; ch < E && hw.size() < max_paths; ++ch) {
                    const uint32_t steps = (ch == c.n_chains - 1) ? c.last_steps : c.steps;
                    for (uint32_t s = 0; s < steps && hw.size() < max_paths; ++s) {
                        const size_t i = (size_t)ch * c.steps + s;
                        if (!std::isfinite(aw[i])) continue;
                        hw.push_back(aw[i]);
                        chain_of.push_back(ch);
                        hpos.insert(hpos.end(), apos.begin() + i * 3 * (N + 1), apos.begin() + (i + 1) * 3 * (N + 1));
                    }
                }
            } catch (...) {
                dpos.release(); dw.release(); dout.release();
                throw;
            }
            dpos.release(); dw.release(); dout.release();
        }
        const uint64_t n = hw.size();
        if (pos && n) std::memcpy(pos, hpos.data(), sizeof(float) * hpos.size());
        if (log10w && n) std::memcpy(log10w, hw.data(), sizeof(double) * n);
        if (n_written) *n_written = n;
        if (dir) write_path_batch(dir, *bc, N, ctx->log10_norm, hpos, hw, chain_of);
        r.total_ms = now_ms() - t0;
        if (res) *res = r;
    });
}

twisty_status twisty_adjoint(twisty_ctx *ctx, const twisty_bc *bc, const twisty_result *fwd, double grad[5])
{
    if (!ctx || !bc || !fwd || !grad) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (ctx->p.form != TWISTY_FORM_COMPENSATED) fail(TWISTY_ERR_UNSUPPORTED, "the adjoint replays the compensated form");
        if (ctx->p.lut_mode != TWISTY_LUT_FP64) fail(TWISTY_ERR_UNSUPPORTED, "the adjoint needs lut_mode FP64 (derivative tables)");
        const twisty_vec3 &sh = ctx->p.eval_end_shift;
        if (sh.x != 0.f || sh.y != 0.f || sh.z != 0.f) fail(TWISTY_ERR_UNSUPPORTED, "eval_end_shift applies to forward passes only");
        prepare(ctx, bc);
        const uint32_t N = ctx->p.num_segments;
        const float ds = bc->arclength / (float)N;
        build_tables(ctx, ds, true);
        const uint32_t bins = ctx->p.num_curvature_steps;
        const ChainSpec &c = ctx->spec;
        DevBuf dtab, dg, dout;
        try {
            ck(dtab.ensure(sizeof(float4) * bins), "alloc");
            ck(dg.ensure(sizeof(double) * 6 * std::max<uint32_t>(c.n_chains, 1)), "alloc");
            ck(dout.ensure(sizeof(double) * 6), "alloc");
            ck(launch_deriv_tables(ctx->dmus.as<double>(), ctx->deps.as<double>(), bins, 1, dtab.as<float4>(), ctx->stream),
               "derivative tables");
            const double ref = fwd->log10_weight - fwd->log10_normalizer - (double)(N - 1) * std::log10(c.absorption_factor);
            CompTuning t = staged_tuning(ctx);
            t.exact_blend = 1;
            ck(launch_comp_adjoint(c, t, ctx->init_seg.as<float>(), ctx->lintab.as<float2>(), ctx->meta,
                                   dtab.as<float4>(), (float)ref, dg.as<double>(), dout.as<double>(), ctx->stream),
               "adjoint kernel");
            double g[6];
            ck(cudaMemcpyAsync(g, dout.p, sizeof(g), cudaMemcpyDeviceToHost, ctx->stream), "read gradient");
            ck(cudaStreamSynchronize(ctx->stream), "adjoint");
            if (!(g[5] > 0.0)) fail(TWISTY_ERR_INVALID_ARGUMENT, "forward result does not match this experiment");
            const double sigma = std::sqrt((double)ctx->p.eps);
            grad[0] = g[0] / g[5];
            grad[1] = g[1] / g[5] * 2.0 * sigma;   // eps = sigma^2
            grad[2] = g[2] / g[5];
            grad[3] = g[3] / g[5];
            grad[4] = g[4] / g[5];
        } catch (...) {
            dtab.release(); dg.release(); dout.release();
            throw;
        }
        dtab.release(); dg.release(); dout.release();
    });
}

twisty_status twisty_weight_histogram(twisty_ctx *ctx, const twisty_bc *bc, double min_weight, double max_weight,
                                      uint32_t n_buckets, uint64_t *counts)
{
    if (!ctx || !bc || !counts || n_buckets == 0 || n_buckets > 12288 || !(max_weight > min_weight))
        return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (ctx->p.form == TWISTY_FORM_FP64) fail(TWISTY_ERR_UNSUPPORTED, "the histogram replays the plain or compensated form");
        if (ctx->p.eval_end_shift.x != 0.f || ctx->p.eval_end_shift.y != 0.f || ctx->p.eval_end_shift.z != 0.f)
            fail(TWISTY_ERR_UNSUPPORTED, "eval_end_shift applies to forward passes only");
        prepare(ctx, bc);
        const ChainSpec &c = ctx->spec;
        cudaStream_t st = ctx->stream;
        DevBuf dw, dout, dcnt;
        struct Release {
            DevBuf *b[3];
            ~Release()
            {
                for (DevBuf *x : b) x->release();
            }
        } rel{{&dw, &dout, &dcnt}};
        ck(dcnt.ensure(sizeof(unsigned long long) * n_buckets), "alloc histogram");
        ck(cudaMemsetAsync(dcnt.p, 0, sizeof(unsigned long long) * n_buckets, st), "memset");
        if (c.n_chains) {
            // the chains replayed in slices of at most 2^24 weighted paths, every weight kept
            const uint32_t per = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(c.n_chains, (1ull << 24) / std::max(1u, c.steps)));
            ck(dw.ensure(sizeof(double) * (size_t)per * c.steps), "alloc histogram");
            ck(dout.ensure(sizeof(ChainOut) * per), "alloc histogram");
            const float x0[3] = {bc->start_pos.x, bc->start_pos.y, bc->start_pos.z};
            for (uint32_t a = 0; a < c.n_chains; a += per) {
                ChainSpec ce = c;
                ce.chain0 = c.chain0 + a;
                ce.n_chains = std::min(per, c.n_chains - a);
                ce.last_steps = (a + ce.n_chains == c.n_chains) ? c.last_steps : c.steps;
                ck(cudaMemsetAsync(dw.p, 0xff, sizeof(double) * (size_t)ce.n_chains * c.steps, st), "memset");  // NaN
                if (ctx->p.form == TWISTY_FORM_PLAIN_FP32)
                    ck(launch_plain_chains(ce, ctx->init_pos.as<float>(), ctx->state.as<float>(), ctx->lut32.as<float>(),
                                           ctx->meta, dout.as<ChainOut>(), st, nullptr, dw.as<double>()),
                       "histogram replay");
                else
                    ck(launch_comp_export(ce, staged_tuning(ctx), ctx->init_seg.as<float>(), ctx->fixtab.as<float2>(),
                                          ctx->lintab.as<float2>(), ctx->meta, x0, nullptr, dw.as<double>(),
                                          dout.as<ChainOut>(), st, ctx->lf),
                       "histogram replay");
                ck(launch_weight_histogram(dw.as<double>(), (uint64_t)ce.n_chains * c.steps, ctx->log10_norm, min_weight,
                                           max_weight, n_buckets, dcnt.as<unsigned long long>(), st),
                   "histogram");
            }
        }
        std::vector<unsigned long long> h(n_buckets);
        ck(cudaMemcpyAsync(h.data(), dcnt.p, sizeof(unsigned long long) * n_buckets, cudaMemcpyDeviceToHost, st), "read histogram");
        ck(cudaStreamSynchronize(st), "histogram");
        for (uint32_t i = 0; i < n_buckets; ++i) counts[i] = h[i];
    });
}

twisty_status twisty_chain_results(twisty_ctx *ctx, double *log10_sum, uint64_t *valid, uint32_t n_chains)
{
    if (!ctx || (!log10_sum && n_chains)) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (!ctx->launched) fail(TWISTY_ERR_INVALID_ARGUMENT, "no pass has run on this context");
        if (n_chains != ctx->spec.n_chains) fail(TWISTY_ERR_INVALID_ARGUMENT, "n_chains must be the pass's chain count");
        if (n_chains == 0) return;
        set_device(ctx);
        std::vector<ChainOut> h(n_chains);
        ck(cudaEventSynchronize(ctx->ev[2]), "sync");
        ck(cudaMemcpyAsync(h.data(), ctx->chain_out.p, sizeof(ChainOut) * n_chains, cudaMemcpyDeviceToHost, ctx->stream),
           "read chain results");
        ck(cudaStreamSynchronize(ctx->stream), "read chain results");
        for (uint32_t i = 0; i < n_chains; ++i) {
            log10_sum[i] = h[i].log10_sum + ctx->log10_norm;
            if (valid) valid[i] = h[i].valid;
        }
    });
}

twisty_status twisty_set_initial_curve(twisty_ctx *ctx, const float *pos, uint32_t n_points)
{
    if (!ctx) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        if (!pos) {
            ctx->user_curve.clear();
        } else {
            ctx->user_curve.assign(pos, pos + 3 * (size_t)n_points);
        }
        ctx->prepared = false;
    });
}

}  // extern "C"

// ------------------------------------------------------------------ autotuner
twisty_status twisty_autotune(twisty_ctx *ctx, const twisty_bc *bc, uint64_t trial_paths, twisty_tuning *best)
{
    if (!ctx || !bc || !best) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        const twisty_params saved = ctx->p;
        validate(saved);
        if (saved.form != TWISTY_FORM_COMPENSATED) fail(TWISTY_ERR_UNSUPPORTED, "the autotuner times the compensated form");
        const uint32_t N = saved.num_segments, bins = saved.num_curvature_steps;
        const uint64_t paths = trial_paths ? trial_paths : (1ull << 22);
        struct Cand {
            int group, spl, warps;
        };
        std::vector<Cand> cands;
        const CompTuning def = comp_default_tuning(N);
        for (int g : {1, 4, 8, 16, 32})
            for (int spl : {2, 3, 4, 5, 6, 8, 9, 12, 16, 17, 20, 24, 28, 32})
                for (int w = 4; w <= 32; w += 4) {
                    CompTuning t{g, spl, w, 0};
                    const uint32_t k_eff = std::min<uint32_t>(saved.max_sub_chain, N - 2);
                    if (!comp_tuning_supported(t, N, k_eff)) continue;
                    // shapes much wider than N waste their lanes; keep the default shape's width
                    if ((uint32_t)(g * spl) >= 4 * N && g * spl > def.group * def.spl) continue;
                    if (comp_smem_bytes(t, bins) > 227 * 1024) continue;
                    cands.push_back(Cand{g, spl, w});
                }
        if (cands.empty()) fail(TWISTY_ERR_UNSUPPORTED, "no compensated kernel shape for this N / max_sub_chain");
        double best_rate = -1.0;
        Cand bestc = cands.front();
        std::string last_err;
        try {
            for (const Cand &cd : cands) {
                ctx->p = saved;
                ctx->p.comp_group = (uint32_t)cd.group;
                ctx->p.comp_spl = (uint32_t)cd.spl;
                ctx->p.comp_warps = (uint32_t)cd.warps;
                ctx->p.paths_to_generate = paths;
                ctx->p.paths_to_skip = 0;   // burn-in scales with the chain count, not the shape
                ctx->p.num_chains = 0;
                try {
                    prepare(ctx, bc);
                    launch(ctx, ctx->stream);   // warm
                    twisty_result r{};
                    collect(ctx, &r);
                    launch(ctx, ctx->stream);
                    collect(ctx, &r);
                    const double rate = (double)r.total_paths * N / (r.perturb_ms * 1e-3);
                    if (r.perturb_ms > 0 && rate > best_rate) {
                        best_rate = rate;
                        bestc = cd;
                    }
                } catch (const Failure &f) {
                    if (f.s != TWISTY_ERR_UNSUPPORTED && f.s != TWISTY_ERR_INVALID_CONFIG) throw;
                    last_err = f.msg;
                }
            }
        } catch (...) {
            ctx->p = saved;
            ctx->prepared = false;
            throw;
        }
        ctx->p = saved;
        ctx->prepared = false;
        if (best_rate < 0) fail(TWISTY_ERR_UNSUPPORTED, "no shape ran: " + last_err);
        tune_record(TuneEntry{ctx->device_name, N, bins, (uint32_t)bestc.group, (uint32_t)bestc.spl,
                              (uint32_t)bestc.warps, best_rate});
        best->num_segments = N;
        best->bins = bins;
        best->group = (uint32_t)bestc.group;
        best->spl = (uint32_t)bestc.spl;
        best->warps = (uint32_t)bestc.warps;
        best->path_segments_per_s = best_rate;
    });
}

twisty_status twisty_default_shape(uint32_t num_segments, uint32_t bins, twisty_shape *out)
{
    if (!out || num_segments < 4 || bins < 2) {
        g_free_err = "twisty_default_shape: null out, N < 4 or bins < 2";
        return TWISTY_ERR_INVALID_ARGUMENT;
    }
    CompTuning t = comp_default_tuning(num_segments);
    if (!comp_tuning_supported(t, num_segments, 2)) {
        g_free_err = "no compensated kernel shape for this N";
        return TWISTY_ERR_UNSUPPORTED;
    }
    t.lut_global = table_through_l1(t, bins, true) ? 1 : 0;
    if (!comp_fit_smem(t, bins, true)) {
        g_free_err = "chain state does not fit in shared memory";
        return TWISTY_ERR_UNSUPPORTED;
    }
    const int bw = std::min(t.warps_per_block, batch_max_threads(t.group, t.spl) / 32);
    out->group = (uint32_t)t.group;
    out->spl = (uint32_t)t.spl;
    out->warps = (uint32_t)t.warps_per_block;
    out->table_in_l1 = (uint32_t)t.lut_global;
    out->smem_bytes = (uint32_t)comp_smem_bytes(t, bins);
    out->batched = batch_shape_supported(BatchShape{t.group, t.spl, bw, 0, 1, 0, 0}, num_segments, 2) ? 1u : 0u;
    return TWISTY_OK;
}

twisty_status twisty_tuning_cache_save(const char *path)
{
    if (!path) return TWISTY_ERR_INVALID_ARGUMENT;
    std::ostringstream o;
    o.precision(17);
    o << "{\n  \"entries\": [";
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (size_t i = 0; i < g_tune.size(); ++i) {
            const TuneEntry &e = g_tune[i];
            std::string dev;
            for (char ch : e.device) {
                if (ch == '"' || ch == '\\') dev.push_back('\\');
                dev.push_back(ch);
            }
            o << (i ? "," : "") << "\n    {\"device\": \"" << dev << "\", \"n\": " << e.n << ", \"bins\": " << e.bins
              << ", \"group\": " << e.group << ", \"spl\": " << e.spl << ", \"warps\": " << e.warps
              << ", \"path_segments_per_s\": " << e.rate << "}";
        }
    }
    o << "\n  ]\n}\n";
    std::ofstream f(path);
    if (!f) {
        g_free_err = std::string("cannot write ") + path;
        return TWISTY_ERR_IO;
    }
    f << o.str();
    return f.good() ? TWISTY_OK : TWISTY_ERR_IO;
}

twisty_status twisty_tuning_cache_load(const char *path)
{
    if (!path) return TWISTY_ERR_INVALID_ARGUMENT;
    std::ifstream f(path);
    if (!f) {
        g_free_err = std::string("cannot read ") + path;
        return TWISTY_ERR_IO;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    Node root;
    std::string err;
    if (!parse_json(ss.str(), root, err)) {
        g_free_err = "tuning cache: " + err;
        return TWISTY_ERR_INVALID_CONFIG;
    }
    const Node *es = root.get("entries");
    if (!es || es->kind != Node::Array) {
        g_free_err = "tuning cache: no entries array";
        return TWISTY_ERR_INVALID_CONFIG;
    }
    std::vector<TuneEntry> got;
    for (const Node &e : es->arr) {
        const Node *dv = e.get("device");
        const char *keys[] = {"n", "bins", "group", "spl", "warps"};
        uint32_t v[5];
        bool ok = dv && dv->kind == Node::String;
        for (int i = 0; i < 5 && ok; ++i) {
            const Node *x = e.get(keys[i]);
            ok = x && x->kind == Node::Number && x->num >= 0 && x->num < 4294967296.0;
            if (ok) v[i] = (uint32_t)x->num;
        }
        if (!ok) {
            g_free_err = "tuning cache: malformed entry";
            return TWISTY_ERR_INVALID_CONFIG;
        }
        CompTuning t{(int)v[2], (int)v[3], (int)v[4], 0};
        if (!comp_tuning_supported(t, v[0], 2)) {
            g_free_err = "tuning cache: unsupported shape";
            return TWISTY_ERR_INVALID_CONFIG;
        }
        const Node *rt = e.get("path_segments_per_s");
        got.push_back(TuneEntry{dv->str, v[0], v[1], v[2], v[3], v[4], (rt && rt->kind == Node::Number) ? rt->num : 0.0});
    }
    for (const TuneEntry &e : got) tune_record(e);
    return TWISTY_OK;
}

// ------------------------------------------------------------ multi-arclength tables
namespace {
constexpr uint32_t kMultiMagic = 0x444D5754u;   // "TWMD"
constexpr uint32_t kMultiVersion = 1;
}  // namespace

twisty_status twisty_multi_ds_tables(twisty_ctx *ctx, float min_ds, float max_ds, uint32_t n_ds, const char *cache_path)
{
    if (!ctx) return TWISTY_ERR_INVALID_ARGUMENT;
    return guard(ctx, [&] {
        const twisty_params &p = ctx->p;
        if (n_ds < 2 || n_ds > 65535u || !(min_ds > 0.0f) || !(max_ds > min_ds))
            fail(TWISTY_ERR_INVALID_ARGUMENT, "need 2 <= n_ds <= 65535 and 0 < min_ds < max_ds");
        if (p.num_curvature_steps < 2 || p.num_steps_int < 4 || (p.num_steps_int & 1u) || !(p.eps > 0.0f))
            fail(TWISTY_ERR_INVALID_CONFIG, "invalid weighting parameters");
        set_device(ctx);
        auto &M = ctx->multi;
        M.ready = false;
        M.n = n_ds;
        M.bins = p.num_curvature_steps;
        M.min_ds = min_ds;
        M.max_ds = max_ds;
        weighting_fingerprint(p, M.wp);
        const uint32_t bins = M.bins;
        // ds grid of the reference (:170-173)
        const float step_ds = (max_ds - min_ds) / (float)(n_ds - 1);
        M.ds.resize(n_ds);
        M.meta.resize(n_ds);
        for (uint32_t i = 0; i < n_ds; ++i) {
            M.ds[i] = min_ds + (float)i * step_ds;
            const float max_k = (float)((2.0 / (double)M.ds[i]) * (double)1.01f);
            M.meta[i] = LutMetaF{0.0f, max_k, max_k / (float)(bins - 1), (int32_t)bins};
        }
        M.host.assign((size_t)n_ds * bins, 0.0f);
        M.min_w.assign(n_ds, 0.0);
        M.max_w.assign(n_ds, 0.0);
        bool loaded = false;
        if (cache_path) {
            std::ifstream f(cache_path, std::ios::binary);
            uint32_t hdr[4] = {0, 0, 0, 0};
            float wp[9], rng[2];
            if (f && f.read(reinterpret_cast<char *>(hdr), sizeof(hdr)) && f.read(reinterpret_cast<char *>(wp), sizeof(wp)) &&
                f.read(reinterpret_cast<char *>(rng), sizeof(rng)) && hdr[0] == kMultiMagic && hdr[1] == kMultiVersion &&
                hdr[2] == n_ds && hdr[3] == bins && std::memcmp(wp, M.wp, sizeof(wp)) == 0 && rng[0] == min_ds &&
                rng[1] == max_ds) {
                f.read(reinterpret_cast<char *>(M.min_w.data()), sizeof(double) * n_ds);
                f.read(reinterpret_cast<char *>(M.max_w.data()), sizeof(double) * n_ds);
                f.read(reinterpret_cast<char *>(M.host.data()), sizeof(float) * M.host.size());
                loaded = (bool)f;
            }
        }
        cudaStream_t st = ctx->stream;
        ck(M.dev.ensure(sizeof(float) * M.host.size()), "alloc multi-ds tables");
        if (loaded) {
            ck(cudaMemcpyAsync(M.dev.p, M.host.data(), sizeof(float) * M.host.size(), cudaMemcpyHostToDevice, st), "upload");
            ck(cudaStreamSynchronize(st), "upload");
        } else {
            std::vector<LutBuildSpec> specs(n_ds);
            for (uint32_t i = 0; i < n_ds; ++i) {
                LutBuildSpec &s = specs[i];
                s = LutBuildSpec{};
                s.mu = p.mu;
                s.eps = p.eps;
                s.scatter = p.scatter;
                s.min_bound = p.min_bound;
                s.max_bound = p.max_bound;
                s.bias = p.bias;
                s.num_steps_int = p.num_steps_int;
                s.bins = bins;
                s.ds = M.ds[i];
                s.min_k = 0.0f;
                s.step = M.meta[i].step;
                s.step64 = ((2.0 / (double)M.ds[i]) * 1.01) / (double)(bins - 1);
            }
            DevBuf dspecs, d64, dmm;
            struct Release {
                DevBuf *b[3];
                ~Release()
                {
                    for (DevBuf *x : b) x->release();
                }
            } rel{{&dspecs, &d64, &dmm}};
            ck(dspecs.ensure(sizeof(LutBuildSpec) * n_ds), "alloc");
            ck(d64.ensure(sizeof(double) * M.host.size()), "alloc");
            ck(dmm.ensure(sizeof(double) * 3 * n_ds), "alloc");
            ck(cudaMemcpyAsync(dspecs.p, specs.data(), sizeof(LutBuildSpec) * n_ds, cudaMemcpyHostToDevice, st), "upload");
            ck(launch_lut_build_batch(dspecs.as<LutBuildSpec>(), n_ds, bins, d64.as<double>(), st), "multi-ds build");
            ck(launch_lut_finalize_batch(n_ds, bins, d64.as<double>(), M.dev.as<float>(), dmm.as<double>(), st),
               "multi-ds finalize");
            std::vector<double> mm(3 * (size_t)n_ds);
            ck(cudaMemcpyAsync(M.host.data(), M.dev.p, sizeof(float) * M.host.size(), cudaMemcpyDeviceToHost, st), "read");
            ck(cudaMemcpyAsync(mm.data(), dmm.p, sizeof(double) * mm.size(), cudaMemcpyDeviceToHost, st), "read");
            ck(cudaStreamSynchronize(st), "multi-ds tables");
            for (uint32_t i = 0; i < n_ds; ++i) {
                M.min_w[i] = mm[3 * i];
                M.max_w[i] = mm[3 * i + 1];
            }
            if (cache_path) {
                std::ofstream f(cache_path, std::ios::binary);
                const uint32_t hdr[4] = {kMultiMagic, kMultiVersion, n_ds, bins};
                const float rng[2] = {min_ds, max_ds};
                f.write(reinterpret_cast<const char *>(hdr), sizeof(hdr));
                f.write(reinterpret_cast<const char *>(M.wp), sizeof(M.wp));
                f.write(reinterpret_cast<const char *>(rng), sizeof(rng));
                f.write(reinterpret_cast<const char *>(M.min_w.data()), sizeof(double) * n_ds);
                f.write(reinterpret_cast<const char *>(M.max_w.data()), sizeof(double) * n_ds);
                f.write(reinterpret_cast<const char *>(M.host.data()), sizeof(float) * M.host.size());
                if (!f) fail(TWISTY_ERR_IO, std::string("cannot write ") + cache_path);
            }
        }
        for (size_t i = 0; i < M.host.size(); ++i)
            if (!std::isfinite(M.host[i])) fail(TWISTY_ERR_LUT_INVALID, "multi-ds table has non-finite entries");
        ++M.gen;
        M.ready = true;
        ctx->lut_ready = false;
    });
}
