// twisty_b200_runner.hpp -- C++ runner classes over the C ABI (include/twisty_b200.h).
//
// Mirrors the reference's runner API so a caller of twisty::ExperimentRunner
// (Twisty/ExperimentRunner.h:29-131) and its subclasses
// FullExperimentRunnerOptimalPerturb (Twisty/FullExperimentRunnerOptimalPerturb.h:26-74)
// and FullExperimentRunnerOptimalPerturbOptimized_GPU
// (Twisty/FullExperimentRunnerOptimalPerturbOptimized_GPU.h:36-47) keeps its code:
//
//   ExperimentParameters params = ExperimentRunner::ParseExperimentParamsFromConfig(json);
//   FullExperimentRunnerOptimalPerturb runner(params);
//   std::optional<ExperimentResults> r = runner.RunExperiment(boundaryConditions);
//
// Differences a caller sees: the config arrives as text (JSON, or the same keys in YAML);
// ExperimentResults::experimentWeight is a long double (x87 range reaches 1e4932; the
// reference uses a 100-digit decimal) and experimentWeightLog10 carries the exact log10;
// failures return std::nullopt with lastError() set, never exit() or a thrown exception.
// Header-only; link with libtwisty_b200.so.
#pragma once

#include "twisty_b200.h"

#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

namespace twisty {
namespace b200 {

struct Vector3 {
    float x = 0.0f, y = 0.0f, z = 0.0f;
    Vector3() = default;
    Vector3(float a, float b, float c) : x(a), y(b), z(c) {}
};

// PerturbUtils::BoundaryConditions (Twisty/CurvePerturbUtils.h:62-68)
struct BoundaryConditions {
    Vector3 m_startPos = Vector3(0.0f, 0.0f, 0.0f);
    Vector3 m_startDir = Vector3(1.0f, 0.0f, 0.0f);
    Vector3 m_endPos = Vector3(0.0f, 0.0f, 0.0f);
    Vector3 m_endDir = Vector3(1.0f, 0.0f, 0.0f);
    float arclength = 0.0f;

    twisty_bc to_c() const
    {
        return twisty_bc{{m_startPos.x, m_startPos.y, m_startPos.z}, {m_startDir.x, m_startDir.y, m_startDir.z},
                         {m_endPos.x, m_endPos.y, m_endPos.z}, {m_endDir.x, m_endDir.y, m_endDir.z}, arclength};
    }
};

// WeightingParameters (Twisty/PathWeightUtils.h:35-48)
enum class WeightingMethod : int32_t { RadiativeTransfer = 0, SimplifiedModel = 1 };
struct WeightingParameters {
    float mu = 0.1f;
    uint32_t numStepsInt = 2000;
    float minBound = 0.0f;
    float maxBound = 100.0f;
    float eps = 0.01f;
    float bias = 1.0f;
    float scatter = 0.0f;
    float absorption = 0.0f;
    uint32_t numCurvatureSteps = 10000;
    WeightingMethod weightingMethod = WeightingMethod::RadiativeTransfer;
};

class ExperimentRunner {
   public:
    enum class PerturbMethod { GeometricRandom, GeometricMinCurvature, GeometricCombined };

    // ExperimentRunner::ExperimentParameters (Twisty/ExperimentRunner.h:42-68) + B200 knobs
    struct ExperimentParameters {
        uint64_t numPathsInExperiment = 0;
        uint64_t numPathsPerBatch = 1000000;
        uint64_t numPathsToSkip = 0;
        uint32_t numSegmentsPerCurve = 4;
        bool allowSaturatePathCount = true;
        float arclength = 0.0f;
        uint32_t exportPathBatchSize = 1000;
        bool exportGeneratedCurves = false;
        std::string experimentName = "Default_Experiment";
        std::string experimentDirPath = "./Default_Experiment/";
        std::string perExperimentDirSubfolder = "";
        std::string pathBatchPrepend = "";
        uint32_t bootstrapSeed = 0;
        uint32_t curvePurturbSeed = 0;
        WeightingParameters weightingParameters;
        PerturbMethod perturbMethod = PerturbMethod::GeometricRandom;
        int32_t maxPerturbThreads = 0;
        int32_t maxWeightThreads = 0;
        bool outputBigFloatWeights = false;
        bool outputPathBatches = false;
        bool useGpu = true;
        // B200
        twisty_form form = TWISTY_FORM_COMPENSATED;
        twisty_lut_mode lutMode = TWISTY_LUT_FP64;
        uint32_t maxSubChain = 25;
        float maxAngle = 3.141592653589793f;
        uint32_t numChains = 0;
        int32_t device = 0;
        uint64_t maxExportedPaths = 1000000;
        // histogram.txt of the path weights (the reference always writes it; here it costs one
        // more pass, so it is asked for): 500 buckets over the reference's range
        bool outputHistogram = false;
        double histogramMinWeight = 4.69653e-16;
        double histogramMaxWeight = 1.17517e-13;
        uint32_t histogramBuckets = 500;
    };

    // ExperimentRunner::ExperimentResults (Twisty/ExperimentRunner.h:73-82)
    struct ExperimentResults {
        long double experimentWeight = 0.0L;
        double experimentWeightLog10 = -INFINITY;
        double normalizerLog10 = 0.0;
        double relStdError = NAN;
        uint64_t totalPathsGenerated = 0;
        uint64_t numFailedPaths = 0;
        long long totalExperimentMs = 0;
        long long setupExperimentMs = 0;
        long long perturbExperimentMs = 0;
        long long weightingExperimentMs = 0;
        // error against FP64 (twisty_result.weight_error_bound, .fp64_rel_error)
        double weightErrorBoundLog10 = 0.0;
        double fp64RelError = NAN;
    };

    // ExperimentRunner::ParseExperimentParamsFromConfig (Twisty/ExperimentRunner.cpp:48-177).
    // Also returns the basicExperiment block when bc is given.
    static ExperimentParameters ParseExperimentParamsFromConfig(const std::string &configText, bool yaml = false,
                                                                BoundaryConditions *bc = nullptr,
                                                                std::string *error = nullptr)
    {
        ExperimentParameters out;
        twisty_params p;
        twisty_bc cbc;
        const twisty_status s = twisty_params_from_config(configText.c_str(), yaml ? 1 : 0, &p, &cbc);
        if (s != TWISTY_OK) {
            if (error) *error = twisty_last_error(nullptr);
            return out;
        }
        out.numPathsInExperiment = p.paths_to_generate;
        out.numPathsToSkip = p.paths_to_skip;
        out.numSegmentsPerCurve = p.num_segments;
        out.bootstrapSeed = p.bootstrap_seed;
        out.curvePurturbSeed = p.perturb_seed;
        out.weightingParameters.mu = p.mu;
        out.weightingParameters.eps = p.eps;
        out.weightingParameters.scatter = p.scatter;
        out.weightingParameters.absorption = p.absorption;
        out.weightingParameters.numStepsInt = p.num_steps_int;
        out.weightingParameters.numCurvatureSteps = p.num_curvature_steps;
        out.weightingParameters.minBound = p.min_bound;
        out.weightingParameters.maxBound = p.max_bound;
        out.weightingParameters.weightingMethod = (WeightingMethod)p.weight_function;
        out.perturbMethod = (PerturbMethod)p.perturb_method;
        out.form = (twisty_form)p.form;
        out.lutMode = (twisty_lut_mode)p.lut_mode;
        out.maxSubChain = p.max_sub_chain;
        out.maxAngle = p.max_angle;
        out.numChains = p.num_chains;
        out.device = p.device;
        if (bc) {
            bc->m_startPos = Vector3(cbc.start_pos.x, cbc.start_pos.y, cbc.start_pos.z);
            bc->m_startDir = Vector3(cbc.start_dir.x, cbc.start_dir.y, cbc.start_dir.z);
            bc->m_endPos = Vector3(cbc.end_pos.x, cbc.end_pos.y, cbc.end_pos.z);
            bc->m_endDir = Vector3(cbc.end_dir.x, cbc.end_dir.y, cbc.end_dir.z);
            bc->arclength = cbc.arclength;
        }
        return out;
    }

    // ExperimentRunner(ExperimentParameters&) (Twisty/ExperimentRunner.cpp:180-192): keeps a
    // reference to the caller's parameters and creates the experiment directory.
    explicit ExperimentRunner(ExperimentParameters &experimentParams) : m_experimentParams(experimentParams)
    {
        m_experimentDirPath = std::filesystem::path(m_experimentParams.experimentDirPath);
        if (!experimentParams.perExperimentDirSubfolder.empty())
            m_experimentDirPath /= experimentParams.perExperimentDirSubfolder;
        std::error_code ec;
        std::filesystem::create_directories(m_experimentDirPath, ec);
    }
    virtual ~ExperimentRunner()
    {
        if (m_ctx) twisty_destroy(m_ctx);
    }
    ExperimentRunner(const ExperimentRunner &) = delete;
    ExperimentRunner &operator=(const ExperimentRunner &) = delete;

    // ExperimentRunner::RunExperiment (Twisty/ExperimentRunner.cpp:196-301)
    std::optional<ExperimentResults> RunExperiment(BoundaryConditions boundaryConditions)
    {
        twisty_params p = to_c();
        p.form = formOfRunner();
        if (!ensure_ctx(p)) return std::nullopt;
        const twisty_bc bc = boundaryConditions.to_c();
        twisty_result r{};
        twisty_status s;
        if (m_experimentParams.outputPathBatches) {
            uint64_t written = 0;
            const std::string dir = m_experimentDirPath.string();
            s = twisty_export_paths(m_ctx, &bc, dir.c_str(), m_experimentParams.maxExportedPaths, nullptr, nullptr,
                                    &written, &r);
        } else {
            s = twisty_run(m_ctx, &bc, &r);
        }
        if (s != TWISTY_OK) {
            m_lastError = std::string(twisty_status_string(s)) + ": " + twisty_last_error(m_ctx);
            return std::nullopt;
        }
        ExperimentResults out;
        out.experimentWeightLog10 = r.log10_weight;
        out.experimentWeight = std::pow(10.0L, (long double)r.log10_weight);
        out.normalizerLog10 = r.log10_normalizer;
        out.relStdError = r.rel_std_error;
        out.totalPathsGenerated = r.total_paths;
        out.numFailedPaths = r.failed_paths;
        out.totalExperimentMs = (long long)r.total_ms;
        out.setupExperimentMs = (long long)r.setup_ms;
        out.perturbExperimentMs = (long long)r.perturb_ms;
        out.weightingExperimentMs = (long long)r.weighting_ms;
        out.weightErrorBoundLog10 = r.weight_error_bound;
        out.fp64RelError = r.fp64_rel_error;
        WriteConvergence(r);
        if (m_experimentParams.outputHistogram && !WriteHistogram(bc)) return std::nullopt;
        return out;
    }

    const std::string &lastError() const { return m_lastError; }
    twisty_ctx *context() const { return m_ctx; }

   protected:
    virtual twisty_form formOfRunner() const { return m_experimentParams.form; }

    // histogram.txt in the reference's layout (FullExperimentRunnerOptimalPerturb.cpp:394-422):
    // a "Histogram" line, then "binMin binMax count" per bucket.
    bool WriteHistogram(const twisty_bc &bc)
    {
        const ExperimentParameters &e = m_experimentParams;
        std::vector<uint64_t> counts(e.histogramBuckets);
        const twisty_status s = twisty_weight_histogram(m_ctx, &bc, e.histogramMinWeight, e.histogramMaxWeight,
                                                        e.histogramBuckets, counts.data());
        if (s != TWISTY_OK) {
            m_lastError = std::string(twisty_status_string(s)) + ": " + twisty_last_error(m_ctx);
            return false;
        }
        std::ofstream f(m_experimentDirPath / "histogram.txt");
        f << "Histogram" << '\n';
        const double lo = e.histogramMinWeight, hi = e.histogramMaxWeight;
        for (uint32_t i = 0; i < e.histogramBuckets; ++i)
            f << lo + (hi - lo) * i / e.histogramBuckets << " " << lo + (hi - lo) * (i + 1) / e.histogramBuckets << " "
              << counts[i] << '\n';
        return true;
    }

    // ConvergenceWeights/ConvergenceWeights.txt, as ExperimentRunner::UpdateConvergenceWeight
    // writes it (Twisty/ExperimentRunner.cpp:399-422): "paths, running mean weight" each time
    // numPathsPerBatch more paths have been added -- here the chains' sums in chain order (a chain
    // is the reference's thread). Best effort: an unwritable directory leaves the result alone.
    void WriteConvergence(const twisty_result &r)
    {
        if (r.num_chains == 0) return;
        std::vector<double> lw(r.num_chains);
        std::vector<uint64_t> valid(r.num_chains);
        if (twisty_chain_results(m_ctx, lw.data(), valid.data(), r.num_chains) != TWISTY_OK) return;
        std::error_code ec;
        const std::filesystem::path dir = m_experimentDirPath / "ConvergenceWeights";
        std::filesystem::create_directories(dir, ec);
        std::ofstream f(dir / "ConvergenceWeights.txt");
        if (!f) return;
        const uint64_t batch = m_experimentParams.numPathsPerBatch ? m_experimentParams.numPathsPerBatch : 1000000;
        uint64_t paths = 0, since = 0;
        long double sum = 0.0L;
        for (uint32_t c = 0; c < r.num_chains; ++c) {
            if (std::isfinite(lw[c])) sum += std::pow(10.0L, (long double)lw[c]);
            paths += valid[c];
            since += valid[c];
            if (since >= batch || c + 1 == r.num_chains) {
                f << paths << ", " << (paths ? sum / (long double)paths : 0.0L) << std::endl;
                since = 0;
            }
        }
    }

    twisty_params to_c() const
    {
        twisty_params p;
        twisty_params_init(&p);
        const ExperimentParameters &e = m_experimentParams;
        const WeightingParameters &w = e.weightingParameters;
        p.paths_to_generate = e.numPathsInExperiment;
        p.paths_to_skip = e.numPathsToSkip;
        p.num_segments = e.numSegmentsPerCurve;
        p.bootstrap_seed = e.bootstrapSeed;
        p.perturb_seed = e.curvePurturbSeed;
        p.weight_function = (int32_t)w.weightingMethod;
        p.perturb_method = (int32_t)e.perturbMethod;
        p.mu = w.mu;
        p.eps = w.eps;
        p.scatter = w.scatter;
        p.absorption = w.absorption;
        p.num_steps_int = w.numStepsInt;
        p.num_curvature_steps = w.numCurvatureSteps;
        p.min_bound = w.minBound;
        p.max_bound = w.maxBound;
        p.bias = w.bias;
        p.form = e.form;
        p.lut_mode = e.lutMode;
        p.max_sub_chain = e.maxSubChain;
        p.max_angle = e.maxAngle;
        p.num_chains = e.numChains;
        p.device = e.device;
        return p;
    }

    bool ensure_ctx(const twisty_params &p)
    {
        twisty_status s;
        if (!m_ctx) {
            s = twisty_create(&p, &m_ctx);
            if (s != TWISTY_OK) {
                m_lastError = std::string(twisty_status_string(s)) + ": " + twisty_last_error(nullptr);
                m_ctx = nullptr;
                return false;
            }
            return true;
        }
        s = twisty_update_params(m_ctx, &p);
        if (s != TWISTY_OK) {
            m_lastError = std::string(twisty_status_string(s)) + ": " + twisty_last_error(m_ctx);
            return false;
        }
        return true;
    }

    ExperimentParameters &m_experimentParams;
    std::filesystem::path m_experimentDirPath;
    twisty_ctx *m_ctx = nullptr;
    std::string m_lastError;
};

// Drop-in for twisty::FullExperimentRunnerOptimalPerturb (CPU runner): the chains run on
// the B200 in the form the parameters select (compensated by default).
class FullExperimentRunnerOptimalPerturb : public ExperimentRunner {
   public:
    explicit FullExperimentRunnerOptimalPerturb(ExperimentParameters &p) : ExperimentRunner(p) {}
};

// Drop-in for twisty::FullExperimentRunnerOptimalPerturbOptimized_GPU, whose kernel design
// (one chain per thread, state in global memory, FP64 log10 per segment) the plain FP32
// form reproduces; the form the parameters select is used, so both names run the same code.
class FullExperimentRunnerOptimalPerturbOptimized_GPU : public ExperimentRunner {
   public:
    explicit FullExperimentRunnerOptimalPerturbOptimized_GPU(ExperimentParameters &p) : ExperimentRunner(p) {}
};

}  // namespace b200
}  // namespace twisty
