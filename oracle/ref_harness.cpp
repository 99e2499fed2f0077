// Oracle pin harness (test infrastructure only; never shipped, never on the product path).
//
// Links the reference's own hot-path sources (compiled from the reference tree by
// oracle/Makefile into oracle/_ref) and drives them on files, so that golden vectors
// and the CPU baseline come from the reference's code rather than from a restatement.
//
// Subcommands (binary layouts are little-endian, documented per mode):
//   lut       <mu> <eps> <scatter> <absorption> <numStepsInt> <bins> <ds> <out>
//             WeightLookupTableIntegral + Initialize (Twisty/PathWeightUtils.cpp:281-348)
//             out: f32 minK, maxK, step, minW, maxW, ds; u32 bins; f32 lut[bins]
//   weigh     <lut> <N> <arclength> <absorption> <paths> <out>
//             UpdateTangentsFromPos (Twisty/CurvePerturbUtils.cpp:147-154),
//             UpdateCurvaturesFromTangents_RadiativeTransfer (:157-166, patched P3),
//             WeightCurveViaCurvatureLog10_CudaSafe (Twisty/PathWeighters.cpp:27-104).
//             paths: u64 P; f32 pos[P][N+1][3]
//             out per path: u8 valid; f64 log10w; f32 curv[N-1]; i32 bin[N-1]
//             Bin indices are read back from the reference weigher itself by weighing each
//             curvature alone against a ramp table lut[i] = i + 1 (weight = 1 + L + d).
//   rotate    <in> <out>   RotateVectorByQuaternion (Twisty/CurvePerturbUtils.cpp:113-127)
//             in: u64 n; f32 rec[n][7] (q0..q3, v0..v2)    out: f32 v'[n][3]
//   cw        <in> <out>   CombinedWeightValues_C (Twisty/CombinedWeightUtils.h:48-174)
//             in: u64 n; u64 split; f64 log10v[n]
//             out: 3 x {f64 max, total, offset; u32 n; u32 pad}; f64 log10 Extract(A), (B), (A+B)
//   norm      <N> <ds> <12 floats: startPos startDir endPos endDir>
//             prints log10 Norm(N, ds, bc) (Twisty/PathWeightUtils.cpp:721-752)
//   bootstrap <N> <arclength> <12 floats> <seed> <out>
//             Curve::SetBoundaryConditions + ResolveEvenNumberOfSegments (patched P2)
//             out: f32 pos[N+1][3]
//   msegment  <lut> <N> <arclength> <12 floats> <absorption> <seed> <paths> <threads> - <out>
//             MSegmentPathGenerationMC's per-path work (Experiments/ExperimentBase.cpp:1246-1386)
//             through the reference's functions; out per path: u8 valid; f64 log10w
//   chain     <config.json> <initcurve|-> <threads> <paths> <out.json>
//             The reference's per-thread Markov-chain loop GeometryRandom
//             (Twisty/FullExperimentRunnerOptimalPerturb.cpp:437-597), orchestrated exactly as
//             RunnerSpecificRunExperiment does (:48-435: per-thread mt19937_64(seed+i), one
//             replicated initial curve, 1e6-path CombinedWeightValues_C chunks, extraction),
//             but with the initial curve read from a file so that any N can run (the
//             reference bootstrapper only accepts N-2 in {4,6,8,12,16,24,...}).
//             initcurve: f32 pos[N+1][3], or '-' for the reference bootstrapper.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <thread>
#include <vector>
#include <chrono>
#include <any>
#include <atomic>
#include <condition_variable>
#include <filesystem>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <sstream>
#include <nlohmann/json.hpp>
#include <boost/multiprecision/cpp_dec_float.hpp>
#include <FMath/FMath.h>

// The reference keeps GeometryRandom private; expose it to this harness only. Every
// standard and third-party header the reference includes is pulled in above, so the
// redefinition touches only the reference's own declarations.
#define private public
#include "FullExperimentRunnerOptimalPerturb.h"
#undef private
#include "CombinedWeightUtils.h"
#include "Curve.h"
#include "CurvePerturbUtils.h"
#include "PathGeneration.h"
#include "PathWeightUtils.h"
#include "PathWeighters.h"

#include <nlohmann/json.hpp>

using twisty::PathWeighting::WeightLookupTableIntegral;

namespace {

template <class T>
void readv(std::ifstream &f, T *p, size_t n)
{
    f.read(reinterpret_cast<char *>(p), sizeof(T) * n);
    if (!f) throw std::runtime_error("short read");
}
template <class T>
void writev(std::ofstream &f, const T *p, size_t n)
{
    f.write(reinterpret_cast<const char *>(p), sizeof(T) * n);
}

struct Lut {
    float minK, maxK, step, minW, maxW, ds;
    uint32_t bins;
    std::vector<float> v;
};

Lut load_lut(const char *path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open lut");
    Lut l;
    readv(f, &l.minK, 1); readv(f, &l.maxK, 1); readv(f, &l.step, 1);
    readv(f, &l.minW, 1); readv(f, &l.maxW, 1); readv(f, &l.ds, 1);
    readv(f, &l.bins, 1);
    l.v.resize(l.bins);
    readv(f, l.v.data(), l.bins);
    return l;
}

twisty::PerturbUtils::BoundaryConditions bc_from(char **a, float arclength)
{
    twisty::PerturbUtils::BoundaryConditions bc;
    bc.m_startPos = Farlor::Vector3(atof(a[0]), atof(a[1]), atof(a[2]));
    bc.m_startDir = Farlor::Vector3(atof(a[3]), atof(a[4]), atof(a[5]));
    bc.m_endPos = Farlor::Vector3(atof(a[6]), atof(a[7]), atof(a[8]));
    bc.m_endDir = Farlor::Vector3(atof(a[9]), atof(a[10]), atof(a[11]));
    bc.arclength = arclength;
    return bc;
}

int mode_lut(int argc, char **argv)
{
    if (argc != 10) return 2;
    twisty::WeightingParameters wp;
    wp.mu = (float)atof(argv[2]);
    wp.eps = (float)atof(argv[3]);
    wp.scatter = (float)atof(argv[4]);
    wp.absorption = (float)atof(argv[5]);
    wp.numStepsInt = (uint32_t)atoi(argv[6]);
    wp.numCurvatureSteps = (uint32_t)atoi(argv[7]);
    wp.minBound = 0.0f;
    wp.maxBound = 10.0f / wp.eps;  // Twisty/ExperimentRunner.cpp:169-171
    const float ds = (float)atof(argv[8]);
    WeightLookupTableIntegral t(wp, ds);
    t.Initialize();
    std::ofstream o(argv[9], std::ios::binary);
    float hdr[6] = {t.GetMinCurvature(), t.GetMaxCurvature(), t.GetCurvatureStepSize(),
          t.GetMinSegmentWeight(), t.GetMaxSegmentWeight(), t.GetDs()};
    writev(o, hdr, 6);
    uint32_t bins = (uint32_t)t.AccessLookupTable().size();
    writev(o, &bins, 1);
    writev(o, t.AccessLookupTable().data(), bins);
    return 0;
}

int mode_weigh(int argc, char **argv)
{
    if (argc != 8) return 2;
    Lut l = load_lut(argv[2]);
    const uint32_t N = (uint32_t)atoi(argv[3]);
    twisty::PerturbUtils::BoundaryConditions bc;
    bc.arclength = (float)atof(argv[4]);
    const float absorption = (float)atof(argv[5]);
    std::ifstream in(argv[6], std::ios::binary);
    uint64_t P = 0;
    readv(in, &P, 1);
    std::vector<Farlor::Vector3> pos(N + 1), tan(N);
    std::vector<float> curv(N - 1), raw((N + 1) * 3);
    std::vector<float> ramp(l.bins);
    for (uint32_t i = 0; i < l.bins; ++i) ramp[i] = (float)(i + 1);
    std::vector<int32_t> bins(N - 1);
    std::ofstream o(argv[7], std::ios::binary);
    for (uint64_t p = 0; p < P; ++p) {
        readv(in, raw.data(), raw.size());
        for (uint32_t i = 0; i <= N; ++i) pos[i] = Farlor::Vector3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
        twisty::PerturbUtils::UpdateTangentsFromPos(pos.data(), tan.data(), N, bc);
        twisty::PerturbUtils::UpdateCurvaturesFromTangents_RadiativeTransfer(tan.data(), curv.data(), N, bc);
        std::vector<float> curvCopy = curv;
        twisty::PathWeighting::PathWeightValue w = twisty::PathWeighting::WeightCurveViaCurvatureLog10_CudaSafe(
              curvCopy.data(), N - 1, l.v.data(), (int32_t)l.bins, l.ds, l.minK, l.maxK, l.step, absorption);
        for (uint32_t i = 0; i + 1 < N; ++i) {
            float c = curv[i];
            twisty::PathWeighting::PathWeightValue r = twisty::PathWeighting::WeightCurveViaCurvatureLog10_CudaSafe(
                  &c, 1, ramp.data(), (int32_t)l.bins, l.ds, l.minK, l.maxK, l.step, 0.0f);
            // ramp blend = (L+1)(1-d) + (L+2)d = L + 1 + d with 0 <= d < step << 1
            const double v = std::pow(10.0, r.weight) - 1.0;
            bins[i] = r.isValid ? (int32_t)std::floor(v - 0.5 * (double)l.step + 0.5) : -1;
        }
        uint8_t valid = w.isValid ? 1 : 0;
        writev(o, &valid, 1);
        writev(o, &w.weight, 1);
        writev(o, curv.data(), N - 1);
        writev(o, bins.data(), N - 1);
    }
    return 0;
}

int mode_rotate(int argc, char **argv)
{
    if (argc != 4) return 2;
    std::ifstream in(argv[2], std::ios::binary);
    uint64_t n = 0;
    readv(in, &n, 1);
    std::ofstream o(argv[3], std::ios::binary);
    for (uint64_t i = 0; i < n; ++i) {
        float r[7];
        readv(in, r, 7);
        float v[3] = {r[4], r[5], r[6]};
        twisty::RotateVectorByQuaternion(r, v);
        writev(o, v, 3);
    }
    return 0;
}

void write_cw(std::ofstream &o, const twisty::CombinedWeightValues_C &c)
{
    writev(o, &c.m_maxWeightLog10, 1);
    writev(o, &c.m_runningTotal, 1);
    writev(o, &c.m_offset, 1);
    uint32_t n[2] = {c.m_numValues, 0};
    writev(o, n, 2);
}

double extract_log10(const twisty::CombinedWeightValues_C &c)
{
    long double v = twisty::ExtractFinalValue(c);
    return (double)std::log10(v);
}

int mode_cw(int argc, char **argv)
{
    if (argc != 4) return 2;
    std::ifstream in(argv[2], std::ios::binary);
    uint64_t n = 0, split = 0;
    readv(in, &n, 1);
    readv(in, &split, 1);
    std::vector<double> v(n);
    readv(in, v.data(), n);
    twisty::CombinedWeightValues_C a, b;
    twisty::CombinedWeightValues_C_Reset(a);
    twisty::CombinedWeightValues_C_Reset(b);
    for (uint64_t i = 0; i < n; ++i) twisty::CombinedWeightValues_C_AddValue(i < split ? a : b, v[i]);
    twisty::CombinedWeightValues_C c = twisty::CombinedWeightValues_C_CombineValues(a, b);
    std::ofstream o(argv[3], std::ios::binary);
    write_cw(o, a);
    write_cw(o, b);
    write_cw(o, c);
    double e[3] = {extract_log10(a), extract_log10(b), extract_log10(c)};
    writev(o, e, 3);
    return 0;
}

int mode_norm(int argc, char **argv)
{
    if (argc != 16) return 2;
    const int N = atoi(argv[2]);
    const float ds = (float)atof(argv[3]);
    twisty::PerturbUtils::BoundaryConditions bc = bc_from(argv + 4, ds * N);
    long double v = twisty::PathWeighting::NormalizerStuff::Norm(N, ds, bc);
    printf("%.21Lg\n", std::log10(v));
    return 0;
}

int mode_bootstrap(int argc, char **argv)
{
    if (argc != 18) return 2;
    const uint32_t N = (uint32_t)atoi(argv[2]);
    const float S = (float)atof(argv[3]);
    twisty::PerturbUtils::BoundaryConditions bc = bc_from(argv + 4, S);
    const uint32_t seed = (uint32_t)strtoul(argv[16], nullptr, 10);
    twisty::Curve curve(N);
    curve.SetBoundaryConditions(bc);
    std::mt19937_64 g(seed);
    const float ds = S / N;
    twisty::PathGeneration::ResolveEvenNumberOfSegments(N - 2, curve.m_positions, 1, N - 1, ds, g);
    std::ofstream o(argv[17], std::ios::binary);
    for (auto &p : curve.m_positions) writev(o, p.m_data.data(), 3);
    return 0;
}

// The reference's independent-sample estimator MSegmentPathGenerationMC
// (Experiments/ExperimentBase.cpp:1246-1386) driven through the reference's own functions: per
// thread t a std::mt19937_64(seed + t) and a contiguous block of paths; per path the fixed points
// of :1253-1260, ResolveEvenNumberOfSegments (patched P2), tangents, curvatures (patched P3)
// and the reference weigher. A placement the reference would throw on marks the path invalid.
int mode_msegment(int argc, char **argv)
{
    if (argc != 23) return 2;
    Lut l = load_lut(argv[2]);
    const uint32_t N = (uint32_t)atoi(argv[3]);
    const float S = (float)atof(argv[4]);
    twisty::PerturbUtils::BoundaryConditions bc = bc_from(argv + 5, S);
    const float absorption = (float)atof(argv[17]);
    const uint64_t seed = strtoull(argv[18], nullptr, 10);
    const uint64_t P = strtoull(argv[19], nullptr, 10);
    const int T = atoi(argv[20]);
    (void)argv[21];
    const float ds = bc.arclength / N;
    const Farlor::Vector3 p0 = bc.m_startPos, p1 = bc.m_startPos + ds * bc.m_startDir;
    const Farlor::Vector3 pm = bc.m_endPos, pm1 = bc.m_endPos - ds * bc.m_endDir;
    std::vector<uint8_t> valid(P, 0);
    std::vector<double> w(P, 0.0);
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) {
        th.emplace_back([&, t] {
            std::mt19937_64 rng(seed + (uint64_t)t);
            const uint64_t a = P * (uint64_t)t / (uint64_t)T, b = P * (uint64_t)(t + 1) / (uint64_t)T;
            std::vector<Farlor::Vector3> pts(N + 1), tan(N);
            std::vector<float> curv(N - 1);
            for (uint64_t p = a; p < b; ++p) {
                pts[0] = p0;
                pts[1] = p1;
                pts[N - 1] = pm1;
                pts[N] = pm;
                try {
                    twisty::PathGeneration::ResolveEvenNumberOfSegments((int)N - 2, pts, 1, N - 1, ds, rng);
                } catch (const std::exception &) {
                    continue;
                }
                twisty::PerturbUtils::UpdateTangentsFromPos(pts.data(), tan.data(), N, bc);
                twisty::PerturbUtils::UpdateCurvaturesFromTangents_RadiativeTransfer(tan.data(), curv.data(), N, bc);
                twisty::PathWeighting::PathWeightValue r = twisty::PathWeighting::WeightCurveViaCurvatureLog10_CudaSafe(
                      curv.data(), N - 1, l.v.data(), (int32_t)l.bins, l.ds, l.minK, l.maxK, l.step, absorption);
                valid[p] = r.isValid ? 1 : 0;
                w[p] = r.weight;
            }
        });
    }
    for (auto &x : th) x.join();
    std::ofstream o(argv[22], std::ios::binary);
    for (uint64_t p = 0; p < P; ++p) {
        writev(o, &valid[p], 1);
        writev(o, &w[p], 1);
    }
    return 0;
}

int mode_chain(int argc, char **argv)
{
    if (argc != 7) return 2;
    nlohmann::json cfg;
    {
        std::ifstream f(argv[2]);
        f >> cfg;
    }
    twisty::ExperimentRunner::ExperimentParameters params
          = twisty::ExperimentRunner::ParseExperimentParamsFromConfig(cfg);
    params.experimentDirPath = std::string(getenv("TMPDIR") ? getenv("TMPDIR") : "/tmp") + "/twisty_ref_harness/";
    const int64_t T = atoll(argv[4]);
    params.numPathsInExperiment = (uint64_t)atoll(argv[5]);
    params.maxPerturbThreads = (int32_t)T;

    twisty::PerturbUtils::BoundaryConditions bc;
    auto &be = cfg["experiment"]["basicExperiment"];
    bc.m_startPos = Farlor::Vector3(be["startPos"][0], be["startPos"][1], be["startPos"][2]);
    bc.m_startDir = Farlor::Vector3(be["startDir"][0], be["startDir"][1], be["startDir"][2]).Normalized();
    bc.m_endPos = Farlor::Vector3(be["endPos"][0], be["endPos"][1], be["endPos"][2]);
    bc.m_endDir = Farlor::Vector3(be["endDir"][0], be["endDir"][1], be["endDir"][2]).Normalized();
    bc.arclength = be["arclength"];
    const uint32_t N = params.numSegmentsPerCurve;

    auto t0 = std::chrono::high_resolution_clock::now();
    const float ds = bc.arclength / N;
    WeightLookupTableIntegral lut(params.weightingParameters, ds);
    lut.Initialize();

    twisty::Curve initialCurve(N);
    initialCurve.SetBoundaryConditions(bc);
    if (std::string(argv[3]) == "-") {
        std::mt19937_64 g(params.bootstrapSeed);
        twisty::PathGeneration::ResolveEvenNumberOfSegments(N - 2, initialCurve.m_positions, 1, N - 1, ds, g);
    } else {
        std::ifstream f(argv[3], std::ios::binary);
        std::vector<float> raw((N + 1) * 3);
        readv(f, raw.data(), raw.size());
        for (uint32_t i = 0; i <= N; ++i)
            initialCurve.m_positions[i] = Farlor::Vector3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
    }
    std::vector<Farlor::Vector3> pos0 = initialCurve.m_positions, tan0(N);
    std::vector<float> curv0(N - 1);
    twisty::PerturbUtils::UpdateTangentsFromPos(pos0.data(), tan0.data(), N, bc);
    twisty::PerturbUtils::UpdateCurvaturesFromTangents_RadiativeTransfer(tan0.data(), curv0.data(), N, bc);

    std::vector<Farlor::Vector3> pos, tan;
    std::vector<float> curv;
    std::vector<std::mt19937_64> rng(T);
    int64_t seed = params.curvePurturbSeed;
    for (int64_t i = 0; i < T; ++i) {
        rng[i] = std::mt19937_64(seed + i);
        pos.insert(pos.end(), pos0.begin(), pos0.end());
        tan.insert(tan.end(), tan0.begin(), tan0.end());
        curv.insert(curv.end(), curv0.begin(), curv0.end());
    }
    const uint64_t P = params.numPathsInExperiment;
    const int64_t nCW = (P + MaxNumPathsPerCombinedWeight - 1) / MaxNumPathsPerCombinedWeight;
    const int64_t cwPerThread = (nCW + T - 1) / T;
    std::vector<twisty::CombinedWeightValues_C> cws(nCW);
    for (auto &c : cws) twisty::CombinedWeightValues_C_Reset(c);
    const long double norm = twisty::PathWeighting::NormalizerStuff::Norm(N, ds, bc);
    twisty::FullExperimentRunnerOptimalPerturb runner(params);
    {
        // GeometryRandom records every accepted path in file-static per-thread histograms
        // (Twisty/FullExperimentRunnerOptimalPerturb.cpp:26-37,562-575) that only
        // RunnerSpecificRunExperiment sizes (:235-246). Size them with a zero-path run of
        // that method on a small geometry its bootstrapper accepts (N=10); nothing else of
        // that run is used.
        twisty::ExperimentRunner::ExperimentParameters primeParams = params;
        primeParams.numPathsInExperiment = 0;
        primeParams.numSegmentsPerCurve = 10;
        twisty::FullExperimentRunnerOptimalPerturb primer(primeParams);
        twisty::PerturbUtils::BoundaryConditions pbc;
        pbc.m_startPos = Farlor::Vector3(0, 0, 0);
        pbc.m_startDir = Farlor::Vector3(1, 0, 0);
        pbc.m_endPos = Farlor::Vector3(5, 0, 0);
        pbc.m_endDir = Farlor::Vector3(1, 0, 0);
        pbc.arclength = 10.0f;
        primer.RunnerSpecificRunExperiment(pbc);
    }
    auto t1 = std::chrono::high_resolution_clock::now();
    {
        std::vector<std::thread> th;
        for (int64_t t = 0; t < T; ++t) {
            th.emplace_back([&, t]() {
                runner.GeometryRandom(t, P, MaxNumPathsPerCombinedWeight * cwPerThread,
                      (uint32_t)params.numPathsToSkip, N, rng, pos, tan, curv, cws, ds,
                      lut.AccessLookupTable().data(), (uint32_t)lut.AccessLookupTable().size(),
                      lut.GetDs(), lut.GetMinCurvature(), lut.GetMaxCurvature(),
                      lut.GetCurvatureStepSize(), bc);
            });
        }
        for (auto &x : th) x.join();
    }
    auto t2 = std::chrono::high_resolution_clock::now();
    long double total = 0.0L;
    uint64_t paths = 0;
    nlohmann::json out;
    out["chunk_log10"] = nlohmann::json::array();
    out["chunk_paths"] = nlohmann::json::array();
    for (auto &c : cws) {
        long double e = twisty::ExtractFinalValue(c);
        total += e;
        paths += c.m_numValues;
        out["chunk_log10"].push_back(c.m_numValues ? (double)std::log10(e) : -1e308);
        out["chunk_paths"].push_back(c.m_numValues);
    }
    total *= norm;
    out["log10_weight"] = (double)std::log10(total);
    out["log10_normalizer"] = (double)std::log10(norm);
    out["paths"] = paths;
    out["threads"] = T;
    out["chunks_per_thread"] = cwPerThread;
    out["setup_ms"] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    out["perturb_ms"] = std::chrono::duration<double, std::milli>(t2 - t1).count();
    out["num_segments"] = N;
    std::ofstream o(argv[6]);
    o << out.dump(1) << std::endl;
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: ref_harness lut|weigh|rotate|cw|norm|bootstrap|chain ...\n");
        return 2;
    }
    std::string m = argv[1];
    try {
        int rc = 2;
        if (m == "lut") rc = mode_lut(argc, argv);
        else if (m == "weigh") rc = mode_weigh(argc, argv);
        else if (m == "rotate") rc = mode_rotate(argc, argv);
        else if (m == "cw") rc = mode_cw(argc, argv);
        else if (m == "norm") rc = mode_norm(argc, argv);
        else if (m == "bootstrap") rc = mode_bootstrap(argc, argv);
        else if (m == "chain") rc = mode_chain(argc, argv);
        else if (m == "msegment") rc = mode_msegment(argc, argv);
        if (rc == 2) fprintf(stderr, "bad arguments for mode %s\n", m.c_str());
        return rc;
    } catch (std::exception &e) {
        fprintf(stderr, "error: %s\n", e.what());
        return 3;
    }
}
