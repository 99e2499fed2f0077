// host_util.h -- host-side pieces of the runner that need no device: config parsing,
// initial-curve construction, geometry checks, the closed-form normaliser.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/twisty_b200.h"

namespace twisty {

// A tiny document model shared by the JSON and YAML readers.
struct Node {
    enum Kind { Null, Bool, Number, String, Object, Array } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::map<std::string, Node> obj;
    std::vector<Node> arr;
    const Node *get(const std::string &k) const;
};

bool parse_json(const std::string &text, Node &out, std::string &err);
bool parse_yaml(const std::string &text, Node &out, std::string &err);

// Fill params/bc from a parsed config (reference schema: experiment.experimentParams.*,
// experiment.basicExperiment.*). Returns false with err set when a required key is
// missing or has the wrong type.
bool params_from_node(const Node &root, twisty_params &p, twisty_bc *bc, std::string &err);

// CalculateMinimumArclength (Twisty/PathGeneration.cpp:12-43).
float min_arclength(const twisty_bc &bc, uint32_t n);

// Initial curve for any N >= 4: points 0, 1, N-1, N fixed by the boundary conditions
// (Twisty/Curve.cpp:20-30), the N-2 free segments laid on a planar circular arc from
// point 1 to point N-1 whose turning angle is solved by bisection so that every segment
// has length exactly ds (computed in double, stored in float). The arc's plane is turned
// about the chord by an angle drawn from the bootstrap seed. Returns false (err set) when
// |x_{N-1} - x_1| > (N-2) ds.
bool bootstrap_arc(const twisty_bc &bc, uint32_t n, uint32_t seed, std::vector<float> &pos, std::string &err);

// The reference's recursive bootstrapper (Twisty/PathGeneration.cpp:47-414 from the call at
// FullExperimentRunnerOptimalPerturb.cpp:122-131) for N with N-2 in {4, 6, 8, 12, 16, 24, 32,
// 48, ...}: the same random stream and arithmetic, the reference's curve for the same
// bootstrapSeed. Returns false (err set) for other N or when the placement fails.
bool bootstrap_resolvable(uint32_t n);
bool bootstrap_reference(const twisty_bc &bc, uint32_t n, uint32_t seed, std::vector<float> &pos, std::string &err);
// kind 0: the reference bootstrapper where it resolves N, else the arc; 1: the reference's
// only; 2: the arc.
bool bootstrap_curve(const twisty_bc &bc, uint32_t n, uint32_t seed, int kind, std::vector<float> &pos, std::string &err);

// The reference's table, rounding for rounding: WeightLookupTableIntegral ctor + Initialize
// (Twisty/PathWeightUtils.cpp:281-348) with Integrate's sorted sum (:371-433) and the float
// phase function (:19-33), on host threads. Bins whose integral cancels to a tiny fraction
// of its terms keep the reference's summation-order rounding only this way, so the
// faithful table mode (the drop-in's bit-parity setup) is built here; the FP64 tables are
// built on the device. out[bins]; minmax = {min, max} weight. Returns false on bad params.
bool lut_faithful_host(float mu, float eps, float scatter, float min_bound, float max_bound, float bias,
                       uint32_t num_steps_int, uint32_t bins, float ds, float *out, float minmax[2]);

// Tables of the compensated form, from the float weight table lut[bins] with bin width
// `step` (curvature units), for paths of n_segments segments:
//  * lin[2*bins]: per bin (L_i, L_{i+1} - L_i) for the exact blend;
//  * fix[2*bins]: per bin (round((log10 L_i - c0) 2^s) as uint32 bits, the change of log10
//    of the blend across the bin, log10(1 + step (L_{i+1}/L_i - 1)), as float), with
//    c0 = min log10 L_i - 64 2^-s so that every entry is at least 64 and a path total
//    stays positive under rounded corrections, and (n_segments + 1) * max entry < 2^31 so
//    that a path total and the difference of two totals are exact in 32 bits (narrow);
//    when that leaves fewer than 22 fraction bits, 32 * max entry < 2^32 (wide = 1: exact
//    32-bit lane sums of up to 32 entries, 64-bit path totals).
// The secant's worst per-segment error in bin i is (step a)^2 / (8 ln 10) with
// a = L_{i+1}/L_i - 1. Bins where it exceeds kSecantBound are steep: their slope is stored
// as NaN, so a path crossing one is flagged and re-weighed through lin by the kernels;
// steep = their count, secant_err = the worst error over the other bins. Returns false (fix
// unusable, the exact blend is needed) when an entry is not positive, more than
// bins / kSteepFraction bins are steep, or fewer than 22 fraction bits fit either way.
constexpr double kSecantBound = 1e-7;
constexpr uint32_t kSteepFraction = 16;
bool compensated_tables(const float *lut, uint32_t bins, float step, uint32_t n_segments, std::vector<float> &lin,
                        std::vector<float> &fix, double &c0, double &inv_scale, int &wide, double &secant_err,
                        uint32_t &steep);

// K4 (Twisty/PathWeightUtils.cpp:643-651) and the z of Norm (:729-732), float math.
double norm_k4_log10(float z, float ds);
float norm_z(const twisty_bc &bc, float ds);

}  // namespace twisty
