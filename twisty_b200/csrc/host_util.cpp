// host_util.cpp -- config readers, initial curve, geometry checks, closed-form normaliser.
#include "host_util.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <limits>
#include <cstdlib>
#include <cstring>
#include <random>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace twisty {

const Node *Node::get(const std::string &k) const
{
    if (kind != Object) return nullptr;
    auto it = obj.find(k);
    return it == obj.end() ? nullptr : &it->second;
}

// ------------------------------------------------------------------------- JSON
namespace {

struct JsonReader {
    const std::string &s;
    size_t i = 0;
    std::string err;
    explicit JsonReader(const std::string &t) : s(t) {}

    void ws()
    {
        while (i < s.size()) {
            if (std::isspace((unsigned char)s[i])) { ++i; continue; }
            // The reference's sample configs are plain JSON; tolerate // and /* */ comments.
            if (s[i] == '/' && i + 1 < s.size() && s[i + 1] == '/') {
                while (i < s.size() && s[i] != '\n') ++i;
                continue;
            }
            if (s[i] == '/' && i + 1 < s.size() && s[i + 1] == '*') {
                const size_t e = s.find("*/", i + 2);
                i = (e == std::string::npos) ? s.size() : e + 2;
                continue;
            }
            break;
        }
    }
    bool fail(const std::string &m)
    {
        if (err.empty()) {
            std::ostringstream o;
            o << m << " at offset " << i;
            err = o.str();
        }
        return false;
    }
    bool str(std::string &out)
    {
        if (s[i] != '"') return fail("expected string");
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            char ch = s[i++];
            if (ch == '\\' && i < s.size()) {
                const char e = s[i++];
                switch (e) {
                    case 'n': ch = '\n'; break;
                    case 't': ch = '\t'; break;
                    case 'r': ch = '\r'; break;
                    case 'b': ch = '\b'; break;
                    case 'f': ch = '\f'; break;
                    case 'u': {
                        if (i + 4 > s.size()) return fail("bad escape");
                        const unsigned v = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
                        i += 4;
                        ch = v < 128 ? (char)v : '?';
                    } break;
                    default: ch = e; break;
                }
            }
            out.push_back(ch);
        }
        if (i >= s.size()) return fail("unterminated string");
        ++i;
        return true;
    }
    bool value(Node &n)
    {
        ws();
        if (i >= s.size()) return fail("unexpected end");
        const char ch = s[i];
        if (ch == '{') {
            ++i;
            n.kind = Node::Object;
            ws();
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!str(k)) return false;
                ws();
                if (i >= s.size() || s[i] != ':') return fail("expected ':'");
                ++i;
                Node v;
                if (!value(v)) return false;
                n.obj[k] = std::move(v);
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == '}') { ++i; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (ch == '[') {
            ++i;
            n.kind = Node::Array;
            ws();
            if (i < s.size() && s[i] == ']') { ++i; return true; }
            for (;;) {
                Node v;
                if (!value(v)) return false;
                n.arr.push_back(std::move(v));
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == ']') { ++i; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (ch == '"') {
            n.kind = Node::String;
            return str(n.str);
        }
        if (s.compare(i, 4, "true") == 0) { n.kind = Node::Bool; n.b = true; i += 4; return true; }
        if (s.compare(i, 5, "false") == 0) { n.kind = Node::Bool; n.b = false; i += 5; return true; }
        if (s.compare(i, 4, "null") == 0) { n.kind = Node::Null; i += 4; return true; }
        const char *b = s.c_str() + i;
        char *e = nullptr;
        const double v = std::strtod(b, &e);
        if (e == b) return fail("bad value");
        n.kind = Node::Number;
        n.num = v;
        i += (size_t)(e - b);
        return true;
    }
};

// ------------------------------------------------------------------------- YAML subset
// Block mappings by indentation, "key: scalar", "key:" followed by a deeper block, flow
// sequences "[a, b, c]", block sequences "- item", '#' comments, quoted strings.
struct YamlLine {
    int indent;
    std::string text;
};

std::string trim(const std::string &x)
{
    size_t a = 0, b = x.size();
    while (a < b && std::isspace((unsigned char)x[a])) ++a;
    while (b > a && std::isspace((unsigned char)x[b - 1])) --b;
    return x.substr(a, b - a);
}

std::string strip_comment(const std::string &x)
{
    bool sq = false, dq = false;
    for (size_t i = 0; i < x.size(); ++i) {
        if (x[i] == '\'' && !dq) sq = !sq;
        else if (x[i] == '"' && !sq) dq = !dq;
        else if (x[i] == '#' && !sq && !dq && (i == 0 || std::isspace((unsigned char)x[i - 1]))) return x.substr(0, i);
    }
    return x;
}

Node yaml_scalar(const std::string &raw)
{
    Node n;
    const std::string v = trim(raw);
    if (v.empty() || v == "~" || v == "null") return n;
    if (v == "true" || v == "True") { n.kind = Node::Bool; n.b = true; return n; }
    if (v == "false" || v == "False") { n.kind = Node::Bool; n.b = false; return n; }
    if ((v.front() == '"' && v.back() == '"') || (v.front() == '\'' && v.back() == '\'')) {
        n.kind = Node::String;
        n.str = v.substr(1, v.size() - 2);
        return n;
    }
    if (v.front() == '[' && v.back() == ']') {
        n.kind = Node::Array;
        std::string inner = v.substr(1, v.size() - 2), cur;
        int depth = 0;
        for (char ch : inner) {
            if (ch == '[') ++depth;
            if (ch == ']') --depth;
            if (ch == ',' && depth == 0) {
                n.arr.push_back(yaml_scalar(cur));
                cur.clear();
            } else {
                cur.push_back(ch);
            }
        }
        if (!trim(cur).empty()) n.arr.push_back(yaml_scalar(cur));
        return n;
    }
    char *e = nullptr;
    const double d = std::strtod(v.c_str(), &e);
    if (e && *e == '\0') {
        n.kind = Node::Number;
        n.num = d;
        return n;
    }
    n.kind = Node::String;
    n.str = v;
    return n;
}

bool yaml_block(const std::vector<YamlLine> &ls, size_t &i, int indent, Node &out, std::string &err)
{
    if (i < ls.size() && ls[i].text.rfind("- ", 0) == 0 && ls[i].indent == indent) {
        out.kind = Node::Array;
        while (i < ls.size() && ls[i].indent == indent && ls[i].text.rfind("- ", 0) == 0) {
            out.arr.push_back(yaml_scalar(ls[i].text.substr(2)));
            ++i;
        }
        return true;
    }
    out.kind = Node::Object;
    while (i < ls.size()) {
        const YamlLine &l = ls[i];
        if (l.indent < indent) return true;
        if (l.indent > indent) {
            err = "unexpected indentation: " + l.text;
            return false;
        }
        const size_t c = l.text.find(':');
        if (c == std::string::npos) {
            err = "expected 'key: value': " + l.text;
            return false;
        }
        std::string key = trim(l.text.substr(0, c));
        if (key.size() >= 2 && (key.front() == '"' || key.front() == '\'')) key = key.substr(1, key.size() - 2);
        const std::string rest = trim(l.text.substr(c + 1));
        ++i;
        if (!rest.empty()) {
            out.obj[key] = yaml_scalar(rest);
        } else if (i < ls.size() && ls[i].indent > indent) {
            Node child;
            if (!yaml_block(ls, i, ls[i].indent, child, err)) return false;
            out.obj[key] = std::move(child);
        } else {
            out.obj[key] = Node();
        }
    }
    return true;
}

}  // namespace

bool parse_json(const std::string &text, Node &out, std::string &err)
{
    JsonReader r(text);
    if (!r.value(out)) {
        err = r.err;
        return false;
    }
    r.ws();
    if (r.i != text.size()) {
        err = "trailing characters after JSON value";
        return false;
    }
    return true;
}

bool parse_yaml(const std::string &text, Node &out, std::string &err)
{
    std::vector<YamlLine> ls;
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        const std::string t = strip_comment(line);
        if (trim(t).empty() || trim(t) == "---") continue;
        int ind = 0;
        while (ind < (int)t.size() && t[ind] == ' ') ++ind;
        if (ind < (int)t.size() && t[ind] == '\t') {
            err = "tabs are not allowed for indentation";
            return false;
        }
        ls.push_back({ind, trim(t)});
    }
    size_t i = 0;
    if (ls.empty()) {
        out.kind = Node::Object;
        return true;
    }
    if (!yaml_block(ls, i, ls[0].indent, out, err)) return false;
    if (i != ls.size()) {
        err = "could not parse line: " + ls[i].text;
        return false;
    }
    return true;
}

namespace {

bool need(const Node *n, Node::Kind k, const char *path, std::string &err)
{
    if (!n || n->kind != k) {
        err = std::string("config key missing or of the wrong type: ") + path;
        return false;
    }
    return true;
}

bool num(const Node *parent, const char *key, const char *path, double &out, std::string &err)
{
    const Node *n = parent ? parent->get(key) : nullptr;
    if (n && n->kind == Node::Bool) { out = n->b ? 1.0 : 0.0; return true; }
    if (!need(n, Node::Number, path, err)) return false;
    out = n->num;
    return true;
}

bool vec3(const Node *parent, const char *key, const char *path, float v[3], std::string &err)
{
    const Node *n = parent ? parent->get(key) : nullptr;
    if (!need(n, Node::Array, path, err)) return false;
    if (n->arr.size() != 3) {
        err = std::string("expected 3 numbers: ") + path;
        return false;
    }
    for (int i = 0; i < 3; ++i) {
        if (n->arr[i].kind != Node::Number) {
            err = std::string("expected 3 numbers: ") + path;
            return false;
        }
        v[i] = (float)n->arr[i].num;
    }
    return true;
}

twisty_vec3 normalized(const float v[3])
{
    const float inv = 1.0f / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    return twisty_vec3{v[0] * inv, v[1] * inv, v[2] * inv};
}

}  // namespace

bool params_from_node(const Node &root, twisty_params &p, twisty_bc *bc, std::string &err)
{
    const Node *ex = root.get("experiment");
    if (!need(ex, Node::Object, "experiment", err)) return false;
    const Node *ep = ex->get("experimentParams");
    if (!need(ep, Node::Object, "experiment.experimentParams", err)) return false;
    double v;
    // ParseExperimentParamsFromConfig (Twisty/ExperimentRunner.cpp:55-171), key for key.
    if (!num(ep, "pathsToGenerate", "experimentParams.pathsToGenerate", v, err)) return false;
    p.paths_to_generate = (uint64_t)v;
    if (!num(ep, "pathsToSkip", "experimentParams.pathsToSkip", v, err)) return false;
    p.paths_to_skip = (uint64_t)v;
    if (!num(ep, "numSegments", "experimentParams.numSegments", v, err)) return false;
    p.num_segments = (uint32_t)v;
    const Node *rnd = ep->get("random");
    if (!need(rnd, Node::Object, "experimentParams.random", err)) return false;
    if (!num(rnd, "bootstrapSeed", "random.bootstrapSeed", v, err)) return false;
    p.bootstrap_seed = (uint32_t)(int64_t)v;
    if (!num(rnd, "perturbSeed", "random.perturbSeed", v, err)) return false;
    p.perturb_seed = (uint32_t)(int64_t)v;
    const Node *w = ep->get("weighting");
    if (!need(w, Node::Object, "experimentParams.weighting", err)) return false;
    if (!num(w, "weightFunction", "weighting.weightFunction", v, err)) return false;
    p.weight_function = ((int)v == 1) ? 1 : 0;
    if (!num(ep, "perturbMethod", "experimentParams.perturbMethod", v, err)) return false;
    p.perturb_method = ((int)v == 1 || (int)v == 2) ? (int)v : 0;
    if (!num(w, "mu", "weighting.mu", v, err)) return false;
    p.mu = (float)v;
    if (!num(w, "eps", "weighting.eps", v, err)) return false;
    p.eps = (float)v;
    if (!num(w, "numStepsInt", "weighting.numStepsInt", v, err)) return false;
    p.num_steps_int = (uint32_t)v;
    if (!num(w, "numCurvatureSteps", "weighting.numCurvatureSteps", v, err)) return false;
    p.num_curvature_steps = (uint32_t)v;
    if (!num(w, "absorption", "weighting.absorption", v, err)) return false;
    p.absorption = (float)v;
    if (p.weight_function == 1) p.absorption = 0.0f;  // ExperimentRunner.cpp:157-162
    if (!num(w, "scatter", "weighting.scatter", v, err)) return false;
    p.scatter = (float)v;
    p.min_bound = 0.0f;
    p.max_bound = 10.0f / p.eps;  // ExperimentRunner.cpp:169-171
    // Optional B200 block: experimentParams.b200 { form, lutMode, maxSubChain, maxAngle, numChains, device,
    // compGroup, compSpl, compWarps, incrementalResync, compTableMemory }
    if (const Node *b = ep->get("b200")) {
        if (b->kind != Node::Object) {
            err = "experimentParams.b200 must be a mapping";
            return false;
        }
        if (b->get("form") && num(b, "form", "b200.form", v, err)) p.form = (int32_t)v;
        if (b->get("lutMode") && num(b, "lutMode", "b200.lutMode", v, err)) p.lut_mode = (int32_t)v;
        if (b->get("maxSubChain") && num(b, "maxSubChain", "b200.maxSubChain", v, err)) p.max_sub_chain = (uint32_t)v;
        if (b->get("maxAngle") && num(b, "maxAngle", "b200.maxAngle", v, err)) p.max_angle = (float)v;
        if (b->get("numChains") && num(b, "numChains", "b200.numChains", v, err)) p.num_chains = (uint32_t)v;
        if (b->get("device") && num(b, "device", "b200.device", v, err)) p.device = (int32_t)v;
        if (b->get("compGroup") && num(b, "compGroup", "b200.compGroup", v, err)) p.comp_group = (uint32_t)v;
        if (b->get("compSpl") && num(b, "compSpl", "b200.compSpl", v, err)) p.comp_spl = (uint32_t)v;
        if (b->get("compWarps") && num(b, "compWarps", "b200.compWarps", v, err)) p.comp_warps = (uint32_t)v;
        if (b->get("incrementalResync") && num(b, "incrementalResync", "b200.incrementalResync", v, err))
            p.incremental_resync = (uint32_t)v;
        if (b->get("compTableMemory") && num(b, "compTableMemory", "b200.compTableMemory", v, err))
            p.comp_table_memory = (uint32_t)v;
        if (!err.empty()) return false;
    }
    if (bc) {
        // Experiments/FullExperiment.cpp:162-191: directions are normalised
        const Node *be = ex->get("basicExperiment");
        if (!need(be, Node::Object, "experiment.basicExperiment", err)) return false;
        float a[3];
        if (!vec3(be, "startPos", "basicExperiment.startPos", a, err)) return false;
        bc->start_pos = twisty_vec3{a[0], a[1], a[2]};
        if (!vec3(be, "startDir", "basicExperiment.startDir", a, err)) return false;
        bc->start_dir = normalized(a);
        if (!vec3(be, "endPos", "basicExperiment.endPos", a, err)) return false;
        bc->end_pos = twisty_vec3{a[0], a[1], a[2]};
        if (!vec3(be, "endDir", "basicExperiment.endDir", a, err)) return false;
        bc->end_dir = normalized(a);
        if (!num(be, "arclength", "basicExperiment.arclength", v, err)) return false;
        bc->arclength = (float)v;
    }
    return true;
}

float min_arclength(const twisty_bc &bc, uint32_t n)
{
    const float M = (float)n;
    const float nsx = bc.start_dir.x + bc.end_dir.x, nsy = bc.start_dir.y + bc.end_dir.y,
                nsz = bc.start_dir.z + bc.end_dir.z;
    const float dx = bc.end_pos.x - bc.start_pos.x, dy = bc.end_pos.y - bc.start_pos.y,
                dz = bc.end_pos.z - bc.start_pos.z;
    const float a = (nsx * nsx + nsy * nsy + nsz * nsz) - ((M - 4.0f) * M + 4.0f);
    const float b = -2.0f * M * (nsx * dx + nsy * dy + nsz * dz);
    const float c = M * M * (dx * dx + dy * dy + dz * dz);
    const float r1 = (-b - std::sqrt(b * b - 4.0f * a * c)) / (2.0f * a);
    const float r2 = (-b + std::sqrt(b * b - 4.0f * a * c)) / (2.0f * a);
    float m = 1000000.0f;
    if (!std::isnan(r1) && r1 > 0.0f) m = std::min(m, r1);
    if (!std::isnan(r2) && r2 > 0.0f) m = std::min(m, r2);
    return m;
}

// ------------------------------------------------------------ reference bootstrapper
// The reference's recursive random placement (Twisty/PathGeneration.cpp:47-414, entered from
// FullExperimentRunnerOptimalPerturb.cpp:122-131) restated with its random stream
// (std::mt19937_64 seeded with bootstrapSeed and the standard library's distributions, drawn in
// the same order) and its float/double arithmetic (FMath-style float vectors; products of a
// vector and a double scalar convert the scalar to float; Normalized = v * (1/sqrt(v.v))), so
// that the same compiler and math library reproduce the reference's curves bit for bit.
namespace {

struct V3 {
    float x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
inline V3 operator*(float s, V3 a) { return a * s; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float mag(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 unit(V3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }

constexpr float kPiF = 3.141592653589793f;

// The reference's quaternion product (RotateQuatByQuat, Twisty/CurvePerturbUtils.cpp:91-111):
// r = A (x) B with its own sign convention, each component summed left to right in float.
void quat_product(const float A[4], const float B[4], float r[4])
{
    const float t0 = A[0] * B[0] - A[1] * B[1] - A[2] * B[2] - A[3] * B[3];
    const float t1 = A[0] * B[1] + A[1] * B[0] - A[2] * B[3] + A[3] * B[2];
    const float t2 = A[0] * B[2] + A[1] * B[3] + A[2] * B[0] - A[3] * B[1];
    const float t3 = A[0] * B[3] - A[1] * B[2] + A[2] * B[1] + A[3] * B[0];
    r[0] = t0;
    r[1] = t1;
    r[2] = t2;
    r[3] = t3;
}

// RotateVectorByQuaternion (:113-127): p = (0, v); p = p (x) q; p = q^-1 (x) p; v = p.xyz.
void rotate_by_quaternion(const float q[4], V3 &v)
{
    float p[4] = {0.0f, v.x, v.y, v.z};
    const float qi[4] = {q[0], -q[1], -q[2], -q[3]};
    quat_product(p, q, p);
    quat_product(qi, p, p);
    v = V3{p[1], p[2], p[3]};
}

// An orthonormal frame around the axis from a to b (the reference picks the helper vector
// (1,0,0), or (0,1,0) when the axis is within 0.999 of it).
void frame(V3 a, V3 b, V3 &xa, V3 &ya, V3 &za)
{
    za = unit(b - a);
    V3 r{1.0f, 0.0f, 0.0f};
    if (std::abs(dot(za, r)) > 0.999f) r = V3{0.0f, 1.0f, 0.0f};
    xa = unit(cross(za, r));
    ya = unit(cross(za, xa));
}

// ResolveTwoSegments: the one point between pts[l] and pts[l+2].
void resolve_two(std::vector<V3> &pts, size_t l, size_t r, double ds, std::mt19937_64 &rng)
{
    const V3 a = pts[l], b = pts[r];
    V3 &out = pts[l + 1];
    const float d = mag(b - a);
    if (std::abs((2.0f * ds) - d) < 0.001f) {
        out = (a + b) * 0.5f;
        return;
    }
    if ((2.0f * ds) < d) throw std::runtime_error("spheres do not intersect (two segments)");
    std::uniform_real_distribution<float> theta_d(0.0f, 2.0f * kPiF);
    const float theta = theta_d(rng);
    if (d < 0.001f) {
        std::uniform_real_distribution<float> u(0, 1);
        const float phi = std::acos(1.0 - 2.0 * u(rng));
        out = a + V3{std::sin(phi) * std::cos(theta), std::sin(phi) * std::sin(theta), std::cos(phi)} * (float)ds;
        return;
    }
    const V3 mid = (a + b) * (float)0.5;
    const V3 axis = unit(b - a);
    V3 helper{1.0f, 0.0f, 0.0f};
    if (std::abs(dot(axis, helper)) >= 0.99) helper = V3{0.0f, 1.0f, 0.0f};
    const V3 normal = unit(cross(axis, helper));
    const float half = d * 0.5f;
    float off = 0.0f;
    if (ds > half) off = (float)std::sqrt((ds * ds) - (half * half));
    V3 pt = mid + normal * off;
    const float s = std::sin(theta / 2.0f);
    const float q[4] = {std::cos(theta / 2.0f), axis.x * s, axis.y * s, axis.z * s};
    V3 shifted = pt - a;
    rotate_by_quaternion(q, shifted);
    out = shifted + a;
}

// ResolveThreeSegments: the two points between pts[l] and pts[l+3].
void resolve_three(std::vector<V3> &pts, size_t l, size_t r, double ds, std::mt19937_64 &rng)
{
    const V3 a = pts[l], b = pts[r];
    V3 &first = pts[l + 1];
    const float d = mag(b - a);
    if (std::abs((3.0f * ds) - d) < 0.001f) {
        first = a + (b - a) * (1.0f / 3.0f);
        resolve_two(pts, l + 1, r, ds, rng);
        return;
    }
    if ((3.0f * ds) < d) throw std::runtime_error("spheres do not intersect (three segments)");
    std::uniform_real_distribution<float> theta_d(0.0f, 2.0f * kPiF);
    const float theta = theta_d(rng);
    if (d < 0.001f) {
        std::uniform_real_distribution<float> u(0, 1);
        const float phi = std::acos(1.0 - 2.0 * u(rng));
        first = a + V3{std::sin(phi) * std::cos(theta), std::sin(phi) * std::sin(theta), std::cos(phi)} * (float)ds;
        resolve_two(pts, l + 1, r, ds, rng);
        return;
    }
    V3 xa, ya, za;
    frame(a, b, xa, ya, za);
    const double d2 = d * d;
    const double r1 = ds, r1s = r1 * r1;
    const double r2 = 2.0f * ds, r2s = r2 * r2;
    double extent = 0.0;
    if ((d + r1) < r2) {
        extent = kPiF;
    } else {
        const double h = 0.5 + (r1s - r2s) / (2.0 * d2);
        double aa = 0.0;
        if (std::abs(r1s - (h * h * d2)) >= 0.001) aa = std::sqrt(r1s - (h * h * d2));
        extent = (h * d < 0.0f) ? kPiF - std::asin(aa / r1) : std::asin(aa / r1);
        if (extent != extent) throw std::runtime_error("phi extent is NaN (three segments)");
    }
    const float umax = 0.5f - std::cos(extent) * 0.5f;
    std::uniform_real_distribution<double> phi_d(0, umax);
    const double phi = std::acos(1.0 - 2.0 * phi_d(rng));
    const V3 dir = xa * (float)std::sin(phi) * std::cos(theta) + ya * (float)std::sin(phi) * std::sin(theta) +
                   za * (float)std::cos(phi);
    first = a + unit(dir) * (float)ds;
    resolve_two(pts, l + 1, r, ds, rng);
}

bool resolvable(int m)
{
    if (m % 2) return false;
    const int h = m / 2;
    return h == 2 || h == 3 || (h % 2 == 0 && resolvable(h));
}

// ResolveEvenNumberOfSegments: the centre point of m segments, then each half.
void resolve_even(int m, std::vector<V3> &pts, size_t l, size_t r, double ds, std::mt19937_64 &rng)
{
    if (m % 2) throw std::runtime_error("even number of segments required");
    const int h = m / 2;
    if (h != 3 && h != 2 && (h % 2) != 0) throw std::runtime_error("segments per side must be 2, 3 or even");
    const V3 a = pts[l], b = pts[r];
    const size_t c = l + h;
    auto halves = [&]() {
        if (h == 2) {
            resolve_two(pts, l, c, ds, rng);
            resolve_two(pts, c, r, ds, rng);
        } else if (h == 3) {
            resolve_three(pts, l, c, ds, rng);
            resolve_three(pts, c, r, ds, rng);
        } else {
            resolve_even(h, pts, l, c, ds, rng);
            resolve_even(h, pts, c, r, ds, rng);
        }
    };
    const double d = mag(b - a);
    if (std::abs((m * ds) - d) < 0.001f) {
        pts[c] = 0.5f * (b + a);
        halves();
        return;
    }
    const double rad = ds * h;
    if ((rad + rad) < d) throw std::runtime_error("spheres do not intersect");
    if (d < 0.001f) {
        std::uniform_real_distribution<double> phi_d(0, 1);
        std::uniform_real_distribution<double> theta_d(0.0f, 2.0f * kPiF);
        std::uniform_real_distribution<float> u(0.0f, 1.0f);
        const double phi = std::acos(1.0 - 2.0 * phi_d(rng));
        const double theta = theta_d(rng);
        const double sr = rad * std::pow(u(rng), 1.0 / 3.0);
        V3 xa, ya, za;
        frame(a, b, xa, ya, za);
        V3 off = xa * (float)std::sin(phi) * (float)std::cos(theta) + ya * (float)std::sin(phi) * (float)std::sin(theta) +
                 za * (float)std::cos(phi);
        off = off * (float)sr;
        pts[c] = a + off;
        halves();
        return;
    }
    const double d2 = d * d;
    const double rad2 = rad * rad;
    const V3 mid = 0.5f * (b + a);
    const double to_mid = mag(mid - a);
    const double hh = 0.5;
    const double aa = std::sqrt(rad2 - (hh * hh * d2));
    const double extent = std::asin(aa / rad);
    std::uniform_int_distribution<int> coin(0, 1);
    const float umax = 0.5f - std::cos(extent) * 0.5f;
    std::uniform_real_distribution<double> phi_d(0, umax);
    std::uniform_real_distribution<double> theta_d(0.0f, 2.0f * kPiF);
    std::uniform_real_distribution<float> u(0.0f, 1.0f);
    const double phi = std::acos(1.0 - 2.0 * phi_d(rng));
    const double theta = theta_d(rng);
    const bool flip = coin(rng);
    const double hyp = to_mid / std::cos(phi);
    const double maxr = h * ds;
    const double minp = hyp / maxr;
    const double sr = maxr * std::pow(minp + (1.0f - minp) * u(rng), 1.0 / 3.0);
    V3 xa, ya, za;
    frame(a, b, xa, ya, za);
    if (!flip) {
        V3 off = xa * (float)std::sin(phi) * (float)std::cos(theta) + ya * (float)std::sin(phi) * (float)std::sin(theta) +
                 za * (float)std::cos(phi);
        off = off * (float)sr;
        pts[c] = a + off;
    } else {
        V3 off = xa * (float)std::sin(phi) * (float)std::cos(theta) + ya * (float)std::sin(phi) * (float)std::sin(theta) +
                 za * (float)std::cos(phi) * -1.0f;
        off = off * (float)sr;
        pts[c] = b + off;
    }
    halves();
}

}  // namespace

bool bootstrap_resolvable(uint32_t n) { return n >= 6 && resolvable((int)n - 2); }

bool bootstrap_reference(const twisty_bc &bc, uint32_t n, uint32_t seed, std::vector<float> &pos, std::string &err)
{
    if (!bootstrap_resolvable(n)) {
        err = "the reference bootstrapper resolves N-2 in {4, 6, 8, 12, 16, 24, 32, 48, ...} only";
        return false;
    }
    // Curve::SetBoundaryConditions (Twisty/Curve.cpp:20-30): points 0, 1, N-1, N fixed
    const float ds = bc.arclength / (float)n;
    std::vector<V3> pts(n + 1, V3{0.0f, 0.0f, 0.0f});
    const V3 sp{bc.start_pos.x, bc.start_pos.y, bc.start_pos.z}, sd{bc.start_dir.x, bc.start_dir.y, bc.start_dir.z};
    const V3 ep{bc.end_pos.x, bc.end_pos.y, bc.end_pos.z}, ed{bc.end_dir.x, bc.end_dir.y, bc.end_dir.z};
    pts[0] = sp;
    pts[1] = sp + sd * ds;
    pts[n - 1] = ep - ed * ds;
    pts[n] = ep;
    std::mt19937_64 rng(seed);
    try {
        resolve_even((int)n - 2, pts, 1, n - 1, ds, rng);
    } catch (const std::exception &e) {
        err = std::string("reference bootstrapper: ") + e.what();
        return false;
    }
    pos.resize(3 * (size_t)(n + 1));
    for (uint32_t i = 0; i <= n; ++i) {
        pos[3 * i] = pts[i].x;
        pos[3 * i + 1] = pts[i].y;
        pos[3 * i + 2] = pts[i].z;
    }
    return true;
}

bool bootstrap_curve(const twisty_bc &bc, uint32_t n, uint32_t seed, int kind, std::vector<float> &pos, std::string &err)
{
    if (kind == 1 || (kind == 0 && bootstrap_resolvable(n))) return bootstrap_reference(bc, n, seed, pos, err);
    if (kind != 0 && kind != 2) {
        err = "unknown bootstrap_kind";
        return false;
    }
    return bootstrap_arc(bc, n, seed, pos, err);
}

bool bootstrap_arc(const twisty_bc &bc, uint32_t n, uint32_t seed, std::vector<float> &pos, std::string &err)
{
    if (n < 4) {
        err = "numSegments must be at least 4";
        return false;
    }
    const float ds = bc.arclength / (float)n;
    pos.assign(3 * (size_t)(n + 1), 0.0f);
    auto set = [&](uint32_t i, float x, float y, float z) {
        pos[3 * i] = x;
        pos[3 * i + 1] = y;
        pos[3 * i + 2] = z;
    };
    // Curve::SetBoundaryConditions (Twisty/Curve.cpp:20-30), in float
    set(0, bc.start_pos.x, bc.start_pos.y, bc.start_pos.z);
    set(1, bc.start_pos.x + bc.start_dir.x * ds, bc.start_pos.y + bc.start_dir.y * ds, bc.start_pos.z + bc.start_dir.z * ds);
    set(n - 1, bc.end_pos.x - bc.end_dir.x * ds, bc.end_pos.y - bc.end_dir.y * ds, bc.end_pos.z - bc.end_dir.z * ds);
    set(n, bc.end_pos.x, bc.end_pos.y, bc.end_pos.z);
    const uint32_t M = n - 2;
    const double a0[3] = {pos[3], pos[4], pos[5]};
    const double a1[3] = {pos[3 * (n - 1)], pos[3 * (n - 1) + 1], pos[3 * (n - 1) + 2]};
    double C[3] = {a1[0] - a0[0], a1[1] - a0[1], a1[2] - a0[2]};
    const double D = std::sqrt(C[0] * C[0] + C[1] * C[1] + C[2] * C[2]);
    const double dsd = (double)ds;
    if (!(D <= (double)M * dsd * (1.0 + 1e-6))) {
        std::ostringstream o;
        o << "infeasible geometry: the " << M << " free segments of length " << ds
          << " cannot span the distance " << D << " between points 1 and N-1";
        err = o.str();
        return false;
    }
    // chord direction u and an in-plane perpendicular w
    double u[3];
    if (D > 1e-12) {
        for (int k = 0; k < 3; ++k) u[k] = C[k] / D;
    } else {
        u[0] = bc.start_dir.x; u[1] = bc.start_dir.y; u[2] = bc.start_dir.z;
        const double l = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int k = 0; k < 3; ++k) u[k] /= l;
    }
    const int ax = (std::fabs(u[0]) <= std::fabs(u[1]) && std::fabs(u[0]) <= std::fabs(u[2])) ? 0
                   : (std::fabs(u[1]) <= std::fabs(u[2])) ? 1 : 2;
    double e[3] = {0, 0, 0};
    e[ax] = 1.0;
    const double eu = e[0] * u[0] + e[1] * u[1] + e[2] * u[2];
    double w[3] = {e[0] - eu * u[0], e[1] - eu * u[1], e[2] - eu * u[2]};
    double wl = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    for (int k = 0; k < 3; ++k) w[k] /= wl;
    const double v[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
    // plane angle from the seed (SplitMix64)
    uint64_t z = (uint64_t)seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double phi = 2.0 * M_PI * (double)(z >> 11) * 0x1p-53;
    double w2[3];
    for (int k = 0; k < 3; ++k) w2[k] = std::cos(phi) * w[k] + std::sin(phi) * v[k];
    // turning angle beta: ds * sin(M beta/2) / sin(beta/2) = D, beta in [0, 2 pi / M]
    auto chord = [&](double beta) {
        if (beta < 1e-300) return (double)M * dsd;
        return dsd * std::sin(0.5 * M * beta) / std::sin(0.5 * beta);
    };
    double lo = 0.0, hi = 2.0 * M_PI / (double)M;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (chord(mid) > D) lo = mid;
        else hi = mid;
    }
    const double beta = 0.5 * (lo + hi);
    double p[3] = {a0[0], a0[1], a0[2]};
    for (uint32_t i = 0; i + 1 < M; ++i) {
        const double th = -0.5 * (double)(M - 1) * beta + (double)i * beta;
        for (int k = 0; k < 3; ++k) p[k] += dsd * (std::cos(th) * u[k] + std::sin(th) * w2[k]);
        set(2 + i, (float)p[0], (float)p[1], (float)p[2]);
    }
    return true;
}

namespace {

constexpr float kTwistyPiF = 3.141592653589793f;  // Twisty/MathConsts.h:8

float gaussian_phase(float p, float m)
{
    const float np = std::sqrt((kTwistyPiF * m) * 0.5f) / (1.0f - std::exp(-2.0f / m));
    const float val = (-m * p * p) * 0.5f;
    return np * std::exp(val);
}

double integrand_rt(double p, double kds, double bds, double eps, double mu)
{
    const double phase = (double)gaussian_phase((float)p, (float)mu);
    const double scattering = p * std::exp(bds * phase - 1.0 * (eps * eps * p * p * 0.5));
    double sin_term = p;
    if (kds > 0.0) sin_term = std::sin(kds * p) / kds;
    return scattering * sin_term;
}

float integrate(float curvature, float mu, float eps, float scatter, float min_bound, float max_bound, float bias,
                uint32_t n, float ds, std::vector<double> &w)
{
    const double kds = (double)(curvature * ds);
    const double bds = (double)(scatter * ds);
    const double h = (double)((max_bound - min_bound) / (float)n);
    const double weight = (double)(1.0f / 3.0f) * h;
    const double start = (double)min_bound;
    const double reg = (double)mu, pm = (double)eps;
    w.assign(n + 1, 0.0);
    w[0] = integrand_rt(start, kds, bds, reg, pm) * weight;
    w[n] = integrand_rt((double)max_bound, kds, bds, reg, pm) * weight;
    for (uint32_t i = 1; i < n / 2; ++i) w[2 * i - 1] = integrand_rt(start + ((double)(2 * i - 1) * h), kds, bds, reg, pm) * weight * 4.0;
    for (uint32_t i = 1; i < n / 2 - 1; ++i) w[2 * i] = integrand_rt(start + ((double)(2 * i) * h), kds, bds, reg, pm) * weight * 2.0;
    std::sort(w.begin(), w.end());
    double sum = 0.0;
    for (double v : w) sum += v;
    const double tp = (double)kTwistyPiF;
    return (float)((sum / (2.0 * tp * tp)) * (double)bias);
}

}  // namespace

bool lut_faithful_host(float mu, float eps, float scatter, float min_bound, float max_bound, float bias,
                       uint32_t num_steps_int, uint32_t bins, float ds, float *out, float minmax[2])
{
    if (bins < 2 || num_steps_int < 4 || (num_steps_int & 1u) || !(ds > 0.0f)) return false;
    const float min_k = 0.0f;
    const float max_k = (float)((2.0 / (double)ds) * (double)1.01f);
    const float step = (max_k - min_k) / (float)(bins - 1);
    unsigned nt = std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<unsigned>(nt, bins);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
        th.emplace_back([=]() {
            std::vector<double> w;
            for (uint32_t i = (uint32_t)((uint64_t)bins * t / nt); i < (uint32_t)((uint64_t)bins * (t + 1) / nt); ++i) {
                const float kappa = min_k + ((float)(int64_t)i * step);
                out[i] = integrate(kappa, mu, eps, scatter, min_bound, max_bound, bias, num_steps_int, ds, w);
            }
        });
    }
    for (auto &x : th) x.join();
    float mn = out[0], mx = out[0];
    for (uint32_t i = 1; i < bins; ++i) {
        if (out[i] < mn && out[i] >= 0.0f) mn = out[i];
        if (out[i] > mx && out[i] >= 0.0f) mx = out[i];
    }
    for (uint32_t i = 0; i < bins; ++i)
        if (out[i] <= 0.0f) out[i] = mn;
    minmax[0] = mn;
    minmax[1] = mx;
    return true;
}

float norm_z(const twisty_bc &bc, float ds)
{
    // Norm: zVec = (x_e - x_s) * (1/ds) - n_e - n_s (PathWeightUtils.cpp:729-732), FMath float ops
    const float inv = 1.0f / ds;
    float zx = (bc.end_pos.x - bc.start_pos.x) * inv, zy = (bc.end_pos.y - bc.start_pos.y) * inv,
          zz = (bc.end_pos.z - bc.start_pos.z) * inv;
    zx = zx - bc.end_dir.x; zy = zy - bc.end_dir.y; zz = zz - bc.end_dir.z;
    zx = zx - bc.start_dir.x; zy = zy - bc.start_dir.y; zz = zz - bc.start_dir.z;
    return std::sqrt(zx * zx + zy * zy + zz * zz);
}

double norm_k4_log10(float z, float ds)
{
    // K4 (PathWeightUtils.cpp:643-651)
    float result = (z < 2.0) ? 1.0f : 0.0f;
    result /= z;
    result = (float)((double)result * (2.0 * (double)3.141592653589793f));
    const float inv_ds = (float)(1.0 / (double)ds);
    result *= (inv_ds * inv_ds * inv_ds);
    return std::log10((double)result);
}

bool compensated_tables(const float *lut, uint32_t bins, float step, uint32_t n_segments, std::vector<float> &lin,
                        std::vector<float> &fix, double &c0, double &inv_scale, int &wide, double &secant_err,
                        uint32_t &steep)
{
    wide = 0;
    lin.assign(2 * (size_t)bins, 0.0f);
    fix.assign(2 * (size_t)bins, 0.0f);
    c0 = 0.0;
    inv_scale = 0.0;
    secant_err = 0.0;
    steep = 0;
    bool positive = true;
    std::vector<double> lg(bins);
    std::vector<unsigned char> is_steep(bins, 0);
    double lo = INFINITY, hi = -INFINITY;
    const double st = (double)step;
    for (uint32_t i = 0; i < bins; ++i) {
        const float a = lut[i], b = lut[i + 1 < bins ? i + 1 : i];
        lin[2 * i] = a;
        lin[2 * i + 1] = b - a;
        if (!(a > 0.0f) || !std::isfinite(a)) {
            positive = false;
            continue;
        }
        lg[i] = std::log10((double)a);
        lo = std::min(lo, lg[i]);
        hi = std::max(hi, lg[i]);
        if (i + 1 < bins) {
            const double r = (double)b / (double)a - 1.0;
            const double e = (st * r) * (st * r) / (8.0 * 2.302585092994046);
            if (e > kSecantBound) {
                is_steep[i] = 1;
                ++steep;
            } else {
                secant_err = std::max(secant_err, e);
            }
        }
    }
    if (!positive) {
        secant_err = INFINITY;
        return false;
    }
    // largest s (at most 30) with range * 2^s + 65 <= (2^31 - 1) / (n_segments + 1); else the
    // wide form, range * 2^s + 65 <= (2^32 - 1) / 32
    const double range = hi - lo;
    double cap = std::floor(2147483647.0 / (double)(n_segments + 1));
    int s = 30;
    while (s > 0 && range * std::ldexp(1.0, s) + 65.0 > cap) --s;
    if (s < 22) {
        wide = 1;
        cap = std::floor(4294967295.0 / 32.0);
        s = 30;
        while (s > 0 && range * std::ldexp(1.0, s) + 65.0 > cap) --s;
    }
    if (s < 22 || steep > bins / kSteepFraction) {
        wide = 0;
        return false;
    }
    inv_scale = std::ldexp(1.0, -s);
    c0 = lo - 64.0 * inv_scale;
    for (uint32_t i = 0; i < bins; ++i) {
        const double e = 64.0 + std::nearbyint((lg[i] - lo) * std::ldexp(1.0, s));
        const uint32_t u = (uint32_t)std::min(e, cap - 1.0);
        std::memcpy(&fix[2 * i], &u, 4);
        double delta = 0.0;
        if (i + 1 < bins) delta = std::log10(1.0 + st * ((double)lut[i + 1] / (double)lut[i] - 1.0));
        fix[2 * i + 1] = is_steep[i] ? std::numeric_limits<float>::quiet_NaN() : (float)delta;
    }
    return true;
}

}  // namespace twisty
