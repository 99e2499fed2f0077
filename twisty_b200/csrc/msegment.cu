// msegment.cu -- independent-sample M-segment Monte Carlo on the device.
//
// The reference's other estimator, MSegmentPathGenerationMC (Experiments/ExperimentBase.cpp:
// 1246-1386): every path is a fresh random curve from the recursive bootstrapper
// (ResolveEvenNumberOfSegments, Twisty/PathGeneration.cpp:47-414) between the fixed points
// 0, 1, N-1, N, weighed like the Markov-chain paths; the estimate is the mean weight.
//
// One thread builds one path, writing its points straight into the path batch in global
// memory (each point is written once and read back by at most three later placements, through
// L1). The recursion runs on a small explicit stack in the reference's order (centre point,
// then the left half, then the right half). The arithmetic follows the reference's mix of float
// vectors and double scalars; the random draws come from Philox-4x32-10, counter (draw index,
// path id lo, path id hi, experiment ^ 'MSEG'), key = seed, one 32-bit output per float draw and
// two per double draw -- the reference's std::mt19937_64 stream is not reproduced (its
// threads' interleaving makes it unreproducible anyway). A placement the reference would
// abort on (spheres that do not intersect, a NaN extent) marks the path invalid (NaN point).
#include "kernels.h"
#include "device_common.cuh"

namespace twisty {
namespace {

constexpr float kPiF = 3.141592653589793f;

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float fdot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 fcross(F3 a, F3 b)
{
    return F3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float fmag(F3 a) { return sqrtf(fdot(a, a)); }
__device__ __forceinline__ F3 funit(F3 a) { return a * (1.0f / sqrtf(fdot(a, a))); }

// Uniform draws from a per-path Philox stream.
struct Draws {
    uint64_t seed;
    uint32_t path_lo, path_hi, tag;
    uint32_t n = 0;
    __device__ uint32_t word()
    {
        uint32_t c0 = n++, c1 = path_lo, c2 = path_hi, c3 = tag;
        dev::philox4x32_10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
        return c0;
    }
    __device__ float uf(float a, float b) { return a + (float)(word() >> 8) * (1.0f / 16777216.0f) * (b - a); }
    __device__ double ud(double a, double b)
    {
        const uint64_t hi = word(), lo = word();
        const double u = (double)(((hi << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
        return a + u * (b - a);
    }
    __device__ int coin() { return (int)(word() & 1u); }
};

struct PathPts {
    float *p;  // [N+1][3]
    __device__ F3 get(uint32_t i) const { return F3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
    __device__ void set(uint32_t i, F3 v) const
    {
        p[3 * i] = v.x;
        p[3 * i + 1] = v.y;
        p[3 * i + 2] = v.z;
    }
};

// RotateQuatByQuat / RotateVectorByQuaternion (Twisty/CurvePerturbUtils.cpp:91-127).
__device__ void quat_product(const float A[4], const float B[4], float r[4])
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

__device__ F3 rotate_by_quaternion(const float q[4], F3 v)
{
    float p[4] = {0.0f, v.x, v.y, v.z};
    const float qi[4] = {q[0], -q[1], -q[2], -q[3]};
    quat_product(p, q, p);
    quat_product(qi, p, p);
    return F3{p[1], p[2], p[3]};
}

__device__ void frame(F3 a, F3 b, F3 &xa, F3 &ya, F3 &za)
{
    za = funit(b - a);
    F3 r{1.0f, 0.0f, 0.0f};
    if (fabsf(fdot(za, r)) > 0.999f) r = F3{0.0f, 1.0f, 0.0f};
    xa = funit(fcross(za, r));
    ya = funit(fcross(za, xa));
}

// ResolveTwoSegments: the point between l and l+2. Returns false when the reference would throw.
__device__ bool resolve_two(const PathPts &P, uint32_t l, uint32_t r, double ds, Draws &g)
{
    const F3 a = P.get(l), b = P.get(r);
    const float d = fmag(b - a);
    if (fabs((2.0f * ds) - (double)d) < 0.001f) {
        P.set(l + 1, (a + b) * 0.5f);
        return true;
    }
    if ((2.0f * ds) < (double)d) return false;
    const float theta = g.uf(0.0f, 2.0f * kPiF);
    if (d < 0.001f) {
        const float phi = (float)acos(1.0 - 2.0 * (double)g.uf(0.0f, 1.0f));
        P.set(l + 1, a + F3{sinf(phi) * cosf(theta), sinf(phi) * sinf(theta), cosf(phi)} * (float)ds);
        return true;
    }
    const F3 mid = (a + b) * 0.5f;
    const F3 axis = funit(b - a);
    F3 helper{1.0f, 0.0f, 0.0f};
    if ((double)fabsf(fdot(axis, helper)) >= 0.99) helper = F3{0.0f, 1.0f, 0.0f};
    const F3 normal = funit(fcross(axis, helper));
    const float half = d * 0.5f;
    float off = 0.0f;
    if (ds > (double)half) off = (float)sqrt((ds * ds) - (double)(half * half));
    const F3 pt = mid + normal * off;
    const float s = sinf(theta / 2.0f);
    const float q[4] = {cosf(theta / 2.0f), axis.x * s, axis.y * s, axis.z * s};
    P.set(l + 1, rotate_by_quaternion(q, pt - a) + a);
    return true;
}

// ResolveThreeSegments: the two points between l and l+3.
__device__ bool resolve_three(const PathPts &P, uint32_t l, uint32_t r, double ds, Draws &g)
{
    const F3 a = P.get(l), b = P.get(r);
    const float d = fmag(b - a);
    if (fabs((3.0f * ds) - (double)d) < 0.001f) {
        P.set(l + 1, a + (b - a) * (1.0f / 3.0f));
        return resolve_two(P, l + 1, r, ds, g);
    }
    if ((3.0f * ds) < (double)d) return false;
    const float theta = g.uf(0.0f, 2.0f * kPiF);
    if (d < 0.001f) {
        const float phi = (float)acos(1.0 - 2.0 * (double)g.uf(0.0f, 1.0f));
        P.set(l + 1, a + F3{sinf(phi) * cosf(theta), sinf(phi) * sinf(theta), cosf(phi)} * (float)ds);
        return resolve_two(P, l + 1, r, ds, g);
    }
    F3 xa, ya, za;
    frame(a, b, xa, ya, za);
    const double d2 = (double)(d * d);
    const double r1 = ds, r1s = r1 * r1;
    const double r2 = 2.0f * ds, r2s = r2 * r2;
    double extent;
    if (((double)d + r1) < r2) {
        extent = kPiF;
    } else {
        const double h = 0.5 + (r1s - r2s) / (2.0 * d2);
        double aa = 0.0;
        if (fabs(r1s - (h * h * d2)) >= 0.001) aa = sqrt(r1s - (h * h * d2));
        extent = (h * d < 0.0) ? (double)kPiF - asin(aa / r1) : asin(aa / r1);
        if (extent != extent) return false;
    }
    const float umax = (float)(0.5f - cos(extent) * 0.5f);
    const double phi = acos(1.0 - 2.0 * g.ud(0.0, (double)umax));
    const F3 dir = xa * (float)sin(phi) * cosf(theta) + ya * (float)sin(phi) * sinf(theta) + za * (float)cos(phi);
    P.set(l + 1, a + funit(dir) * (float)ds);
    return resolve_two(P, l + 1, r, ds, g);
}

// The centre point of m segments between l and r (ResolveEvenNumberOfSegments' placement);
// the halves are handled by the caller.
__device__ bool place_centre(const PathPts &P, int m, uint32_t l, uint32_t r, double ds, Draws &g)
{
    const int h = m / 2;
    const uint32_t c = l + (uint32_t)h;
    const F3 a = P.get(l), b = P.get(r);
    const double d = fmag(b - a);
    if (fabs((m * ds) - d) < 0.001f) {
        P.set(c, (b + a) * 0.5f);
        return true;
    }
    const double rad = ds * h;
    if ((rad + rad) < d) return false;
    F3 xa, ya, za;
    if (d < 0.001f) {
        const double phi = acos(1.0 - 2.0 * g.ud(0.0, 1.0));
        const double theta = g.ud(0.0, (double)(2.0f * kPiF));
        const double sr = rad * pow((double)g.uf(0.0f, 1.0f), 1.0 / 3.0);
        frame(a, b, xa, ya, za);
        F3 off = xa * (float)sin(phi) * (float)cos(theta) + ya * (float)sin(phi) * (float)sin(theta) + za * (float)cos(phi);
        P.set(c, a + off * (float)sr);
        return true;
    }
    const double d2 = d * d;
    const F3 mid = (b + a) * 0.5f;
    const double to_mid = fmag(mid - a);
    const double aa = sqrt(rad * rad - (0.25 * d2));
    const double extent = asin(aa / rad);
    const float umax = (float)(0.5f - cos(extent) * 0.5f);
    const double phi = acos(1.0 - 2.0 * g.ud(0.0, (double)umax));
    const double theta = g.ud(0.0, (double)(2.0f * kPiF));
    const bool flip = g.coin() != 0;
    const double hyp = to_mid / cos(phi);
    const double maxr = h * ds;
    const double minp = hyp / maxr;
    const double sr = maxr * pow(minp + (1.0f - minp) * (double)g.uf(0.0f, 1.0f), 1.0 / 3.0);
    frame(a, b, xa, ya, za);
    F3 off = xa * (float)sin(phi) * (float)cos(theta) + ya * (float)sin(phi) * (float)sin(theta);
    if (!flip) {
        off = off + za * (float)cos(phi);
        P.set(c, a + off * (float)sr);
    } else {
        off = off + za * (float)cos(phi) * -1.0f;
        P.set(c, b + off * (float)sr);
    }
    return true;
}

struct MSegSpec {
    uint32_t n_segments;
    float ds;
    float p0[3], p1[3], pm1[3], pm[3];
    uint64_t seed;
    uint32_t experiment;
    uint64_t path0;
    uint64_t n_paths;
};

__global__ void __launch_bounds__(128) msegment_paths_kernel(MSegSpec s, float *__restrict__ pos)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_paths) return;
    const uint32_t N = s.n_segments;
    const PathPts P{pos + i * 3 * (uint64_t)(N + 1)};
    P.set(0, F3{s.p0[0], s.p0[1], s.p0[2]});
    P.set(1, F3{s.p1[0], s.p1[1], s.p1[2]});
    P.set(N - 1, F3{s.pm1[0], s.pm1[1], s.pm1[2]});
    P.set(N, F3{s.pm[0], s.pm[1], s.pm[2]});
    const uint64_t path = s.path0 + i;
    Draws g{s.seed, (uint32_t)path, (uint32_t)(path >> 32), s.experiment ^ 0x4D534547u};
    const double ds = s.ds;
    // explicit stack of (m, l, r) spans, left half on top (the reference's order)
    struct Span {
        int m;
        uint32_t l, r;
    };
    Span stack[40];
    int top = 0;
    stack[top++] = Span{(int)N - 2, 1u, N - 1};
    bool ok = true;
    while (top > 0 && ok) {
        const Span sp = stack[--top];
        ok = place_centre(P, sp.m, sp.l, sp.r, ds, g);
        if (!ok) break;
        const int h = sp.m / 2;
        const uint32_t c = sp.l + (uint32_t)h;
        if (h == 2) {
            ok = resolve_two(P, sp.l, c, ds, g) && resolve_two(P, c, sp.r, ds, g);
        } else if (h == 3) {
            ok = resolve_three(P, sp.l, c, ds, g) && resolve_three(P, c, sp.r, ds, g);
        } else {
            // the host validated N - 2 as resolvable, so h is even and the stack stays
            // within 2 entries per level of a depth below 20
            if (top + 2 > 40) {
                ok = false;
                break;
            }
            stack[top++] = Span{h, c, sp.r};
            stack[top++] = Span{h, sp.l, c};
        }
    }
    if (!ok) {
        const float nan = __int_as_float(0x7fffffff);
        P.set(2, F3{nan, nan, nan});
    }
}

// Weighed paths as per-path "chains" for the FP64 reduction (independent samples: the
// spread over them gives the estimate's standard error).
__global__ void __launch_bounds__(256) pack_paths_kernel(const double *__restrict__ w, const uint8_t *__restrict__ valid,
                                                         uint64_t n, ChainOut *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ChainOut o;
    o.log10_sum = valid[i] ? w[i] : -INFINITY;
    o.valid = valid[i] ? 1u : 0u;
    o.failed = valid[i] ? 0u : 1u;
    o.clamped = 0;
    o.pad = 0;
    out[i] = o;
}

}  // namespace

cudaError_t launch_msegment_paths(uint32_t n_segments, float ds, const float p0[3], const float p1[3],
                                  const float pm1[3], const float pm[3], uint64_t seed, uint32_t experiment,
                                  uint64_t path0, uint64_t n_paths, float *pos, cudaStream_t st)
{
    if (n_paths == 0) return cudaSuccess;
    MSegSpec s{};
    s.n_segments = n_segments;
    s.ds = ds;
    for (int k = 0; k < 3; ++k) {
        s.p0[k] = p0[k];
        s.p1[k] = p1[k];
        s.pm1[k] = pm1[k];
        s.pm[k] = pm[k];
    }
    s.seed = seed;
    s.experiment = experiment;
    s.path0 = path0;
    s.n_paths = n_paths;
    const uint64_t blocks = (n_paths + 127) / 128;
    msegment_paths_kernel<<<(unsigned)blocks, 128, 0, st>>>(s, pos);
    return cudaGetLastError();
}

cudaError_t launch_pack_paths(const double *w, const uint8_t *valid, uint64_t n, ChainOut *out, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    pack_paths_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w, valid, n, out);
    return cudaGetLastError();
}

}  // namespace twisty
