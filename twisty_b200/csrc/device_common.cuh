// device_common.cuh -- device helpers shared by every chain kernel.
//
//  * Philox-4x32-10 (Salmon et al., SC'11) and the mapping of one Philox output to a
//    chain step's proposal (sub-chain length k, left index, rotation angle). The mapping
//    ranges are the reference CPU runner's (Twisty/FullExperimentRunnerOptimalPerturb.cpp:
//    483-490,501-502) with k_max and the angle range as parameters.
//  * sin/cos of the half angle as fixed Taylor polynomials, so that every kernel form
//    draws bit-identical rotations from the same counter.
//  * The reference's FP32 operations written with explicit round-to-nearest intrinsics
//    (__fmul_rn, __fadd_rn, ...) so that no compiler contraction changes them: the drop-in
//    form reproduces the reference bit for bit from these.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace twisty {
namespace dev {

constexpr float kPiF = 3.141592653589793f;  // Twisty/MathConsts.h:8

__device__ __forceinline__ void philox4x32_10(uint32_t &c0, uint32_t &c1, uint32_t &c2, uint32_t &c3,
                                              uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
    }
}

struct Proposal {
    uint32_t k;     // rotated sub-chain spans points left..left+k
    uint32_t left;  // pivot point index
    float angle;    // rotation angle
};

// Counter (step, chain, experiment, 'TWST'), key (seed lo, seed hi).
__device__ __forceinline__ Proposal draw_step(uint64_t seed, uint32_t experiment, uint32_t chain,
                                              uint32_t step, uint32_t n_segments, uint32_t k_eff,
                                              float max_angle)
{
    uint32_t c0 = step, c1 = chain, c2 = experiment, c3 = 0x54575354u;
    philox4x32_10(c0, c1, c2, c3, (uint32_t)seed, (uint32_t)(seed >> 32));
    Proposal p;
    p.k = 2u + __umulhi(c0, k_eff - 1u);
    p.left = 1u + __umulhi(c1, n_segments - p.k - 1u);
    const float u = __fadd_rn(__fmul_rn((float)(((int32_t)c2) >> 8), 0x1p-23f), 0x1p-24f);
    p.angle = __fmul_rn(u, max_angle);
    return p;
}

// sin(angle/2), cos(angle/2) for |angle| <= pi (degree-13/14 Taylor, Horner with FMA).
__device__ __forceinline__ void sincos_half(float angle, float &s, float &c)
{
    const float a = __fmul_rn(angle, 0.5f);
    const float z = __fmul_rn(a, a);
    float ps = 1.0f / 6227020800.0f;
    ps = __fmaf_rn(ps, z, -1.0f / 39916800.0f);
    ps = __fmaf_rn(ps, z, 1.0f / 362880.0f);
    ps = __fmaf_rn(ps, z, -1.0f / 5040.0f);
    ps = __fmaf_rn(ps, z, 1.0f / 120.0f);
    ps = __fmaf_rn(ps, z, -1.0f / 6.0f);
    s = __fmaf_rn(__fmul_rn(a, z), ps, a);
    float pc = -1.0f / 87178291200.0f;
    pc = __fmaf_rn(pc, z, 1.0f / 479001600.0f);
    pc = __fmaf_rn(pc, z, -1.0f / 3628800.0f);
    pc = __fmaf_rn(pc, z, 1.0f / 40320.0f);
    pc = __fmaf_rn(pc, z, -1.0f / 720.0f);
    pc = __fmaf_rn(pc, z, 1.0f / 24.0f);
    pc = __fmaf_rn(pc, z, -0.5f);
    c = __fmaf_rn(z, pc, 1.0f);
}

// ---------------------------------------------------------------------------------
// Reference FP32 semantics (IEEE, left to right, no contraction)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ float rdot3(float x, float y, float z)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}

// Farlor::Vector3::Normalized as x * (1/sqrt(x.x)) (pinned FMath boundary, identical to the
// reference's _CudaSafe tangent code, Twisty/CurvePerturbUtils.cpp:209-214).
__device__ __forceinline__ float rinvnorm(float x, float y, float z)
{
    return __fdiv_rn(1.0f, __fsqrt_rn(rdot3(x, y, z)));
}

// RotateQuatByQuat (Twisty/CurvePerturbUtils.cpp:91-111).
__device__ __forceinline__ void rquat_mul(const float a[4], const float b[4], float r[4])
{
    const float t0 = __fsub_rn(__fsub_rn(__fsub_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2])), __fmul_rn(a[3], b[3]));
    const float t1 = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(a[0], b[1]), __fmul_rn(a[1], b[0])), __fmul_rn(a[2], b[3])), __fmul_rn(a[3], b[2]));
    const float t2 = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(a[0], b[2]), __fmul_rn(a[1], b[3])), __fmul_rn(a[2], b[0])), __fmul_rn(a[3], b[1]));
    const float t3 = __fadd_rn(__fadd_rn(__fsub_rn(__fmul_rn(a[0], b[3]), __fmul_rn(a[1], b[2])), __fmul_rn(a[2], b[1])), __fmul_rn(a[3], b[0]));
    r[0] = t0;
    r[1] = t1;
    r[2] = t2;
    r[3] = t3;
}

// RotateVectorByQuaternion (Twisty/CurvePerturbUtils.cpp:113-127): q^-1 (x) (p (x) q).
__device__ __forceinline__ void rrotate(const float q[4], float &x, float &y, float &z)
{
    float pq[4] = {0.0f, x, y, z};
    const float inv[4] = {q[0], -q[1], -q[2], -q[3]};
    float t[4];
    rquat_mul(pq, q, t);
    rquat_mul(inv, t, pq);
    x = pq[1];
    y = pq[2];
    z = pq[3];
}

struct LutMeta {
    float min_k, max_k, step;
    int32_t bins;
};

// One segment of WeightCurveViaCurvatureLog10_CudaSafe (Twisty/PathWeighters.cpp:41-96),
// returning the left bin index (or -1 for a NaN curvature) and the double blend value.
// clamped counts curvatures outside [min_k, max_k] beyond the 1e-3 snap.
__device__ __forceinline__ int32_t rbin_blend(float c, const float *__restrict__ lut, const LutMeta &m,
                                              double &blend, uint32_t &clamped)
{
    if (isnan(c)) return -1;
    if ((c < m.min_k) && (double)fabsf(__fsub_rn(c, m.min_k)) < 1e-3) c = m.min_k;
    if ((c > m.max_k) && (double)fabsf(__fsub_rn(m.max_k, c)) < 1e-3) c = m.max_k;
    if (c < m.min_k) { c = m.min_k; ++clamped; }
    if (c > m.max_k) { c = m.max_k; ++clamped; }
    const float dist = __fsub_rn(c, m.min_k);
    const float real_idx = __fdiv_rn(dist, m.step);
    int32_t left = (int32_t)floorf(real_idx);
    // The clamps above keep left in [0, bins-1] for a consistent (min, max, step) triple;
    // the guard keeps a caller-supplied inconsistent triple inside the table.
    left = min(max(left, 0), m.bins - 1);
    const int32_t right = (left == m.bins - 1) ? left : left + 1;
    const float lv = lut[left], rv = lut[right];
    const float interp = __fsub_rn(dist, __fmul_rn((float)left, m.step));
    blend = (double)__fadd_rn(__fmul_rn(lv, __fsub_rn(1.0f, interp)), __fmul_rn(rv, interp));
    return left;
}

// ---------------------------------------------------------------------------------
// Base-10 scaled running sum: CombinedWeightValues_C (Twisty/CombinedWeightUtils.h:28-174)
// ---------------------------------------------------------------------------------
struct CombinedWeight {
    double max_log10;
    double total;
    double offset;
    uint32_t n;
    uint32_t pad;
};

__device__ __forceinline__ void cw_reset(CombinedWeight &c)
{
    c.max_log10 = 0.0;
    c.total = 0.0;
    c.offset = 0.0;
    c.n = 0;
    c.pad = 0;
}

__device__ __forceinline__ void cw_add(CombinedWeight &c, double v)
{
    if (c.n == 0) {
        c.max_log10 = v;
        c.offset = 300.0 - (v + 6.0);
        c.total += pow(10.0, v + c.offset);
        c.n++;
        return;
    }
    if (c.max_log10 >= v) {
        c.total += pow(10.0, v + c.offset);
        c.n++;
        return;
    }
    const double new_offset = 300.0 - (v + 6.0);
    const double delta = new_offset - c.offset;
    c.total = pow(10.0, log10(c.total) + delta);
    c.max_log10 = v;
    c.offset = new_offset;
    c.total += pow(10.0, v + c.offset);
    c.n++;
}

__device__ __forceinline__ CombinedWeight cw_combine(CombinedWeight a, CombinedWeight b)
{
    if (a.n > 0 && b.n == 0) return a;
    if (b.n > 0 && a.n == 0) return b;
    if (b.max_log10 > a.max_log10) {
        const CombinedWeight t = b;
        b = a;
        a = t;
    }
    CombinedWeight r;
    cw_reset(r);
    r.max_log10 = a.max_log10;
    r.n = a.n + b.n;
    r.offset = a.offset;
    if (a.max_log10 == b.max_log10) {
        r.total = a.total + b.total;
        return r;
    }
    const double delta = a.offset - b.offset;
    r.total = a.total + pow(10.0, log10(b.total) + delta);
    return r;
}

// log10 of ExtractFinalValue (Twisty/CombinedWeightUtils.h:160-174).
__device__ __forceinline__ double cw_log10(const CombinedWeight &c)
{
    return c.n ? log10(c.total) - c.offset : -INFINITY;
}

}  // namespace dev
}  // namespace twisty
