// comp_body.cuh -- the compensated B200 form of the Markov-chain hot path: the chain body
// shared by the single-run kernels (chain_comp.cu) and the batched kernels (batch.cu).
//
// Algorithm: the reference's GeometryRandom loop (Twisty/FullExperimentRunnerOptimalPerturb.cpp:
// 469-595): per step, rotate the points strictly between a random pivot `left` and
// `right = left + k` about the axis x_right - x_left by a random angle, recompute every
// tangent and curvature, gather each curvature's weight from the table, sum the log10
// weights, and accumulate the path weight into the experiment's running sum.
//
// B200 layout and arithmetic:
//  * G lanes cooperate on one chain (G = 1, 4, 8, 16 or 32); lane j owns the SPL contiguous
//    segments j*SPL .. j*SPL+SPL-1. The chain lives in shared memory as its unit tangents
//    t_i and segment lengths l_i. Rotating the points between left and right about the
//    chord x_right - x_left turns every tangent t_left .. t_{right-1} by the same rotation
//    (the chord is the axis and stays fixed) and leaves the lengths alone; each rotated
//    tangent is renormalised by one Newton step, so |t_i| = 1 to an ulp and the full
//    recompute needs no normalisation: kappa_i = |t_{i+1} - t_i| N/S.
//  * Three planes per warp: (t.x, t.y) as float2, t.z, and l. Segment s = j*SPL + m of the
//    chain in lanes q*G..q*G+G-1 sits in row m, column q*G + j of each plane; a lane's own
//    segments are a base register plus immediate offsets, so a tangent is one 8-byte and
//    one 4-byte LDS (12 bytes, the shared-memory bandwidth the full recompute needs; the
//    full recompute reads consecutive columns of one row: conflict-free). Row pitches
//    (32 + 16/SPL float2, 32 + G/SPL floats) shift successive rows by distinct banks so
//    the k consecutive segments of a rotation fall in distinct banks (at most 2-way
//    conflicts); one-lane shapes keep rows of 32 (comp_pitch_xy). The next lane's first
//    tangent comes by shuffle.
//  * Rotation: the chord is summed across the group (for full-warp groups as 32-bit fixed
//    point with the warp reduction instruction, scaled by the chain's longest segment so
//    that 64 segments cannot overflow; otherwise by float shuffles), normalised, and each
//    tangent in the sub-chain is turned by Rodrigues' formula (groups of 1 and 4 lanes: by
//    v + (R - I) v, the matrix built once per step) with the angle's sin and 1 - cos taken
//    from the proposal's half-angle sine and cosine. Forward passes of short chains turn the
//    complement of a sub-chain longer than half the path instead (chain_body).
//  * The table is staged once per CTA in shared memory as float2. In the fixed-point form
//    entry i holds round((log10 L_i - c0) 2^s) as uint32 bits and the change of log10 of
//    the blend across the bin (secant): a segment costs one 8-byte LDS, one integer add
//    (exact) and one FMA (the interpolation correction). Each lane rounds its correction
//    sum to the same fixed point, the group adds the lanes' totals with integer shuffles
//    (exact), and the chain's running log-sum-exp keeps its reference exponent as an
//    integer path total, so a path's weight relative to the running maximum is exp2 of an
//    exact integer difference. The host scales the table so that N+1 entries stay below
//    2^31; when that leaves fewer than 22 fraction bits, or the secant would lose more
//    than ~1e-7 per segment, the host selects the exact form instead: (L_i, L_{i+1} - L_i),
//    a log2 per segment, a Kahan-compensated FP32 sum combined across lanes by TwoSum and
//    a log-sum-exp over (hi, lo) float pairs.
//  * Incremental variant (ChainSpec.incr_resync = R > 0, fixed-point tables only): a rotation
//    turns the tangents of its sub-chain together, so of the path's curvatures only the two
//    at its ends change (interior ones are invariant up to rounding). Each weighted step
//    evaluates those two terms before and after the rotation and adds the difference to the
//    path's integer total; every R-th weighted step recomputes the total in full. This is an
//    algorithmic change of the recompute-everything definition and is reported separately.
//  * FP64 appears only per chain (assembling its log10 sum), in the per-CTA log-sum-exp of
//    the chains and in the global reduction (and per path in the exact form).
//  * Proposals: lane j of a group draws the Philox proposal of step base+j (one draw per
//    lane per G steps) and shuffles broadcast it.
#pragma once
#include "kernels.h"
#include "device_common.cuh"

#include <algorithm>
#include <cfloat>

namespace twisty {

// Shared by the translation units that instantiate the chain kernels (plain structs).
struct CompConsts {
    float kscale;        // (N/S) / step : |t_{i+1}-t_i| -> fractional bin index; the chain kernels keep
                         // their tangents scaled to length kscale, so |t'_{i+1}-t'_i| is the index
    float roff;          // -min_k / step
    float rmax;          // (max_k - min_k) / step
    float rsnap;         // 1e-3 / step: overshoot that counts as clamped
    float step;
    int32_t bins;
    float fscale;        // 2^s of the fixed-point table
    float l2s;           // 2^-s log2(10): fixed-point units -> log2
    int32_t wide;        // 64-bit path totals (the table's LogFixed.wide)
    double lw_offset;    // (N-1) c0 of the fixed-point table
    double inv_scale;    // 2^-s of the fixed-point table
};

struct ModeArgs {
    double log10_abs;    // log10 of the per-segment absorption factor
    // linear table (L_i, L_{i+1} - L_i) of the fixed-point table's curve: paths that cross a
    // steep bin (NaN slope) are re-weighed through it
    const float2 *lin;
    // export
    float *exp_pos;      // [chains][steps][N+1][3]
    double *exp_w;       // [chains][steps] log10 weights (absorption included, normaliser not)
    float x0[3];
    // adjoint: per bin (dL/dmu_s, its change to the next bin, dL/deps, its change to the next
    // bin) -- the derivative tables in the linear table's form, one 16-byte load per segment
    const float4 *dtab;
    float ref_log10;     // log10 of the forward sum of path weights (normaliser and absorption excluded)
    double *grad;        // [chains][6]: d/dmu_s, d/deps, d/dx, d/dy, d/dz (log10 units), sum of weights
};

namespace {

constexpr uint32_t FULL = 0xffffffffu;
constexpr int kMaxSubChain = 64;  // largest k the rotation rounds cover
constexpr float kLog2_10 = 3.32192809488736234787f;
constexpr float kLog10_2 = 0.30102999566398119521f;
constexpr float kInvLn10 = 0.43429448190325182765f;


__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float ex2_approx(float x)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <int G>
__device__ __forceinline__ void group_sum3(float &x, float &y, float &z)
{
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        x += __shfl_xor_sync(FULL, x, o);
        y += __shfl_xor_sync(FULL, y, o);
        z += __shfl_xor_sync(FULL, z, o);
    }
}

template <int G, class T>
__device__ __forceinline__ T group_sum(T v)
{
#pragma unroll
    for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// TwoSum-combine the lanes' Kahan pairs (hi, lo) of one group.
template <int G>
__device__ __forceinline__ void group_sum_pair(float &hi, float &lo)
{
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const float oh = __shfl_xor_sync(FULL, hi, o);
        const float ol = __shfl_xor_sync(FULL, lo, o);
        const float s = hi + oh;
        const float bp = s - hi;
        const float e = (hi - (s - bp)) + (oh - bp);
        hi = s;
        lo = lo + ol + e;
    }
}

__device__ __forceinline__ void kahan_add(float &s, float &c, float x)
{
    const float y = x - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

// Fractional bin index of |t_{i+1}-t_i|^2 and its bin. CLAMP handles tables whose curvature
// range a path can leave; tables spanning [0, 2.02 N/S] (the reference's) cannot be left by
// unit tangents (|t_{i+1}-t_i| <= 2). r >= 0 or NaN after the clamp. Returns the fraction
// r - L within bin L. floor(r) comes without conversion instructions (which share the MUFU
// pipe with the square root): r + 2^23 rounded toward -infinity carries floor(r) in its low
// mantissa bits for 0 <= r < 2^23. NaN and infinity, which only a degenerate zero-length
// chord can produce, land past the last bin, are bounded to it and get a NaN fraction.
template <bool B>
struct BoolTag {
    static constexpr bool value = B;
};

template <bool CLAMP>
__device__ __forceinline__ float bin_of(float qq, const CompConsts &k, bool valid, uint32_t &clamped, int32_t &L)
{
    // qq is |t'_{i+1} - t'_i|^2 of tangents scaled to length kscale: its root is the
    // fractional bin of a table starting at curvature 0 (tables that need no clamping do)
    float r = CLAMP ? sqrt_approx(qq) + k.roff : sqrt_approx(qq);
    if (CLAMP) {
        if (r < 0.0f) r = 0.0f;
        if (r > k.rmax) {
            clamped += (valid && r - k.rmax >= k.rsnap) ? 1u : 0u;
            r = k.rmax;
        }
    }
    const float fl = __fadd_rd(r, 8388608.0f);
    L = (int32_t)min(__float_as_uint(fl) - 0x4B000000u, (uint32_t)k.bins - 1u);
    return r - (fl - 8388608.0f);
}

// Walk the curvatures this lane owns: seg(i, qq, valid) for curvature i = base+m-1 (between
// segments base+m-1 and base+m), the last one with the next lane's first tangent.
// tan(m, x, y, z) gives the unit tangent of segment j*SPL+m (zero past the last segment);
// next(t0, n) the next lane's first tangent given this lane's (t0). Every slot is evaluated,
// with valid = false past curvature N-2, so no table load hides behind a branch (padding
// tangents are zero: their |t_{i+1}-t_i|^2 is 0 or 1, a bin in the table). FULLN: N == G*SPL,
// only the group's last boundary is invalid.
template <int G, int SPL, bool FULLN, class TanFn, class NextFn, class SegFn>
__device__ __forceinline__ void for_curvatures(uint32_t j, uint32_t N, TanFn tan, NextFn next, SegFn seg)
{
    float t0x = 0.f, t0y = 0.f, t0z = 0.f, px = 0.f, py = 0.f, pz = 0.f;
    const uint32_t base = j * SPL;
#pragma unroll
    for (int m = 0; m < SPL; ++m) {
        float tx, ty, tz;
        tan(m, tx, ty, tz);
        if (m == 0) {
            t0x = tx; t0y = ty; t0z = tz;
        } else {
            const float dx = tx - px, dy = ty - py, dz = tz - pz;
            seg(base + m - 1, fmaf(dx, dx, fmaf(dy, dy, dz * dz)), FULLN || base + m <= N - 1);
        }
        px = tx; py = ty; pz = tz;
    }
    float nx, ny, nz;
    next(t0x, t0y, t0z, nx, ny, nz);
    const float dx = nx - px, dy = ny - py, dz = nz - pz;
    seg(base + SPL - 1, fmaf(dx, dx, fmaf(dy, dy, dz * dz)), base + SPL <= N - 1);
}

// next() for tangents held in registers: the next lane's t0 by shuffle.
template <int G>
struct ShflNext {
    __device__ __forceinline__ void operator()(float t0x, float t0y, float t0z, float &nx, float &ny, float &nz) const
    {
        if constexpr (G == 1) {   // a one-lane chain has no next lane: its last slot is padding
            nx = t0x; ny = t0y; nz = t0z;
        } else {
            nx = __shfl_down_sync(FULL, t0x, 1, G);
            ny = __shfl_down_sync(FULL, t0y, 1, G);
            nz = __shfl_down_sync(FULL, t0z, 1, G);
        }
    }
};

// Table entry L. GLOBAL: the table is in global memory, read through L1 by an unconditional
// non-coherent load, so that the compiler cannot turn the padded slots' loads into predicated
// ones (measured: with plain loads the padded curvature loop ran 15 % slower through L1).
template <bool GLOBAL>
__device__ __forceinline__ float2 tab_load(const float2 *__restrict__ tab, int32_t L)
{
    if constexpr (GLOBAL) {
        float2 e;
        asm("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(e.x), "=f"(e.y) : "l"(tab + L));
        return e;
    } else {
        return tab[L];
    }
}

// Generic full recompute of one path's log10 weight (absorption excluded), for the exact
// table or, with 64-bit lane sums, for the fixed-point table at any lane width. bin_sink(i,
// bin) receives every curvature's bin (-1 for NaN).
template <int G, int SPL, bool EXACT, bool CLAMP, bool GLOBAL = false, class TanFn, class NextFn, class BinFn>
__device__ __forceinline__ double path_log10(uint32_t j, uint32_t N, const float2 *__restrict__ tab,
                                             const CompConsts &k, TanFn tan, NextFn next, BinFn bin_sink,
                                             uint32_t &clamped)
{
    unsigned long long isum = 0;
    float csum = 0.f, ks = 0.f, kc = 0.f;
    auto seg = [&](uint32_t i, float qq, bool valid) {
        int32_t L;
        const float frac = bin_of<CLAMP>(qq, k, valid, clamped, L);
        if (valid) bin_sink(i, isnan(frac) ? -1 : L);
        const float2 e = tab_load<GLOBAL>(tab, L);
        if (EXACT) {
            const float term = __log2f(fmaf(frac * k.step, e.y, e.x)) * kLog10_2;
            kahan_add(ks, kc, valid ? term : 0.0f);
        } else {
            isum += valid ? __float_as_uint(e.x) : 0u;
            const float c2 = fmaf(frac, e.y, csum);
            csum = valid ? c2 : csum;
        }
    };
    // a chain that fills its group's slots: slot validity known at compile time
    if (N == (uint32_t)(G * SPL))
        for_curvatures<G, SPL, true>(j, N, tan, next, seg);
    else
        for_curvatures<G, SPL, false>(j, N, tan, next, seg);
    if (EXACT) {
        float hi = ks, lo = -kc;
        group_sum_pair<G>(hi, lo);
        return (double)hi + (double)lo;
    }
    const unsigned long long is = group_sum<G>(isum);
    const float cs = group_sum<G>(csum);
    return k.lw_offset + (double)is * k.inv_scale + (double)cs;
}

// Fixed-point full recompute for chains: the group's total of table entries plus rounded
// interpolation corrections, in units of 2^-s. Each lane's sum is exact in 32 bits (its true
// value lies in [0, 2^32) by the table's scale); the group total is added in 32 bits for a
// narrow table, in 64 bits for a wide one (both exact). *bad is set when any curvature of
// the path is NaN.
template <int G, int SPL, bool CLAMP, bool GLOBAL, class TanFn, class NextFn>
__device__ __forceinline__ unsigned long long path_fixed(uint32_t j, uint32_t gbase, uint32_t N, const float2 *__restrict__ tab,
                                               const CompConsts &k, TanFn tan, NextFn next, bool &bad,
                                               uint32_t &clamped)
{
    uint32_t isum = 0;
    float csum = 0.f;
    auto seg = [&](uint32_t, float qq, bool valid) {
        int32_t L;
        const float frac = bin_of<CLAMP>(qq, k, valid, clamped, L);
        const float2 e = tab_load<GLOBAL>(tab, L);
        isum += valid ? __float_as_uint(e.x) : 0u;
        // a padding slot leaves the sum alone even where the slope is NaN (a steep bin)
        const float c2 = fmaf(frac, e.y, csum);
        csum = valid ? c2 : csum;
    };
    if (N == (uint32_t)(G * SPL))
        for_curvatures<G, SPL, true>(j, N, tan, next, seg);
    else
        for_curvatures<G, SPL, false>(j, N, tan, next, seg);
    const uint32_t nan_lanes = __ballot_sync(FULL, isnan(csum));
    constexpr uint32_t gmask = (G == 32) ? FULL : ((1u << G) - 1u);
    bad = ((nan_lanes >> gbase) & gmask) != 0u;
    isum += (uint32_t)__float2int_rn(csum * k.fscale);
    if (k.wide) return group_sum<G>((unsigned long long)isum);
    return (unsigned long long)group_sum<G>(isum);
}

// Row pitches of a warp's planes (float2 and float elements). With several lanes per chain
// the rows are padded so that the consecutive segments of one rotation, spread over lanes and
// rows, fall in distinct banks. With one lane per chain every lane is its own chain: a rotation
// has the lanes at unrelated rows, and an unpadded row of 32 puts lane i in bank (pair) i mod
// 16 (32) whatever its row, so no access conflicts (the padded pitch measured the one-lane
// kernel bound by shared-memory wavefronts at 92 % of their peak).
__host__ __device__ constexpr int comp_pitch_xy(int G, int SPL)
{
    return G == 1 ? 32 : 32 + ((16 / SPL) > 1 ? (16 / SPL) : 1);
}
__host__ __device__ constexpr int comp_pitch_z(int G, int SPL)
{
    return G == 1 ? 32 : 32 + ((G / SPL) > 1 ? (G / SPL) : 1);
}

template <int G, int SPL>
struct Layout {
    static constexpr int PXY = comp_pitch_xy(G, SPL);  // float2 plane pitch
    static constexpr int PZ = comp_pitch_z(G, SPL);    // float plane pitch
    static constexpr int XY_BYTES = SPL * PXY * 8;
    static constexpr int Z_BYTES = SPL * PZ * 4;
    // xy, z planes; rounded to 16 bytes so that every warp's float2 plane (and what follows the
    // last warp) stays aligned when SPL * PZ is odd
    static constexpr int WARP_BYTES = (XY_BYTES + Z_BYTES + 15) / 16 * 16;
    __device__ __forceinline__ static uint32_t xy(uint32_t col, uint32_t m) { return m * (uint32_t)PXY + col; }
    __device__ __forceinline__ static uint32_t z(uint32_t col, uint32_t m) { return m * (uint32_t)PZ + col; }
};

constexpr size_t warp_state_bytes(int G, int SPL)
{
    return ((size_t)SPL * comp_pitch_xy(G, SPL) * 8 + (size_t)SPL * comp_pitch_z(G, SPL) * 4 + 15) / 16 * 16;
}

// Threads per CTA the chain kernel of a shape is compiled for (its register budget: 65536 /
// threads). With 12 or more segments per lane every shape fits 768 threads (24 warps) in 80
// registers without spills (forward variants), and the extra warps pay: N = 256 +6 %, 512
// +13 %, 1024 +24 % over the 16 (8) warps of a 512-thread budget.
__host__ __device__ constexpr int comp_max_threads(int G, int SPL)
{
    return (SPL >= 12) ? 768 : 1024;
}

// The segment lengths, one array per CTA: rotations never change a length, and every chain of
// a CTA starts from the same initial curve, so all its chains share them (G * SPL floats,
// padding segments 1).
__host__ __device__ constexpr size_t cta_len_bytes(int G, int SPL) { return ((size_t)G * SPL * 4 + 15) / 16 * 16; }

// The planes of one warp's chains (tangents) and the CTA's segment lengths.
struct Planes {
    float2 *xy;
    float *z;
    float *l;    // CTA-wide, by segment index
};

enum { kModeForward = 0, kModeExport = 1, kModeAdjoint = 2 };


// Receiver-position gradient of one path's log10 weight, computed by one lane from the last
// three segments: moving the receiver moves points N-1 and N together, so only the segment
// vector v_{N-2} changes, hence t_{N-2} and the curvatures kappa_{N-3}, kappa_{N-2}. The
// reference's interpolation weight is in curvature units (PathWeighters.cpp:79-82), so its
// segment weight is almost constant within a bin and jumps by nearly L_{b+1} - L_b at each
// edge: its pathwise derivative misses almost all of the change an expectation over paths
// sees. The slope taken is that of the expected weight: averaged over a bin the staircase is
// the table's linear interpolant taken half a bin to the left, whose slope at fractional bin r
// is (L_{J+1} - L_J) / step with J = floor(r - 1/2); divided by the weight itself.
__device__ __forceinline__ void receiver_grad(const float t3[3], const float t2[3], const float t1[3], float len2,
                                              const float2 *lin, const CompConsts &k, float inv_ds, float g[3])
{
    const float r2 = 1.0f / len2;  // d t2 / d v2 = (I - t2 t2^T) / |v2|
    g[0] = g[1] = g[2] = 0.f;
    for (int which = 0; which < 2; ++which) {
        float d[3];
        float sign;
        if (which == 0) { for (int q = 0; q < 3; ++q) d[q] = t2[q] - t3[q]; sign = 1.f; }   // kappa_{N-3}
        else { for (int q = 0; q < 3; ++q) d[q] = t1[q] - t2[q]; sign = -1.f; }             // kappa_{N-2}
        const float dn = sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (!(dn > 0.f)) continue;
        float r = fmaf(dn, k.kscale, k.roff);
        if (r < 0.f) r = 0.f;
        if (r > k.rmax) continue;  // clamped: flat
        // the linear table (L_i, L_{i+1} - L_i): the blend at r and the slope of bin J
        const int32_t L = min((int32_t)r, k.bins - 1);
        const float2 e = lin[L];
        const float dd = (r - (float)L) * k.step;
        const float blend = fmaf(dd, e.y, e.x);
        const int32_t J = min(max((int32_t)floorf(r - 0.5f), 0), k.bins - 2);
        const float sl = lin[J].y;
        const float dlog = sl / (k.step * blend) * kInvLn10;  // d log10 w / d kappa
        const float dk = dlog * inv_ds * sign / dn;                  // d kappa / d t = inv_ds d/|d|
        const float dt = d[0] * t2[0] + d[1] * t2[1] + d[2] * t2[2];
        for (int q = 0; q < 3; ++q) g[q] += dk * (d[q] - dt * t2[q]) * r2;
    }
}

// The CTA's segment lengths from the initial segment vectors (padding segments 1), computed as
// the chain body computes them (|v| = |v|^2 rsqrt(|v|^2)); the CTA synchronises before use.
__device__ __forceinline__ void fill_lengths(float *s_len, const float *__restrict__ init_seg, uint32_t n, uint32_t slots)
{
    for (uint32_t s = threadIdx.x; s < slots; s += blockDim.x) {
        float len = 1.f;
        if (s < n) {
            const float x = init_seg[3 * s], y = init_seg[3 * s + 1], z = init_seg[3 * s + 2];
            const float ss = fmaf(x, x, fmaf(y, y, z * z));
            len = ss * rsqrtf(ss);
        }
        s_len[s] = len;
    }
}

// Stage a table of `bins` float2 entries into shared memory (float4 vector loads).
__device__ __forceinline__ void stage_table(float4 *smem4, const float2 *__restrict__ tab_g, int bins)
{
    for (int i = threadIdx.x; i < bins / 2; i += blockDim.x) smem4[i] = reinterpret_cast<const float4 *>(tab_g)[i];
    if ((bins & 1) && threadIdx.x == 0) reinterpret_cast<float2 *>(smem4)[bins - 1] = tab_g[bins - 1];
}

// Exact-blend weight of the group's current path through the linear table, for paths of a
// fixed-point table that cross a steep bin. Not inlined: it runs rarely, and inlined its
// registers would count against the hot loop's.
template <int G, int SPL, bool CLAMP>
__device__ __noinline__ double steep_fallback(Planes st, uint32_t gbase, uint32_t j, uint32_t N,
                                              const float2 *__restrict__ lin, CompConsts kc)
{
    using Lay = Layout<G, SPL>;
    const uint32_t own = gbase + j;
    auto tan = [&](int m, float &x, float &y, float &z) {
        const float2 a = st.xy[Lay::xy(own, m)];
        x = a.x;
        y = a.y;
        z = st.z[Lay::z(own, m)];
    };
    uint32_t unused = 0;
    return path_log10<G, SPL, true, CLAMP, true>(j, N, lin, kc, tan, ShflNext<G>{}, [](uint32_t, int32_t) {}, unused);
}

// One Markov chain run by the G lanes of one group on its own records st (tangent, length;
// warp-local slots): initial state from init_seg (segment vectors), burn_in + steps
// proposals, a full recompute of every weighted path, and the chain's running log-sum-exp.
// Writes out[chain] (when out is set and the chain is real) and returns the chain's log10 sum.
// STEEP: the fixed-point table has steep bins (NaN slopes); paths crossing one are re-weighed
// through ma.lin. Without it a NaN slope cannot occur and a NaN total means a NaN curvature.
template <int G, int SPL, bool EXACT, bool CLAMP, bool SHIFT, int MODE, bool INCR = false, bool STEEP = false,
          bool TAB_GLOBAL = false>
__device__ __forceinline__ double chain_body(const ChainSpec &c, const CompConsts &kc,
                                             const float *__restrict__ init_seg, const float2 *s_tab, Planes st,
                                             uint32_t gbase, uint32_t j, uint32_t chain, bool real_chain,
                                             ChainOut *__restrict__ out, const ModeArgs &ma)
{
    constexpr bool FIX = !EXACT && MODE != kModeAdjoint;
    const uint32_t N = c.n_segments;
    using Lay = Layout<G, SPL>;
    // segment record (tangent, length) of segment index s = owner*SPL + m
    // the tangents are stored at length kscale; records handed to export and the adjoint are unit
    const float inv_ks = 1.0f / kc.kscale;
    auto load_rec = [&](uint32_t owner, uint32_t m) {
        const float2 a = st.xy[Lay::xy(gbase + owner, m)];
        return make_float4(a.x * inv_ks, a.y * inv_ks, st.z[Lay::z(gbase + owner, m)] * inv_ks, st.l[owner * SPL + m]);
    };

    float max_len = 0.f;
#pragma unroll
    for (int m = 0; m < SPL; ++m) {
        const uint32_t s = j * SPL + m;
        float x = 0.f, y = 0.f, z = 0.f, len = 1.f;
        if (s < N) {
            x = init_seg[3 * s];
            y = init_seg[3 * s + 1];
            z = init_seg[3 * s + 2];
            const float ss = fmaf(x, x, fmaf(y, y, z * z));
            const float r = rsqrtf(ss);
            len = ss * r;
            x *= r; y *= r; z *= r;
            const float h = fmaf(-0.5f, fmaf(x, x, fmaf(y, y, z * z)), 1.5f);   // one Newton step to |t| = 1
            x *= h * kc.kscale; y *= h * kc.kscale; z *= h * kc.kscale;       // stored at length kscale
            max_len = fmaxf(max_len, len);
        }
        st.xy[Lay::xy(gbase + j, m)] = make_float2(x, y);
        st.z[Lay::z(gbase + j, m)] = z;
    }
#pragma unroll
    for (int o = 1; o < G; o <<= 1) max_len = fmaxf(max_len, __shfl_xor_sync(FULL, max_len, o));
    // fixed-point chord scale: a segment is at most 2^24 units, 64 of them at most 2^30
    const float chord_scale = 16777216.0f / (max_len * kc.kscale);   // the tangents have length kscale
    const float renorm = -0.5f * inv_ks * inv_ks;   // Newton step to |t'| = kscale: 1.5 + renorm |t'|^2
    __syncwarp();

    const uint32_t steps_c = real_chain ? ((chain == c.n_chains - 1) ? c.last_steps : c.steps) : 0;
    const uint32_t total = c.burn_in + c.steps;
    const uint32_t gchain = c.chain0 + (real_chain ? chain : 0);
    // rotation rounds: sub-chains have at most k_eff segments (a step takes the warp's longest)
    const uint32_t max_rounds = (c.k_eff + G - 1) / G;
    // Shorter side (forward passes of shapes that hold at most 36 segments, and 4 x 12, where a
    // sub-chain can be longer than half the path): turning the complement of the sub-chain, [right, N)
    // and [0, left), by -theta about the same chord gives the moved path up to one rotation of
    // the whole path, and the weights see only curvatures, which that rotation leaves alone.
    // The chain then lives in a frame that turns with it. The sub-chain's chord is d minus the
    // complement's, d = the sum of l_s t_s over the whole path in that frame: carried through
    // every complement move (d <- R(-theta) d) and re-summed from the state every 16 steps, so
    // that its rounding cannot build up over a long chain. (The 4 x 16 shape, N = 37..64, is
    // left out: it gained 2 % at N = 48 and its code lost 5 % at N = 64, where no sub-chain is
    // longer than half the path; 4 x 12 took N = 37..48 from it, +5-10 % with the shorter side
    // over without.) The incremental form turns the same side, so that it follows
    // the full recompute's trajectory. Shapes of 4 or fewer segments per lane on more than one
    // lane are left out too: at their 64-register budget the second code path spilled (4 x 4,
    // N = 13..16, measured 5-25 % slower).
    constexpr bool CMPL = MODE == kModeForward && !SHIFT && G < 32 && (G * SPL <= 36 || (G == 4 && SPL == 12)) &&
                          (G == 1 || SPL > 4);
    const bool cmpl_on = CMPL && N < 2 * c.k_eff;
    float dX = 0.f, dY = 0.f, dZ = 0.f;
    float lse_m = 0.f, lse_s = 0.f, lse_c = 0.f;  // exact form: running max (float) and Kahan sum
    unsigned long long lse_t = 0;                   // fixed form: running max as a path total
    uint32_t valid = 0, failed = 0, clamped = 0;
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    // incremental form: the current path's integer total and whether a NaN curvature was met
    // since the last full recompute
    unsigned long long inc_tot = 0;
    bool inc_bad = false;
    uint32_t inc_since_full = 0;   // incremental steps since the last full recompute
    // tangent of segment s (any lane's) and the fixed-point term of the curvature between two
    // tangents, with its interpolation correction rounded on its own
    auto tan_at = [&](uint32_t s, float &x, float &y, float &z) {
        const float2 a = st.xy[Lay::xy(gbase + s / SPL, s % SPL)];
        x = a.x;
        y = a.y;
        z = st.z[Lay::z(gbase + s / SPL, s % SPL)];
    };
    auto term = [&](float ax, float ay, float az, float bx, float by, float bz, bool &nan) -> uint32_t {
        const float dx = bx - ax, dy = by - ay, dz = bz - az;
        int32_t L;
        uint32_t unused = 0;
        const float frac = bin_of<CLAMP>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), kc, false, unused, L);
        const float2 e = s_tab[L];
        const float cor = frac * e.y;
        nan |= isnan(cor);   // a NaN curvature or a steep bin's NaN slope
        return __float_as_uint(e.x) + (uint32_t)__float2int_rn(cor * kc.fscale);
    };

    const uint32_t own = gbase + j;
    // tangent of this lane's segment m; with SHIFT the weights see the receiver moved:
    // v_{N-2} = l t + shift, renormalised
    auto tan_smem = [&](int m, float &x, float &y, float &z) {
        const float2 a = st.xy[Lay::xy(own, m)];
        x = a.x;
        y = a.y;
        z = st.z[Lay::z(own, m)];
        if (SHIFT && j * SPL + m == N - 2) {
            const float l = st.l[j * SPL + m] * inv_ks;
            x = fmaf(l, x, c.eval_shift[0]);
            y = fmaf(l, y, c.eval_shift[1]);
            z = fmaf(l, z, c.eval_shift[2]);
            const float r = rsqrtf(fmaf(x, x, fmaf(y, y, z * z))) * kc.kscale;
            x *= r; y *= r; z *= r;
        }
    };
    const ShflNext<G> next_smem{};
    auto no_bins = [](uint32_t, int32_t) {};

    for (uint32_t base = 0; base < total; base += G) {
        const dev::Proposal pr = dev::draw_step(c.seed, c.experiment, gchain, base + j, N, c.k_eff, c.max_angle);
        float psn, pcs;
        dev::sincos_half(pr.angle, psn, pcs);
        const uint32_t nstep = min((uint32_t)G, total - base);
        for (uint32_t jj = 0; jj < nstep; ++jj) {
            const uint32_t k = __shfl_sync(FULL, pr.k, jj, G);
            const uint32_t left = __shfl_sync(FULL, pr.left, jj, G);
            const float sn = __shfl_sync(FULL, psn, jj, G);
            const float cs = __shfl_sync(FULL, pcs, jj, G);
            const uint32_t right = left + k;
            // the segments this chain turns: the sub-chain, or its complement where that is
            // shorter, on the steps where that takes two or more rounds off the warp's rotation
            // (a step that turns complements pays for the wrap and for carrying d: saving one
            // round of three, as at N = 13 and 14 on 4 x 4, measured slower)
            bool cm = false, use_c = false;
            uint32_t kmax;   // the longest turned side among the warp's chains
            if constexpr (CMPL) {
                if (cmpl_on && ((base + jj) & 15u) == 0u) {
                    dX = 0.f; dY = 0.f; dZ = 0.f;
#pragma unroll
                    for (int m = 0; m < SPL; ++m) {   // padding slots hold zero tangents
                        const float2 a = st.xy[Lay::xy(own, m)];
                        const float l = st.l[j * SPL + m];
                        dX = fmaf(l, a.x, dX);
                        dY = fmaf(l, a.y, dY);
                        dZ = fmaf(l, st.z[Lay::z(own, m)], dZ);
                    }
                    group_sum3<G>(dX, dY, dZ);
                }
                // whole-warp reductions: every chain of a warp belongs to one experiment (a CTA
                // runs one experiment's work item at a time), so cmpl_on is the same in every lane
                kmax = __reduce_max_sync(FULL, k);
                if (cmpl_on) {
                    const uint32_t kc = __reduce_max_sync(FULL, min(k, N - k));
                    use_c = (kc + G - 1) / G + 2 <= (kmax + G - 1) / G;   // the same for the whole warp
                    if (use_c) {
                        cm = N - k < k;
                        kmax = kc;
                    }
                }
            } else {
                kmax = k;
#pragma unroll
                for (int o = G; o < 32; o <<= 1) kmax = max(kmax, __shfl_xor_sync(FULL, kmax, o));
            }
            const uint32_t rounds = min((kmax + G - 1) / G, max_rounds);
            // incremental form: the two end curvatures before the rotation (kappa_{left-1} and
            // kappa_{right-1}; left >= 1 and right <= N-1, so all four tangents exist)
            bool incr_now = false;
            uint32_t t_old = 0;
            float e0x = 0.f, e0y = 0.f, e0z = 0.f, e3x = 0.f, e3y = 0.f, e3z = 0.f;
            if constexpr (INCR) {
                incr_now = base + jj > c.burn_in && inc_since_full + 1 < c.incr_resync;
                if (incr_now) {
                    float a1x, a1y, a1z, b0x, b0y, b0z;
                    tan_at(left - 1, e0x, e0y, e0z);
                    tan_at(left, a1x, a1y, a1z);
                    tan_at(right - 1, b0x, b0y, b0z);
                    tan_at(right, e3x, e3y, e3z);
                    t_old = term(e0x, e0y, e0z, a1x, a1y, a1z, inc_bad) + term(b0x, b0y, b0z, e3x, e3y, e3z, inc_bad);
                }
            }
            // chord x_right - x_left = sum of l_s t_s over the k segments left .. right-1
            // (k <= N - 2 < G * SPL, so a sub-chain never needs more than SPL rounds; a
            // complement turned instead is shorter than its sub-chain)
            constexpr int R = (kMaxSubChain + G - 1) / G < SPL ? (kMaxSubChain + G - 1) / G : SPL;
            // more than 4 rounds (8-lane groups) under the 64-register budget of 1024-thread
            // CTAs (SPL < 16): the rotation pass reloads its tangents instead of keeping every
            // round's in registers (measured: no spills, N <= 64 up to 27 % faster)
            constexpr bool RELOAD = R > 4 && (SPL < 16 || G < 8);
            constexpr int RK = RELOAD ? 1 : R;
            // The move: the chord of the turned segments, the axis, the rotation. WRAP: the warp
            // turns complements this step (the chains with cm), which wrap past segment N-1 to 0,
            // turn by -theta and carry d; a step that turns none runs the plain code.
            auto turn = [&](auto wrap_tag) {
                constexpr bool WRAP = decltype(wrap_tag)::value;
                const bool cmw = WRAP && cm;
                const uint32_t first = cmw ? right : left;
                const uint32_t cnt = cmw ? N - k : k;
                auto seg_of = [&](uint32_t idx) {
                    uint32_t s = first + idx;
                    if (WRAP && s >= N) s -= N;
                    return s;
                };
                float vx[RK], vy[RK], vz[RK];
                uint32_t va[RK], vb[RK];
                float cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r > 0 && (uint32_t)r >= rounds) break;
                    const uint32_t idx = j + r * G;
                    const uint32_t s = seg_of(idx);
                    const int ri = RELOAD ? 0 : r;
                    va[ri] = Lay::xy(gbase + s / SPL, s % SPL);
                    vb[ri] = Lay::z(gbase + s / SPL, s % SPL);
                    if (WRAP ? idx < cnt : s < right) {
                        const float2 a = st.xy[va[ri]];
                        vx[ri] = a.x;
                        vy[ri] = a.y;
                        vz[ri] = st.z[vb[ri]];
                        const float l = st.l[s];
                        cx = fmaf(l, vx[ri], cx);
                        cy = fmaf(l, vy[ri], cy);
                        cz = fmaf(l, vz[ri], cz);
                    }
                }
                if constexpr (G == 32) {
                    int ix = __float2int_rn(cx * chord_scale);
                    int iy = __float2int_rn(cy * chord_scale);
                    int iz = __float2int_rn(cz * chord_scale);
                    ix = __reduce_add_sync(FULL, ix);
                    iy = __reduce_add_sync(FULL, iy);
                    iz = __reduce_add_sync(FULL, iz);
                    cx = (float)ix;
                    cy = (float)iy;
                    cz = (float)iz;
                } else {
                    group_sum3<G>(cx, cy, cz);
                }
                if (cmw) { cx = dX - cx; cy = dY - cy; cz = dZ - cz; }   // the sub-chain's chord
                // Rodrigues by +theta about the unit chord a -- the rotation the reference's
                // quaternion sandwich q^-1 p q applies with its product convention:
                // v cos + (a x v) sin + a (a.v)(1 - cos), sin = 2 s c, 1 - cos = 2 s^2 (half angle s, c)
                const float inv = rsqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz)));
                const float ax = cx * inv, ay = cy * inv, az = cz * inv;
                const float sth = (cmw ? -2.f : 2.f) * sn * cs, omc = 2.f * sn * sn;
                // Groups of 1 or 4 lanes (up to 32 or 8 rounds): the rotation as v + M v with
                // M = R - I = sin(theta) [a]x + (1 - cos(theta)) (a a^T - I), built once per step,
                // 9 FMAs per segment against 19 for the Rodrigues form (the correction is added
                // to v, so it rounds like the Rodrigues terms do). Measured +4.6-5.5 % at
                // N = 8..24 and +1-2 % at N = 32..96; with 8-lane groups (4 rounds) 1.9 % slower
                // at N = 128, so those keep the Rodrigues form.
                constexpr bool RMAT = G <= 4;
                float m00 = 0.f, m01 = 0.f, m02 = 0.f, m10 = 0.f, m11 = 0.f, m12 = 0.f, m20 = 0.f, m21 = 0.f, m22 = 0.f;
                if constexpr (RMAT) {
                    const float oax = omc * ax, oay = omc * ay, oaz = omc * az;
                    const float sax = sth * ax, say = sth * ay, saz = sth * az;
                    m00 = fmaf(oax, ax, -omc);
                    m11 = fmaf(oay, ay, -omc);
                    m22 = fmaf(oaz, az, -omc);
                    m01 = fmaf(oax, ay, -saz);
                    m10 = fmaf(oax, ay, saz);
                    m02 = fmaf(oax, az, say);
                    m20 = fmaf(oax, az, -say);
                    m12 = fmaf(oay, az, -sax);
                    m21 = fmaf(oay, az, sax);
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r > 0 && (uint32_t)r >= rounds) break;
                    const uint32_t idx = j + r * G;
                    const uint32_t s = seg_of(idx);
                    const int ri = RELOAD ? 0 : r;
                    if (RELOAD) {
                        va[0] = Lay::xy(gbase + s / SPL, s % SPL);
                        vb[0] = Lay::z(gbase + s / SPL, s % SPL);
                    }
                    if (WRAP ? idx < cnt : s < right) {
                        if (RELOAD) {
                            const float2 a = st.xy[va[0]];
                            vx[0] = a.x;
                            vy[0] = a.y;
                            vz[0] = st.z[vb[0]];
                        }
                        const float x = vx[ri], y = vy[ri], z = vz[ri];
                        float nx, ny, nz;
                        if constexpr (RMAT) {
                            nx = fmaf(m00, x, fmaf(m01, y, fmaf(m02, z, x)));
                            ny = fmaf(m10, x, fmaf(m11, y, fmaf(m12, z, y)));
                            nz = fmaf(m20, x, fmaf(m21, y, fmaf(m22, z, z)));
                        } else {
                            const float crx = ay * z - az * y, cry = az * x - ax * z, crz = ax * y - ay * x;
                            const float ad = (ax * x + ay * y + az * z) * omc;
                            nx = fmaf(ax, ad, fmaf(sth, crx, fmaf(-omc, x, x)));
                            ny = fmaf(ay, ad, fmaf(sth, cry, fmaf(-omc, y, y)));
                            nz = fmaf(az, ad, fmaf(sth, crz, fmaf(-omc, z, z)));
                        }
                        const float h = fmaf(renorm, fmaf(nx, nx, fmaf(ny, ny, nz * nz)), 1.5f);
                        st.xy[va[ri]] = make_float2(nx * h, ny * h);
                        st.z[vb[ri]] = nz * h;
                    }
                }
                if constexpr (WRAP) {
                    // the whole path's chord turns with the complement (selected, not branched)
                    const float crx = ay * dZ - az * dY, cry = az * dX - ax * dZ, crz = ax * dY - ay * dX;
                    const float ad = (ax * dX + ay * dY + az * dZ) * omc;
                    const float nX = fmaf(ax, ad, fmaf(sth, crx, fmaf(-omc, dX, dX)));
                    const float nY = fmaf(ay, ad, fmaf(sth, cry, fmaf(-omc, dY, dY)));
                    const float nZ = fmaf(az, ad, fmaf(sth, crz, fmaf(-omc, dZ, dZ)));
                    dX = cm ? nX : dX;
                    dY = cm ? nY : dY;
                    dZ = cm ? nZ : dZ;
                }
            };
            if constexpr (CMPL) {
                if (use_c) turn(BoolTag<true>{});
                else turn(BoolTag<false>{});
            } else {
                turn(BoolTag<false>{});
            }
            __syncwarp();
            const uint32_t step = base + jj;
            if (step < c.burn_in) continue;
            const uint32_t wstep = step - c.burn_in;
            const bool active = wstep < steps_c;

            if (FIX) {
                bool bad = false;
                unsigned long long tot = 0;
                bool need_full = true;
                if constexpr (INCR) {
                    if (incr_now) {
                        // the two end curvatures after the rotation; the interior ones keep their terms
                        // (a turned complement moved the outer tangents of the two joints instead)
                        float a1x, a1y, a1z, b0x, b0y, b0z;
                        if (cm) {
                            tan_at(left - 1, e0x, e0y, e0z);
                            tan_at(right, e3x, e3y, e3z);
                        }
                        tan_at(left, a1x, a1y, a1z);
                        tan_at(right - 1, b0x, b0y, b0z);
                        const uint32_t t_new =
                              term(e0x, e0y, e0z, a1x, a1y, a1z, inc_bad) + term(b0x, b0y, b0z, e3x, e3y, e3z, inc_bad);
                        inc_tot += (unsigned long long)(long long)(int32_t)(t_new - t_old);
                        need_full = inc_bad;
                    }
                }
                // one decision per warp: the full recompute shuffles across the whole warp, and
                // every chain of the warp then stays on the same resync schedule
                if (INCR && !__any_sync(FULL, need_full)) {
                    tot = inc_tot;
                    ++inc_since_full;
                } else {
                    tot = path_fixed<G, SPL, CLAMP, TAB_GLOBAL>(j, gbase, N, s_tab, kc, tan_smem, next_smem, bad, clamped);
                    // a NaN slope marks a steep bin, where the secant would err by more than
                    // 1e-7: weigh such paths (rare) with the exact blend through the linear
                    // table; only a NaN curvature leaves a path invalid
                    if constexpr (STEEP) {
                        if (__any_sync(FULL, bad)) {
                            const double wx = steep_fallback<G, SPL, CLAMP>(st, gbase, j, N, ma.lin, kc);
                            if (bad && !isnan(wx)) {
                                bad = false;
                                tot = (unsigned long long)llrint(fmax(0.0, (wx - kc.lw_offset) * (double)kc.fscale));
                            }
                        }
                    }
                    inc_tot = tot;
                    inc_bad = bad;
                    inc_since_full = 0;
                }
                if (MODE == kModeExport) {
                    const double w = bad ? NAN : kc.lw_offset + (double)tot * kc.inv_scale;
                    // positions below
                    if (active) {
                        const size_t pidx = (size_t)chain * c.steps + wstep;
                        if (j == 0) ma.exp_w[pidx] = isnan(w) ? NAN : w + (N - 1) * ma.log10_abs;
                    }
                }
                if (MODE == kModeExport && ma.exp_pos) {
                    // positions x_0 + prefix sums of l_s t_s, in double; every lane takes part in
                    // the scan, only active chains write (a weights-only replay passes no buffer)
                    double px = 0.0, py = 0.0, pz = 0.0;
                    double lx[SPL], ly[SPL], lz[SPL];
#pragma unroll
                    for (int m = 0; m < SPL; ++m) {
                        const float4 v = load_rec(j, m);
                        const double l = (j * SPL + m < N) ? (double)v.w : 0.0;
                        px += l * (double)v.x;
                        py += l * (double)v.y;
                        pz += l * (double)v.z;
                        lx[m] = px; ly[m] = py; lz[m] = pz;
                    }
                    double ex = px, ey = py, ez = pz;  // inclusive scan of lane totals
#pragma unroll
                    for (int o = 1; o < G; o <<= 1) {
                        const double ux = __shfl_up_sync(FULL, ex, o, G), uy = __shfl_up_sync(FULL, ey, o, G),
                                     uz = __shfl_up_sync(FULL, ez, o, G);
                        if ((int)j >= o) { ex += ux; ey += uy; ez += uz; }
                    }
                    ex -= px; ey -= py; ez -= pz;  // exclusive
                    if (active) {
                        const size_t pidx = (size_t)chain * c.steps + wstep;
                        float *dst = ma.exp_pos + pidx * 3 * (size_t)(N + 1);
                        if (j == 0) { dst[0] = ma.x0[0]; dst[1] = ma.x0[1]; dst[2] = ma.x0[2]; }
#pragma unroll
                        for (int m = 0; m < SPL; ++m) {
                            const uint32_t s = j * SPL + m;
                            if (s < N) {
                                dst[3 * (s + 1)] = (float)((double)ma.x0[0] + ex + lx[m]);
                                dst[3 * (s + 1) + 1] = (float)((double)ma.x0[1] + ey + ly[m]);
                                dst[3 * (s + 1) + 2] = (float)((double)ma.x0[2] + ez + lz[m]);
                            }
                        }
                    }
                }
                if (!active) continue;
                if (bad) {
                    ++failed;
                    continue;
                }
                if (valid == 0) {
                    lse_t = tot;
                    lse_s = 1.f;
                    lse_c = 0.f;
                } else {
                    // exact integer difference: narrow totals stay below 2^31, wide ones are 64-bit
                    const float dt = kc.wide ? (float)(long long)(tot - lse_t)
                                             : (float)(int32_t)((uint32_t)tot - (uint32_t)lse_t);
                    const float x = dt * kc.l2s;
                    float term = 1.f;
                    if (x > 0.f) {
                        const float f = ex2_approx(-x);
                        lse_s *= f;
                        lse_c *= f;
                        lse_t = tot;
                    } else {
                        term = ex2_approx(x);
                    }
                    kahan_add(lse_s, lse_c, term);
                }
                ++valid;
                continue;
            }

            double w;
            if (MODE == kModeAdjoint) {
                // log10 weight and d/d(mu_s), d/d(eps) of this lane's segments (exact blend): the
                // blend from the staged linear table, the derivative blends from one 16-byte load
                float s = 0.f, cc = 0.f, gmu = 0.f, geps = 0.f;
                auto adj_seg = [&](uint32_t, float qq, bool valid) {
                    float r = sqrt_approx(qq) + kc.roff;   // scaled tangents: the root is the bin index
                    if (r < 0.f) r = 0.f;
                    if (r > kc.rmax) r = kc.rmax;
                    // floor(r) by a round-down add, as bin_of takes it (no float/int conversions
                    // on the MUFU pipe, which the blend's log2 and reciprocal already load;
                    // measured 1.8 % off the differentiation configuration's adjoint call)
                    const float fl = __fadd_rd(r, 8388608.0f);
                    const int32_t L = (int32_t)min(__float_as_uint(fl) - 0x4B000000u, (uint32_t)kc.bins - 1u);
                    const float d = (r - (fl - 8388608.0f)) * kc.step;
                    const float2 e = s_tab[L];
                    const float4 dv = __ldg(ma.dtab + L);
                    const float v = fmaf(d, e.y, e.x);
                    kahan_add(s, cc, valid ? __log2f(v) * kLog10_2 : 0.0f);
                    const float iv = __fdividef(1.0f, v);
                    gmu += valid ? fmaf(d, dv.y, dv.x) * iv : 0.0f;
                    geps += valid ? fmaf(d, dv.w, dv.z) * iv : 0.0f;
                };
                // a chain that fills its group's slots walks them with validity known at compile
                // time (every curvature but the group's last boundary), as the forward recompute does
                if (N == (uint32_t)(G * SPL))
                    for_curvatures<G, SPL, true>(j, N, tan_smem, next_smem, adj_seg);
                else
                    for_curvatures<G, SPL, false>(j, N, tan_smem, next_smem, adj_seg);
                float hi = s, lo = -cc;
                group_sum_pair<G>(hi, lo);
                w = (double)hi + (double)lo;
                float g3[3] = {0.f, 0.f, 0.f};
                if (j == 0) {
                    const float4 v3 = load_rec((N - 3) / SPL, (N - 3) % SPL);
                    const float4 v2 = load_rec((N - 2) / SPL, (N - 2) % SPL);
                    const float4 v1 = load_rec((N - 1) / SPL, (N - 1) % SPL);
                    const float t3[3] = {v3.x, v3.y, v3.z}, t2[3] = {v2.x, v2.y, v2.z}, t1[3] = {v1.x, v1.y, v1.z};
                    receiver_grad(t3, t2, t1, v2.w, s_tab, kc, c.inv_ds, g3);
                }
                if (active && !isnan(w)) {
                    const float wt = exp2f((float)(w - (double)ma.ref_log10) * kLog2_10);
                    acc[0] += wt * gmu * kInvLn10;
                    acc[1] += wt * geps * kInvLn10;
                    acc[2] += wt * g3[0];
                    acc[3] += wt * g3[1];
                    acc[4] += wt * g3[2];
                    if (j == 0) acc[5] += wt;
                }
            } else {
                w = path_log10<G, SPL, true, CLAMP, TAB_GLOBAL>(j, N, s_tab, kc, tan_smem, next_smem, no_bins, clamped);
            }
            if (MODE == kModeExport && !ma.exp_pos && active && j == 0)   // weights-only replay
                ma.exp_w[(size_t)chain * c.steps + wstep] = isnan(w) ? NAN : w + (N - 1) * ma.log10_abs;
            if (MODE == kModeExport && ma.exp_pos) {
                double px = 0.0, py = 0.0, pz = 0.0;
                double lx[SPL], ly[SPL], lz[SPL];
#pragma unroll
                for (int m = 0; m < SPL; ++m) {
                    const float4 v = load_rec(j, m);
                    const double l = (j * SPL + m < N) ? (double)v.w : 0.0;
                    px += l * (double)v.x;
                    py += l * (double)v.y;
                    pz += l * (double)v.z;
                    lx[m] = px; ly[m] = py; lz[m] = pz;
                }
                double ex = px, ey = py, ez = pz;
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    const double ux = __shfl_up_sync(FULL, ex, o, G), uy = __shfl_up_sync(FULL, ey, o, G),
                                 uz = __shfl_up_sync(FULL, ez, o, G);
                    if ((int)j >= o) { ex += ux; ey += uy; ez += uz; }
                }
                ex -= px; ey -= py; ez -= pz;
                if (active) {
                    const size_t pidx = (size_t)chain * c.steps + wstep;
                    float *dst = ma.exp_pos + pidx * 3 * (size_t)(N + 1);
                    if (j == 0) { dst[0] = ma.x0[0]; dst[1] = ma.x0[1]; dst[2] = ma.x0[2]; }
#pragma unroll
                    for (int m = 0; m < SPL; ++m) {
                        const uint32_t s = j * SPL + m;
                        if (s < N) {
                            dst[3 * (s + 1)] = (float)((double)ma.x0[0] + ex + lx[m]);
                            dst[3 * (s + 1) + 1] = (float)((double)ma.x0[1] + ey + ly[m]);
                            dst[3 * (s + 1) + 2] = (float)((double)ma.x0[2] + ez + lz[m]);
                        }
                    }
                    if (j == 0) ma.exp_w[pidx] = isnan(w) ? NAN : w + (N - 1) * ma.log10_abs;
                }
            }
            if (!active) continue;
            if (isnan(w)) {
                ++failed;
                continue;
            }
            const float hi = (float)w;
            const float lo = (float)(w - (double)hi);
            if (valid == 0) {
                lse_m = hi;
                lse_s = exp2f(lo * kLog2_10);
                lse_c = 0.f;
                valid = 1;
            } else {
                const float x = (hi - lse_m) + lo;
                float term;
                if (x > 0.f) {
                    const float f = exp2f((lse_m - hi) * kLog2_10);
                    lse_s *= f;
                    lse_c *= f;
                    lse_m = hi;
                    term = exp2f(lo * kLog2_10);
                } else {
                    term = exp2f(x * kLog2_10);
                }
                kahan_add(lse_s, lse_c, term);
                ++valid;
            }
        }
    }
    clamped = group_sum<G>(clamped);
    if (MODE == kModeAdjoint) {
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[i] = group_sum<G>(acc[i]);
        if (j == 0 && real_chain)
            for (int i = 0; i < 6; ++i) ma.grad[(size_t)chain * 6 + i] = (double)acc[i];
    }
    double chain_log10 = -INFINITY;
    if (valid) {
        const double head = FIX ? kc.lw_offset + (double)lse_t * kc.inv_scale : (double)lse_m;
        chain_log10 = head + log10((double)lse_s - (double)lse_c) + (double)(N - 1) * ma.log10_abs;
    }
    if (j == 0 && real_chain && out) {
        ChainOut o;
        o.log10_sum = chain_log10;
        o.valid = valid;
        o.failed = failed;
        o.clamped = clamped;
        o.pad = 0;
        out[chain] = o;
    }
    return real_chain ? chain_log10 : -INFINITY;
}

CompConsts make_consts(float inv_ds, const LutMetaF &m, uint32_t n_segments, const LogFixed &lf)
{
    CompConsts k;
    k.kscale = inv_ds / m.step;
    k.roff = -m.min_k / m.step;
    k.rmax = (m.max_k - m.min_k) / m.step;
    k.rsnap = 1e-3f / m.step;
    k.step = m.step;
    k.bins = m.bins;
    k.lw_offset = (double)(n_segments - 1) * lf.c0;
    k.inv_scale = lf.inv_scale;
    k.fscale = lf.inv_scale > 0.0 ? (float)(1.0 / lf.inv_scale) : 0.0f;
    k.l2s = (float)(lf.inv_scale * 3.321928094887362);
    k.wide = lf.wide;
    return k;
}

// A table whose range covers every curvature unit tangents can produce, |t_{i+1}-t_i| <= 2
// (with margin for rounding), needs no clamping.
bool table_needs_clamp(const CompConsts &k) { return !(k.roff == 0.0f && k.rmax >= 2.0001f * k.kscale); }

}  // namespace
}  // namespace twisty
