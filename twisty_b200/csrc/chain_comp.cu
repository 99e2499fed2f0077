// chain_comp.cu -- the compensated B200 form of the Markov-chain hot path.
//
// Algorithm: the reference's GeometryRandom loop (Twisty/FullExperimentRunnerOptimalPerturb.cpp:
// 469-595): per step, rotate the points strictly between a random pivot `left` and
// `right = left + k` about the axis x_right - x_left by a random angle, recompute every
// tangent and curvature, gather each curvature's weight from the table, sum the log10
// weights, and accumulate the path weight into the experiment's running sum.
//
// B200 layout and arithmetic:
//  * G lanes cooperate on one chain (G = 8, 16 or 32); lane j owns the SPL contiguous
//    segments j*SPL .. j*SPL+SPL-1. The chain lives in shared memory as its N segment
//    vectors v_i = x_{i+1} - x_i (three planes x/y/z). A rotation of the points between
//    left and right about the chord x_right - x_left maps every segment vector
//    v_left .. v_{right-1} by the same rotation (the chord is the axis, so it is fixed),
//    which keeps segment-scale magnitudes (|v| ~ ds) instead of absolute positions in the
//    FP32 state: the rounding of the state is relative to ds, not to |x|.
//  * Shared-memory address of segment s = j*SPL + m of the chain in lanes q*G..q*G+G-1:
//    row m, column (q*G + j + m*C) mod 32 with C = max(1, G/SPL). Rows make the full
//    recompute (all lanes, same m) conflict-free; the column shift spreads the k
//    consecutive segments of a rotation over distinct banks (at most 2-way conflicts).
//  * The table is staged once per CTA in shared memory as float2 (log10 L_i, secant slope),
//    so a segment's log-weight is one 8-byte LDS and one FMA; when the secant is not
//    accurate to 1e-7 per segment the host selects EXACT mode ((L_i, L_{i+1}-L_i) and a
//    log2). The per-path log10 sum is Kahan-compensated in FP32 and combined across lanes
//    with TwoSum; the chain's running sum is a log-sum-exp accumulator rescaled by its
//    running maximum (FP32 with a compensated mantissa sum). FP64 appears only in the
//    per-CTA log-sum-exp reduction of the chains and the global reduction.
//  * Proposals: lane j of a group draws the Philox proposal of step base+j (one draw per
//    lane per G steps) and shuffles broadcast it, so the RNG costs 1/G of a draw per lane
//    per step.
#include "kernels.h"
#include "device_common.cuh"

#include <cfloat>

namespace twisty {
namespace {

constexpr uint32_t FULL = 0xffffffffu;
constexpr int kMaxSubChain = 64;            // largest k the rotation rounds cover
constexpr float kLog2_10 = 3.32192809488736234787f;
constexpr float kLog10_2 = 0.30102999566398119521f;
constexpr float kInvLn10 = 0.43429448190325182765f;

struct CompConsts {
    float kscale;        // (N/S) / step : |t_{i+1}-t_i| -> fractional bin index
    float roff;          // -min_k / step
    float rmax;          // (max_k - min_k) / step
    float rsnap;         // 1e-3 / step: overshoot that counts as clamped
    float step;
    int32_t bins;
};

__device__ __forceinline__ float sqrt_approx(float x)
{
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
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

template <int G>
__device__ __forceinline__ uint32_t group_sum_u(uint32_t v)
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

// Log-weight of one segment given |t_{i+1}-t_i|^2; NaN propagates to mark the path invalid.
template <bool EXACT>
__device__ __forceinline__ float segment_term(float qq, const float2 *__restrict__ tab, const CompConsts &k,
                                              uint32_t &clamped, int32_t *bin_out)
{
    float r = fmaf(sqrt_approx(qq), k.kscale, k.roff);
    if (r < 0.0f) r = 0.0f;
    if (r > k.rmax) {
        clamped += (r - k.rmax >= k.rsnap) ? 1u : 0u;
        r = k.rmax;
    }
    const int32_t L = min((int32_t)r, k.bins - 1);
    if (bin_out) *bin_out = isnan(r) ? -1 : L;
    const float d = (r - (float)L) * k.step;
    const float2 e = tab[L];
    if (EXACT) return __log2f(fmaf(d, e.y, e.x)) * kLog10_2;
    return fmaf(d, e.y, e.x);
}

// Full recompute of one path's log10 weight from its segment vectors. seg(m, x, y, z)
// loads segment j*SPL+m of this lane. Returns the group-wide (hi, lo).
template <int G, int SPL, bool EXACT, class SegFn, class BinFn>
__device__ __forceinline__ void path_log10(uint32_t j, uint32_t N, const float2 *__restrict__ tab,
                                           const CompConsts &k, SegFn seg, BinFn bin_sink, float &hi,
                                           float &lo, uint32_t &clamped)
{
    float s = 0.0f, c = 0.0f;
    float t0x = 0.f, t0y = 0.f, t0z = 0.f, px = 0.f, py = 0.f, pz = 0.f;
    const uint32_t base = j * SPL;
#pragma unroll
    for (int m = 0; m < SPL; ++m) {
        float vx, vy, vz;
        seg(m, vx, vy, vz);
        const float rs = rsqrtf(fmaf(vx, vx, fmaf(vy, vy, vz * vz)));
        const float tx = vx * rs, ty = vy * rs, tz = vz * rs;
        if (m == 0) {
            t0x = tx; t0y = ty; t0z = tz;
        } else if (base + m <= N - 1) {
            const float dx = tx - px, dy = ty - py, dz = tz - pz;
            int32_t b;
            const float term = segment_term<EXACT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), tab, k, clamped, &b);
            bin_sink(base + m - 1, b);
            kahan_add(s, c, term);
        }
        px = tx; py = ty; pz = tz;
    }
    const float nx = __shfl_down_sync(FULL, t0x, 1, G);
    const float ny = __shfl_down_sync(FULL, t0y, 1, G);
    const float nz = __shfl_down_sync(FULL, t0z, 1, G);
    if (base + SPL <= N - 1) {
        const float dx = nx - px, dy = ny - py, dz = nz - pz;
        int32_t b;
        const float term = segment_term<EXACT>(fmaf(dx, dx, fmaf(dy, dy, dz * dz)), tab, k, clamped, &b);
        bin_sink(base + SPL - 1, b);
        kahan_add(s, c, term);
    }
    hi = s;
    lo = -c;
    group_sum_pair<G>(hi, lo);
}

template <int G, int SPL>
struct Layout {
    static constexpr int C = (G / SPL) > 1 ? (G / SPL) : 1;
    __device__ __forceinline__ static uint32_t addr(uint32_t lane_in_warp_base, uint32_t owner, uint32_t m)
    {
        return m * 32u + ((lane_in_warp_base + owner + m * C) & 31u);
    }
};

enum { kModeForward = 0, kModeExport = 1, kModeAdjoint = 2 };

// Receiver-position gradient of one path's log10 weight, computed by one lane from the
// last three segment vectors: moving the receiver moves points N-1 and N together, so only
// v_{N-2} changes, hence t_{N-2} and the curvatures kappa_{N-3}, kappa_{N-2}. The table's
// slope is taken per bin, (L_{i+1} - L_i) / step, the derivative of the curve the table
// samples (the reference's interpolation weight in curvature units makes its own weight
// almost piecewise constant within a bin, a slope finite differences do not see).
__device__ __forceinline__ void receiver_grad(const float *sx, const float *sy, const float *sz, uint32_t a3,
                                              uint32_t a2, uint32_t a1, const float *__restrict__ lut,
                                              const CompConsts &k, float inv_ds, float g[3])
{
    const float v3x = sx[a3], v3y = sy[a3], v3z = sz[a3];   // v_{N-3}
    const float v2x = sx[a2], v2y = sy[a2], v2z = sz[a2];   // v_{N-2}
    const float v1x = sx[a1], v1y = sy[a1], v1z = sz[a1];   // v_{N-1}
    const float r3 = rsqrtf(fmaf(v3x, v3x, fmaf(v3y, v3y, v3z * v3z)));
    const float r2 = rsqrtf(fmaf(v2x, v2x, fmaf(v2y, v2y, v2z * v2z)));
    const float r1 = rsqrtf(fmaf(v1x, v1x, fmaf(v1y, v1y, v1z * v1z)));
    const float t3[3] = {v3x * r3, v3y * r3, v3z * r3};
    const float t2[3] = {v2x * r2, v2y * r2, v2z * r2};
    const float t1[3] = {v1x * r1, v1y * r1, v1z * r1};
    // d t2 / d v2 = (I - t2 t2^T) * r2
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
        const int32_t L = min((int32_t)r, k.bins - 1);
        const int32_t R = min(L + 1, k.bins - 1);
        const float lv = __ldg(lut + L), rv = __ldg(lut + R);
        const float dd = (r - (float)L) * k.step;
        const float blend = fmaf(dd, rv - lv, lv);
        // d log10(w)/d kappa, per unit curvature
        const float dlog = (rv - lv) / (k.step * blend) * kInvLn10;
        const float dk = dlog * inv_ds * sign / dn;  // d kappa / d t = inv_ds * d/|d| (sign per term)
        // project through (I - t2 t2^T) r2
        const float dt = d[0] * t2[0] + d[1] * t2[1] + d[2] * t2[2];
        for (int q = 0; q < 3; ++q) g[q] += dk * (d[q] - dt * t2[q]) * r2;
    }
}

struct ModeArgs {
    // export
    float *exp_pos;      // [chains][steps][N+1][3]
    double *exp_w;       // [chains][steps] log10 weights (absorption included, normaliser not)
    float x0[3];
    double log10_abs;
    // adjoint
    const float *lut;    // float table
    const float *dmu;    // d table / d mu_s
    const float *deps;   // d table / d eps
    float ref_log10;     // log10 of the forward sum of path weights (normaliser excluded)
    double *grad;        // [chains][6]: d/dmu_s, d/deps, d/dx, d/dy, d/dz (log10 units), sum of weights
};

// Stage a table of `bins` float2 entries into shared memory (float4 vector loads).
__device__ __forceinline__ void stage_table(float4 *smem4, const float2 *__restrict__ tab_g, int bins)
{
    for (int i = threadIdx.x; i < bins / 2; i += blockDim.x) smem4[i] = reinterpret_cast<const float4 *>(tab_g)[i];
    if ((bins & 1) && threadIdx.x == 0) reinterpret_cast<float2 *>(smem4)[bins - 1] = tab_g[bins - 1];
}

// One Markov chain run by the G lanes of one group, on its own shared-memory segment
// planes sx/sy/sz: initial state from init_seg, burn_in + steps proposals, a full
// recompute of every weighted path, and the chain's running log-sum-exp. Writes out[chain]
// (when out is set and the chain is real) and returns the chain's log10 sum.
template <int G, int SPL, bool EXACT, int MODE>
__device__ __forceinline__ double chain_body(const ChainSpec &c, const CompConsts &kc,
                                             const float *__restrict__ init_seg, const float2 *s_tab, float *sx,
                                             float *sy, float *sz, uint32_t gbase, uint32_t j, uint32_t chain,
                                             bool real_chain, ChainOut *__restrict__ out, const ModeArgs &ma)
{
    const uint32_t N = c.n_segments;
    using Lay = Layout<G, SPL>;

#pragma unroll
    for (int m = 0; m < SPL; ++m) {
        const uint32_t s = j * SPL + m;
        const uint32_t a = Lay::addr(gbase, j, m);
        const bool in = s < N;
        sx[a] = in ? init_seg[3 * s] : 0.f;
        sy[a] = in ? init_seg[3 * s + 1] : 0.f;
        sz[a] = in ? init_seg[3 * s + 2] : 0.f;
    }
    __syncwarp();

    const uint32_t steps_c = real_chain ? ((chain == c.n_chains - 1) ? c.last_steps : c.steps) : 0;
    const uint32_t total = c.burn_in + c.steps;
    const uint32_t gchain = c.chain0 + (real_chain ? chain : 0);
    float lse_m = 0.f, lse_s = 0.f, lse_c = 0.f;
    uint32_t valid = 0, failed = 0, clamped = 0;
    float acc[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};

    auto seg_smem = [&](int m, float &x, float &y, float &z) {
        const uint32_t a = Lay::addr(gbase, j, m);
        x = sx[a];
        y = sy[a];
        z = sz[a];
        if (c.has_eval_shift && j * SPL + m == N - 2) {
            x += c.eval_shift[0];
            y += c.eval_shift[1];
            z += c.eval_shift[2];
        }
    };
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
            // chord x_right - x_left = sum of the k segment vectors left .. right-1
            constexpr int R = (kMaxSubChain + G - 1) / G;
            float vx[R], vy[R], vz[R];
            uint32_t va[R];
            float cx = 0.f, cy = 0.f, cz = 0.f;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t s = left + j + r * G;
                va[r] = Lay::addr(gbase, s / SPL, s % SPL);
                if (s < right) {
                    vx[r] = sx[va[r]];
                    vy[r] = sy[va[r]];
                    vz[r] = sz[va[r]];
                    cx += vx[r];
                    cy += vy[r];
                    cz += vz[r];
                }
            }
            group_sum3<G>(cx, cy, cz);
            const float inv = rsqrtf(fmaf(cx, cx, fmaf(cy, cy, cz * cz)));
            const float qx = cx * inv * sn, qy = cy * inv * sn, qz = cz * inv * sn, qw = cs;
            // rotation of q^-1 p q (the reference's quaternion sandwich), as a matrix
            const float r00 = 1.f - 2.f * (qy * qy + qz * qz), r01 = 2.f * (qx * qy - qw * qz), r02 = 2.f * (qx * qz + qw * qy);
            const float r10 = 2.f * (qx * qy + qw * qz), r11 = 1.f - 2.f * (qx * qx + qz * qz), r12 = 2.f * (qy * qz - qw * qx);
            const float r20 = 2.f * (qx * qz - qw * qy), r21 = 2.f * (qy * qz + qw * qx), r22 = 1.f - 2.f * (qx * qx + qy * qy);
            __syncwarp();
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t s = left + j + r * G;
                if (s < right) {
                    const float x = vx[r], y = vy[r], z = vz[r];
                    sx[va[r]] = fmaf(r00, x, fmaf(r01, y, r02 * z));
                    sy[va[r]] = fmaf(r10, x, fmaf(r11, y, r12 * z));
                    sz[va[r]] = fmaf(r20, x, fmaf(r21, y, r22 * z));
                }
            }
            __syncwarp();
            const uint32_t step = base + jj;
            if (step < c.burn_in) continue;
            const uint32_t wstep = step - c.burn_in;
            const bool active = wstep < steps_c;
            float hi, lo;
            if (MODE == kModeAdjoint) {
                // log10 weight and d/d(mu_s), d/d(eps) of this lane's segments (exact blend)
                float s = 0.f, cc = 0.f, gmu = 0.f, geps = 0.f;
                float t0x = 0.f, t0y = 0.f, t0z = 0.f, px = 0.f, py = 0.f, pz = 0.f;
                const uint32_t b0 = j * SPL;
                auto seg_term = [&](float qq) {
                    float r = fmaf(sqrt_approx(qq), kc.kscale, kc.roff);
                    if (r < 0.f) r = 0.f;
                    if (r > kc.rmax) r = kc.rmax;
                    const int32_t L = min((int32_t)r, kc.bins - 1);
                    const int32_t Rb = min(L + 1, kc.bins - 1);
                    const float d = (r - (float)L) * kc.step;
                    const float lv = __ldg(ma.lut + L), rv = __ldg(ma.lut + Rb);
                    const float v = fmaf(d, rv - lv, lv);
                    kahan_add(s, cc, __log2f(v) * kLog10_2);
                    const float ml = __ldg(ma.dmu + L), mr = __ldg(ma.dmu + Rb);
                    const float el = __ldg(ma.deps + L), er = __ldg(ma.deps + Rb);
                    gmu += fmaf(d, mr - ml, ml) / v;
                    geps += fmaf(d, er - el, el) / v;
                };
#pragma unroll
                for (int m = 0; m < SPL; ++m) {
                    float x, y, z;
                    seg_smem(m, x, y, z);
                    const float rs = rsqrtf(fmaf(x, x, fmaf(y, y, z * z)));
                    const float tx = x * rs, ty = y * rs, tz = z * rs;
                    if (m == 0) { t0x = tx; t0y = ty; t0z = tz; }
                    else if (b0 + m <= N - 1) {
                        const float dx = tx - px, dy = ty - py, dz = tz - pz;
                        seg_term(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
                    }
                    px = tx; py = ty; pz = tz;
                }
                const float nx = __shfl_down_sync(FULL, t0x, 1, G);
                const float ny = __shfl_down_sync(FULL, t0y, 1, G);
                const float nz = __shfl_down_sync(FULL, t0z, 1, G);
                if (b0 + SPL <= N - 1) {
                    const float dx = nx - px, dy = ny - py, dz = nz - pz;
                    seg_term(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
                }
                hi = s;
                lo = -cc;
                group_sum_pair<G>(hi, lo);
                float g3[3] = {0.f, 0.f, 0.f};
                if (j == 0)
                    receiver_grad(sx, sy, sz, Lay::addr(gbase, (N - 3) / SPL, (N - 3) % SPL),
                                  Lay::addr(gbase, (N - 2) / SPL, (N - 2) % SPL),
                                  Lay::addr(gbase, (N - 1) / SPL, (N - 1) % SPL), ma.lut, kc, c.inv_ds, g3);
                if (active && !(isnan(hi) || isnan(lo))) {
                    const float wt = exp2f(((hi - ma.ref_log10) + lo) * kLog2_10);
                    acc[0] += wt * gmu * kInvLn10;
                    acc[1] += wt * geps * kInvLn10;
                    acc[2] += wt * g3[0];
                    acc[3] += wt * g3[1];
                    acc[4] += wt * g3[2];
                    if (j == 0) acc[5] += wt;
                }
            } else {
                path_log10<G, SPL, EXACT>(j, N, s_tab, kc, seg_smem, no_bins, hi, lo, clamped);
            }
            if (MODE == kModeExport) {
                // positions x_0 + prefix sums of the segment vectors, in double; every lane
                // takes part in the scan, only active chains write
                double px = 0.0, py = 0.0, pz = 0.0;
                double lx[SPL], ly[SPL], lz[SPL];
#pragma unroll
                for (int m = 0; m < SPL; ++m) {
                    const uint32_t a = Lay::addr(gbase, j, m);
                    const bool in = j * SPL + m < N;
                    px += in ? (double)sx[a] : 0.0;
                    py += in ? (double)sy[a] : 0.0;
                    pz += in ? (double)sz[a] : 0.0;
                    lx[m] = px; ly[m] = py; lz[m] = pz;
                }
                double ex = px, ey = py, ez = pz;   // inclusive scan of lane totals
#pragma unroll
                for (int o = 1; o < G; o <<= 1) {
                    const double ux = __shfl_up_sync(FULL, ex, o, G), uy = __shfl_up_sync(FULL, ey, o, G),
                                 uz = __shfl_up_sync(FULL, ez, o, G);
                    if ((int)j >= o) { ex += ux; ey += uy; ez += uz; }
                }
                ex -= px; ey -= py; ez -= pz;       // exclusive
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
                    if (j == 0)
                        ma.exp_w[pidx] = (isnan(hi) || isnan(lo)) ? NAN : (double)hi + (double)lo + (N - 1) * ma.log10_abs;
                }
            }
            if (!active) continue;
            if (isnan(hi) || isnan(lo)) {
                ++failed;
            } else if (valid == 0) {
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
    clamped = group_sum_u<G>(clamped);
    if (MODE == kModeAdjoint) {
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            float v = acc[i];
#pragma unroll
            for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(FULL, v, o);
            acc[i] = v;
        }
        if (j == 0 && real_chain)
            for (int i = 0; i < 6; ++i) ma.grad[(size_t)chain * 6 + i] = (double)acc[i];
    }
    const double chain_log10 = valid ? (double)lse_m + log10((double)lse_s - (double)lse_c) +
                                       (double)(N - 1) * ma.log10_abs
                                     : -INFINITY;
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

template <int G, int SPL, bool EXACT, int MAXT, int MODE>
__global__ void __launch_bounds__(MAXT, 1) comp_chain_kernel(ChainSpec c, CompConsts kc,
                                                             const float *__restrict__ init_seg,
                                                             const float2 *__restrict__ tab_g,
                                                             ChainOut *__restrict__ out,
                                                             double2 *__restrict__ block_partials, ModeArgs ma)
{
    extern __shared__ float4 smem4[];
    const int bins = kc.bins;
    const float2 *s_tab = reinterpret_cast<const float2 *>(smem4);
    const int tab_f4 = (bins + 1) / 2;  // float2 entries, padded to float4
    float *s_state = reinterpret_cast<float *>(smem4 + tab_f4);
    const int warps = blockDim.x >> 5;
    double *s_res = reinterpret_cast<double *>(s_state + warps * 3 * SPL * 32);
    stage_table(smem4, tab_g, bins);
    __syncthreads();

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q = lane / G, j = lane % G;
    constexpr int CPW = 32 / G;
    const uint32_t chain = (blockIdx.x * warps + warp) * CPW + q;
    float *sx = s_state + warp * 3 * SPL * 32;
    const double cl = chain_body<G, SPL, EXACT, MODE>(c, kc, init_seg, s_tab, sx, sx + SPL * 32, sx + 2 * SPL * 32,
                                                      q * G, j, chain, chain < c.n_chains, out, ma);
    if (j == 0) s_res[warp * CPW + q] = cl;
    __syncthreads();
    // Per-CTA log-sum-exp of the chains, rescaled by the block maximum (FP64).
    if (warp == 0 && block_partials) {
        const int nres = warps * CPW;
        double mx = -INFINITY;
        for (int i = lane; i < nres; i += 32) mx = fmax(mx, s_res[i]);
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, o));
        double sum = 0.0;
        if (mx > -INFINITY)
            for (int i = lane; i < nres; i += 32) sum += (s_res[i] > -INFINITY) ? exp10(s_res[i] - mx) : 0.0;
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
        if (lane == 0) block_partials[blockIdx.x] = make_double2(mx, sum);
    }
}

// Compensated weigher of given paths: one group of 32 lanes per path.
template <int SPL, bool EXACT>
__global__ void __launch_bounds__(256) weigh_comp_kernel(const float *__restrict__ pos, uint64_t n_paths, uint32_t N,
                                                          CompConsts kc, const float2 *__restrict__ tab,
                                                          double log10_absorption, double *__restrict__ log10w,
                                                          uint8_t *__restrict__ valid, int32_t *__restrict__ bins)
{
    const uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t j = threadIdx.x & 31;
    if (p >= n_paths) return;  // whole warps exit together
    const float *pp = pos + p * 3 * (uint64_t)(N + 1);
    auto seg = [&](int m, float &x, float &y, float &z) {
        const uint32_t s = j * SPL + m;
        if (s < N) {
            x = pp[3 * s + 3] - pp[3 * s];
            y = pp[3 * s + 4] - pp[3 * s + 1];
            z = pp[3 * s + 5] - pp[3 * s + 2];
        } else {
            x = y = z = 0.f;
        }
    };
    int32_t *brow = bins ? bins + p * (N - 1) : nullptr;
    auto sink = [&](uint32_t i, int32_t b) {
        if (brow) brow[i] = b;
    };
    uint32_t clamped = 0;
    float hi, lo;
    path_log10<32, SPL, EXACT>(j, N, tab, kc, seg, sink, hi, lo, clamped);
    if (j == 0) {
        const bool ok = !(isnan(hi) || isnan(lo));
        log10w[p] = ok ? (double)hi + (double)lo + (double)(N - 1) * log10_absorption : 0.0;
        if (valid) valid[p] = ok ? 1 : 0;
    }
}

template <int G, int SPL, bool EXACT, int MODE>
cudaError_t launch_t(const ChainSpec &c, const CompConsts &kc, int warps, const float *init_seg, const float2 *tab,
                     ChainOut *out, double2 *partials, const ModeArgs &ma, size_t smem, uint32_t blocks, cudaStream_t st)
{
    constexpr int MAXT = (SPL >= 16) ? 512 : 1024;
    if (warps * 32 > MAXT) return cudaErrorInvalidConfiguration;
    auto kern = comp_chain_kernel<G, SPL, EXACT, MAXT, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<blocks, warps * 32, smem, st>>>(c, kc, init_seg, tab, out, partials, ma);
    return cudaGetLastError();
}

template <int G, int SPL>
cudaError_t launch_g(int mode, const ChainSpec &c, const CompConsts &kc, const CompTuning &t, const float *init_seg,
                     const float2 *tab, ChainOut *out, double2 *partials, const ModeArgs &ma, size_t smem,
                     uint32_t blocks, cudaStream_t st)
{
    const int w = t.warps_per_block;
    if (mode == kModeAdjoint)
        return launch_t<G, SPL, true, kModeAdjoint>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st);
    if (mode == kModeExport) {
        if (t.exact_blend) return launch_t<G, SPL, true, kModeExport>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st);
        return launch_t<G, SPL, false, kModeExport>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st);
    }
    if (t.exact_blend) return launch_t<G, SPL, true, kModeForward>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st);
    return launch_t<G, SPL, false, kModeForward>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st);
}

CompConsts make_consts(float inv_ds, const LutMetaF &m)
{
    CompConsts k;
    k.kscale = inv_ds / m.step;
    k.roff = -m.min_k / m.step;
    k.rmax = (m.max_k - m.min_k) / m.step;
    k.rsnap = 1e-3f / m.step;
    k.step = m.step;
    k.bins = m.bins;
    return k;
}

}  // namespace

CompTuning comp_default_tuning(uint32_t n)
{
    CompTuning t;
    t.exact_blend = 0;
    if (n <= 16) { t.group = 8; t.spl = 2; t.warps_per_block = 32; }
    else if (n <= 32) { t.group = 8; t.spl = 4; t.warps_per_block = 32; }
    else if (n <= 64) { t.group = 8; t.spl = 8; t.warps_per_block = 32; }
    else if (n <= 128) { t.group = 16; t.spl = 8; t.warps_per_block = 32; }
    else if (n <= 256) { t.group = 32; t.spl = 8; t.warps_per_block = 32; }
    else if (n <= 512) { t.group = 32; t.spl = 16; t.warps_per_block = 16; }
    else { t.group = 32; t.spl = 32; t.warps_per_block = 8; }
    return t;
}

bool comp_tuning_supported(const CompTuning &t, uint32_t n, uint32_t k_eff)
{
    const bool shape = (t.group == 8 && (t.spl == 2 || t.spl == 4 || t.spl == 8 || t.spl == 16)) ||
                       (t.group == 16 && (t.spl == 4 || t.spl == 8 || t.spl == 16)) ||
                       (t.group == 32 && (t.spl == 4 || t.spl == 8 || t.spl == 16 || t.spl == 32));
    return shape && (uint32_t)(t.group * t.spl) >= n && n >= 4 && k_eff <= (uint32_t)kMaxSubChain &&
           t.warps_per_block >= 1 && t.warps_per_block * 32 <= ((t.spl >= 16) ? 512 : 1024);
}

uint32_t comp_default_chains(uint32_t n, int sm_count)
{
    const CompTuning t = comp_default_tuning(n);
    return (uint32_t)sm_count * t.warps_per_block * (32 / t.group);
}

size_t comp_smem_bytes(const CompTuning &t, uint32_t bins)
{
    const size_t tab = (size_t)((bins + 1) / 2) * sizeof(float4);
    const size_t state = (size_t)t.warps_per_block * 3 * t.spl * 32 * sizeof(float);
    const size_t res = (size_t)t.warps_per_block * (32 / t.group) * sizeof(double);
    return tab + state + res;
}

uint32_t comp_blocks(const ChainSpec &c, const CompTuning &t)
{
    const uint32_t per_block = t.warps_per_block * (32 / t.group);
    return (c.n_chains + per_block - 1) / per_block;
}

namespace {
cudaError_t launch_mode(int mode, const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *logtab,
                        const float2 *lintab, LutMetaF m, ChainOut *out, double2 *block_partials, const ModeArgs &ma,
                        cudaStream_t st)
{
    if (!comp_tuning_supported(t, c.n_segments, c.k_eff)) return cudaErrorInvalidValue;
    if (c.n_chains == 0) return cudaSuccess;
    const CompConsts kc = make_consts(c.inv_ds, m);
    const size_t smem = comp_smem_bytes(t, (uint32_t)m.bins);
    const uint32_t blocks = comp_blocks(c, t);
    const float2 *tab = (t.exact_blend || mode == kModeAdjoint) ? lintab : logtab;
#define TWISTY_CASE(GG, SS) \
    if (t.group == GG && t.spl == SS) return launch_g<GG, SS>(mode, c, kc, t, init_seg, tab, out, block_partials, ma, smem, blocks, st);
    TWISTY_CASE(8, 2)
    TWISTY_CASE(8, 4)
    TWISTY_CASE(8, 8)
    TWISTY_CASE(8, 16)
    TWISTY_CASE(16, 4)
    TWISTY_CASE(16, 8)
    TWISTY_CASE(16, 16)
    TWISTY_CASE(32, 4)
    TWISTY_CASE(32, 8)
    TWISTY_CASE(32, 16)
    TWISTY_CASE(32, 32)
#undef TWISTY_CASE
    return cudaErrorInvalidValue;
}

__global__ void __launch_bounds__(1024) grad_reduce_kernel(const double *__restrict__ g, uint32_t n, double *__restrict__ out)
{
    __shared__ double red[6][32];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        for (int k = 0; k < 6; ++k) a[k] += g[(size_t)i * 6 + k];
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(FULL, a[k], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < 6; ++k) red[k][w] = a[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[threadIdx.x][i];
        out[threadIdx.x] = v;
    }
}
}  // namespace

cudaError_t launch_comp_chains(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *logtab,
                               const float2 *lintab, LutMetaF m, ChainOut *out, double2 *block_partials,
                               cudaStream_t st)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    return launch_mode(kModeForward, c, t, init_seg, logtab, lintab, m, out, block_partials, ma, st);
}

cudaError_t launch_comp_export(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *logtab,
                               const float2 *lintab, LutMetaF m, const float x0[3], float *exp_pos, double *exp_w,
                               ChainOut *out, cudaStream_t st)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    ma.exp_pos = exp_pos;
    ma.exp_w = exp_w;
    ma.x0[0] = x0[0];
    ma.x0[1] = x0[1];
    ma.x0[2] = x0[2];
    return launch_mode(kModeExport, c, t, init_seg, logtab, lintab, m, out, nullptr, ma, st);
}

cudaError_t launch_comp_adjoint(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *lintab,
                                LutMetaF m, const float *lut, const float *dmu, const float *deps, float ref_log10,
                                double *grad_chains, double *grad_out, cudaStream_t st)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    ma.lut = lut;
    ma.dmu = dmu;
    ma.deps = deps;
    ma.ref_log10 = ref_log10;
    ma.grad = grad_chains;
    cudaError_t e = launch_mode(kModeAdjoint, c, t, init_seg, lintab, lintab, m, nullptr, nullptr, ma, st);
    if (e != cudaSuccess) return e;
    grad_reduce_kernel<<<1, 1024, 0, st>>>(grad_chains, c.n_chains, grad_out);
    return cudaGetLastError();
}

cudaError_t launch_weigh_comp(const float *pos, uint64_t n_paths, uint32_t n_segments, float inv_ds,
                              const float2 *logtab, const float2 *lintab, int exact_blend, LutMetaF m,
                              double log10_absorption, double *log10w, uint8_t *valid, int32_t *bins, cudaStream_t st)
{
    if (n_paths == 0) return cudaSuccess;
    const CompConsts kc = make_consts(inv_ds, m);
    const uint64_t blocks = (n_paths * 32 + 255) / 256;
    const float2 *tab = exact_blend ? lintab : logtab;
#define TWISTY_W(SS)                                                                                           \
    if (n_segments <= 32u * SS) {                                                                              \
        if (exact_blend)                                                                                       \
            weigh_comp_kernel<SS, true><<<(unsigned)blocks, 256, 0, st>>>(pos, n_paths, n_segments, kc, tab,  \
                                                                          log10_absorption, log10w, valid, bins); \
        else                                                                                                   \
            weigh_comp_kernel<SS, false><<<(unsigned)blocks, 256, 0, st>>>(pos, n_paths, n_segments, kc, tab, \
                                                                           log10_absorption, log10w, valid, bins); \
        return cudaGetLastError();                                                                             \
    }
    TWISTY_W(1)
    TWISTY_W(2)
    TWISTY_W(4)
    TWISTY_W(8)
    TWISTY_W(16)
    TWISTY_W(32)
#undef TWISTY_W
    return cudaErrorInvalidValue;
}

}  // namespace twisty
