// chain_comp.cu -- single-run entry points of the compensated form: the weigher of given
// paths, the launchers and the kernel-shape table. The chain kernel (comp_launch.cuh, body in
// comp_body.cuh) is instantiated per shape in comp_shapes_{a..i}.cu, compiled in parallel.
#include "comp_launch.cuh"

namespace twisty {
namespace {

// Compensated weigher of given paths: one group of 32 lanes per path; tangents from the
// positions, normalised here.
template <int SPL, bool EXACT>
__global__ void __launch_bounds__(256) weigh_comp_kernel(const float *__restrict__ pos, uint64_t n_paths, uint32_t N,
                                                          CompConsts kc, const float2 *__restrict__ tab,
                                                          const float2 *__restrict__ lin,
                                                          double log10_absorption, double *__restrict__ log10w,
                                                          uint8_t *__restrict__ valid, int32_t *__restrict__ bins)
{
    const uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t j = threadIdx.x & 31;
    if (p >= n_paths) return;  // whole warps exit together
    const float *pp = pos + p * 3 * (uint64_t)(N + 1);
    auto tan = [&](int m, float &x, float &y, float &z) {
        const uint32_t s = j * SPL + m;
        if (s < N) {
            x = pp[3 * s + 3] - pp[3 * s];
            y = pp[3 * s + 4] - pp[3 * s + 1];
            z = pp[3 * s + 5] - pp[3 * s + 2];
            const float r = rsqrtf(fmaf(x, x, fmaf(y, y, z * z))) * kc.kscale;   // tangents at length kscale
            x *= r; y *= r; z *= r;
        } else {
            x = y = z = 0.f;
        }
    };
    int32_t *brow = bins ? bins + p * (N - 1) : nullptr;
    auto sink = [&](uint32_t i, int32_t b) {
        if (brow) brow[i] = b;
    };
    uint32_t clamped = 0;
    double w = path_log10<32, SPL, EXACT, true, true>(j, N, tab, kc, tan, ShflNext<32>{}, sink, clamped);
    if (!EXACT && isnan(w)) {
        // a steep bin (NaN slope) or a NaN curvature: the exact blend through the linear table
        w = path_log10<32, SPL, true, true, true>(j, N, lin, kc, tan, ShflNext<32>{}, sink, clamped);
    }
    if (j == 0) {
        const bool ok = !isnan(w);
        log10w[p] = ok ? w + (double)(N - 1) * log10_absorption : 0.0;
        if (valid) valid[p] = ok ? 1 : 0;
    }
}

cudaError_t launch_mode(int mode, const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *fixtab,
                        const float2 *lintab, LutMetaF m, ChainOut *out, double2 *block_partials, const ModeArgs &ma,
                        const LogFixed &lf, cudaStream_t st)
{
    if (!comp_tuning_supported(t, c.n_segments, c.k_eff)) return cudaErrorInvalidValue;
    if (c.has_eval_shift && mode != kModeForward) return cudaErrorInvalidValue;
    if (c.n_chains == 0) return cudaSuccess;
    const bool shift = c.has_eval_shift != 0;
    const bool exact = t.exact_blend || mode == kModeAdjoint || lf.inv_scale == 0.0 || shift;
    const CompConsts kc = make_consts(c.inv_ds, m, c.n_segments, lf);
    const size_t smem = comp_smem_bytes(t, (uint32_t)m.bins);
    const uint32_t blocks = comp_blocks(c, t);
    const float2 *tab = exact ? lintab : fixtab;
    const bool clamp = table_needs_clamp(kc);
    const bool steep = !exact && lf.steep > 0;
    ModeArgs mb = ma;
    mb.lin = lintab;
    const CompLaunch a{mode, exact, clamp, shift, steep, c, kc, t, init_seg, tab, out, block_partials, mb, smem, blocks, st};
    cudaError_t e = cudaSuccess;
    if (launch_comp_shapes_a(a, e) || launch_comp_shapes_b(a, e) || launch_comp_shapes_c(a, e) ||
        launch_comp_shapes_d(a, e) || launch_comp_shapes_e(a, e) || launch_comp_shapes_f(a, e) ||
        launch_comp_shapes_g(a, e) || launch_comp_shapes_h(a, e) ||
        launch_comp_shapes_i(a, e))
        return e;
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

// One CTA per range of chains: the sums of their 6 gradient entries (the batched adjoint).
__global__ void __launch_bounds__(256) grad_reduce_segments_kernel(const double *__restrict__ g,
                                                                   const uint2 *__restrict__ ranges,
                                                                   double *__restrict__ out)
{
    __shared__ double red[6][8];
    const uint2 r = ranges[blockIdx.x];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t i = threadIdx.x; i < r.y; i += blockDim.x)
        for (int k = 0; k < 6; ++k) a[k] += g[(size_t)(r.x + i) * 6 + k];
    for (int k = 0; k < 6; ++k)
        for (int o = 16; o > 0; o >>= 1) a[k] += __shfl_xor_sync(FULL, a[k], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < 6; ++k) red[k][w] = a[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v += red[threadIdx.x][i];
        out[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// Derivative tables in the linear table's form: per bin (dmu_i, dmu_{i+1} - dmu_i, deps_i,
// deps_{i+1} - deps_i), the last bin's changes 0; tables of `bins` entries back to back.
__global__ void deriv_table_kernel(const double *__restrict__ dmu, const double *__restrict__ deps, uint32_t bins,
                                   size_t n, float4 *__restrict__ out)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const bool last = (i % bins) == bins - 1;
        const float m0 = (float)dmu[i], e0 = (float)deps[i];
        const float m1 = last ? m0 : (float)dmu[i + 1], e1 = last ? e0 : (float)deps[i + 1];
        out[i] = make_float4(m0, m1 - m0, e0, e1 - e0);
    }
}

}  // namespace

cudaError_t launch_grad_reduce_segments(const double *grad_chains, const uint2 *ranges, uint32_t n, double *out,
                                        cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    grad_reduce_segments_kernel<<<n, 256, 0, st>>>(grad_chains, ranges, out);
    return cudaGetLastError();
}

cudaError_t launch_deriv_tables(const double *dmu, const double *deps, uint32_t bins, uint32_t n_tables, float4 *out,
                                cudaStream_t st)
{
    const size_t n = (size_t)bins * n_tables;
    if (n == 0) return cudaSuccess;
    const size_t blocks = std::min<size_t>((n + 255) / 256, 148 * 16);
    deriv_table_kernel<<<(unsigned)blocks, 256, 0, st>>>(dmu, deps, bins, n, out);
    return cudaGetLastError();
}


bool comp_table_needs_clamp(float inv_ds, const LutMetaF &m)
{
    return table_needs_clamp(make_consts(inv_ds, m, 2, LogFixed{0.0, 0.0, 0, 0}));
}

// Shapes measured fastest on B200 by twisty_autotune (4096-bin tables, k <= 32): 16 segments
// per lane keep 16 independent table loads in flight per lane, which outweighs the halved
// warp count above N = 64. The 12- and 24-segment shapes cover the N between powers of two
// with less padding (measured: N = 192, 384, 768 18-27 % faster than the next power of two).
// Fewer lanes per chain with more segments each (8 x {20, 24}, 16 x {20, 24, 28}) put two or
// four chains in a warp and measured 13-32 % faster than the 16- and 32-lane shapes padded to
// the same N (N = 160, 192, 320, 384, 448), 4 x 20 11 % above 8 x 12 at N = 80 (4 x 24, 4 x 28
// within 1 % of 8 x 12 / 8 x 16 at N = 96, 112; 4 x 32 below 8 x 16 at 128); 16 x 32 at N = 512
// measured only 2 % above 32 x 16
// and would drop to 12 warps through L1 for large tables, so 32 x 16 stays. The 24-segment
// shapes run 24 warps, which leave no room to stage a table: they stage one at 20 warps when
// that fits (comp_stage_min_warps) and gather it through L1 at 24 otherwise; the 20-segment
// shapes do the same with tables too large to stage at 24 warps; 16 x 28 stages at 16 and
// gathers at 20. 32 x 32 stays at 12 warps: 16 warps through L1 measured even
// with it at N = 1024.
// Up to N = 32, 4-lane groups put 8 chains in a warp, which share the per-step work of the
// proposal broadcast, the group reductions and the log-sum-exp (N = 16: +23 %, 32: +12 %
// over 8 lanes); up to N = 12 one lane carries a whole chain, 32 chains per warp, with no group
// reductions at all (N = 5: +76 %, 8: +54 %, 10: +9 % over 4 lanes). The shapes with one
// segment per lane more than a power of two (3, 5, 9, 17)
// serve N = 2^k + 2, the N of the reference's own configurations (10, 18, 34, 66, 130, 258,
// 514), which would otherwise pad to the next power of two.
// Since short chains turn the shorter side of each move (comp_body), one lane per chain
// also wins at N = 13..24 on long passes: 1 x 16 (N = 13..16) and 1 x 24 (17..24) at 16 warps
// measured +35-42 % and +15-19 % over 4 x {4, 5, 8} on passes of 2^32 path-segments. They run
// twice as many chains, each of which pays the burn-in, at 0.72 (1 x 16) and 0.81 (1 x 24) of
// the cost per weighted step (both fitted to those runs), so they win once a pass's paths reach
// about 58000 and 125000 times its burn-in steps per chain; the thresholds below round those up.
// (At 2^24 paths and 256 burn-in steps: 1 x 16 +5 % at N = 16, 1 x 24 4-10 % slower.)
// With unpadded one-lane rows (comp_pitch_xy), 1 x 16 at 24 warps carries 1.5x the chains of
// 16 warps at 0.883 of the cost per step: +9.6 % at N = 16 on passes of 2^32 path-segments,
// +4 % at 2^26 paths, 7 % slower at 2^24; it takes over at paths >= 210000 x burn-in.
// 4 x 12, which also turns the shorter side, serves N = 37..48 with less padding than 4 x 16:
// +16-19 % at N = 37, 40 and +8-13 % at 44, 48, on passes of 2^24 paths and of 2^32
// path-segments alike (+3-8 % without the shorter side). The batched kernels have neither
// one-lane shape nor 4 x 12.
CompTuning comp_default_tuning(uint32_t n, bool batched, uint64_t paths, uint64_t burn_in)
{
    CompTuning t;
    t.exact_blend = 0;
    const bool lane16 = !batched && paths / 60000u >= burn_in;
    const bool lane16_24w = !batched && paths / 210000u >= burn_in;
    const bool lane24 = !batched && paths / 130000u >= burn_in;
    if (n <= 8) { t.group = 1; t.spl = 8; t.warps_per_block = 32; }
    else if (n <= 12) { t.group = 1; t.spl = 12; t.warps_per_block = 24; }
    else if (n <= 16 && lane16_24w) { t.group = 1; t.spl = 16; t.warps_per_block = 24; }
    else if (n <= 16 && lane16) { t.group = 1; t.spl = 16; t.warps_per_block = 16; }
    else if (n <= 16) { t.group = 4; t.spl = 4; t.warps_per_block = 32; }
    else if (n <= 24 && lane24) { t.group = 1; t.spl = 24; t.warps_per_block = 16; }
    else if (n <= 20) { t.group = 4; t.spl = 5; t.warps_per_block = 32; }
    else if (n <= 32) { t.group = 4; t.spl = 8; t.warps_per_block = 32; }
    else if (n <= 36) { t.group = 4; t.spl = 9; t.warps_per_block = 32; }
    else if (n <= 48 && !batched) { t.group = 4; t.spl = 12; t.warps_per_block = 24; }
    else if (n <= 64) { t.group = 4; t.spl = 16; t.warps_per_block = 24; }
    else if (n <= 68) { t.group = 4; t.spl = 17; t.warps_per_block = 24; }
    else if (n <= 72) { t.group = 8; t.spl = 9; t.warps_per_block = 32; }
    else if (n <= 80) { t.group = 4; t.spl = 20; t.warps_per_block = 24; }
    else if (n <= 96) { t.group = 8; t.spl = 12; t.warps_per_block = 24; }
    else if (n <= 128) { t.group = 8; t.spl = 16; t.warps_per_block = 24; }
    else if (n <= 136) { t.group = 8; t.spl = 17; t.warps_per_block = 24; }
    else if (n <= 160) { t.group = 8; t.spl = 20; t.warps_per_block = 24; }
    else if (n <= 192) { t.group = 8; t.spl = 24; t.warps_per_block = 24; }
    else if (n <= 256) { t.group = 16; t.spl = 16; t.warps_per_block = 24; }
    else if (n <= 272) { t.group = 16; t.spl = 17; t.warps_per_block = 24; }
    else if (n <= 320) { t.group = 16; t.spl = 20; t.warps_per_block = 24; }
    else if (n <= 384) { t.group = 16; t.spl = 24; t.warps_per_block = 24; }
    else if (n <= 448) { t.group = 16; t.spl = 28; t.warps_per_block = 20; }
    else if (n <= 512) { t.group = 32; t.spl = 16; t.warps_per_block = 24; }
    else if (n <= 544) { t.group = 32; t.spl = 17; t.warps_per_block = 24; }
    else if (n <= 640) { t.group = 32; t.spl = 20; t.warps_per_block = 24; }
    else if (n <= 768) { t.group = 32; t.spl = 24; t.warps_per_block = 24; }
    else if (n <= 896) { t.group = 32; t.spl = 28; t.warps_per_block = 16; }
    else { t.group = 32; t.spl = 32; t.warps_per_block = 12; }
    return t;
}

// The fewest warps per CTA at which staging the table in shared memory is kept over gathering
// it through L1 at the shape's full warps. The 24-segment shapes at 24 warps have no room for a
// table; at 20 warps a staged table measured above L1 at 24 (32 x 24: 1-5 % at N = 640, 768;
// 16 x 24: 3 % at N = 384; 8 x 24: 4 % at N = 192, 4096 bins) and L1 at 24 3-13 % above 16
// staged warps (32 x 24, N = 600-768, 4096 to 20000 bins). The 20-segment shapes at 24 warps
// stage tables of up to ~4096 bins; an 8192-bin table staged at 20 warps measured above L1 at 24
// (8 x 20: 3.0 % at N = 144, 3.9 % at 160; 16 x 20: 1.3 % at 320, 0.1 % at 300; 32 x 20: 0.7 %
// at 640, 0.0 % at 600; 4 x 20: 0.4 % at 80; passes of 2^32 path-segments). 16 x 28 staged at
// 16 warps measured 5 % above L1 at 20 (N = 448). Other shapes stage only at full warps.
int comp_stage_min_warps(const CompTuning &t)
{
    if ((t.spl == 24 || t.spl == 20) && t.warps_per_block == 24) return 20;
    if (t.group == 16 && t.spl == 28 && t.warps_per_block == 20) return 16;
    return t.warps_per_block;
}

bool comp_tuning_supported(const CompTuning &t, uint32_t n, uint32_t k_eff)
{
    const int s = t.spl;
    const bool shape = (t.group == 1 && (s == 8 || s == 12 || s == 16 || s == 24)) ||
                       (t.group == 4 && (s == 2 || s == 3 || s == 4 || s == 5 || s == 8 || s == 9 || s == 12 || s == 16 ||
                                         s == 17 || s == 20 || s == 24 || s == 28 || s == 32)) ||
                       (t.group == 8 && (s == 2 || s == 4 || s == 8 || s == 9 || s == 12 || s == 16 || s == 17 || s == 20 ||
                                         s == 24 || s == 32)) ||
                       (t.group == 16 && (s == 4 || s == 8 || s == 12 || s == 16 || s == 17 || s == 20 || s == 24 ||
                                          s == 28 || s == 32)) ||
                       (t.group == 32 && (s == 4 || s == 8 || s == 12 || s == 16 || s == 17 || s == 20 || s == 24 ||
                                          s == 28 || s == 32));
    return shape && (uint32_t)(t.group * t.spl) >= n && n >= 4 && k_eff <= (uint32_t)kMaxSubChain &&
           t.warps_per_block >= 1 && t.warps_per_block * 32 <= comp_max_threads(t.group, t.spl);
}

size_t comp_smem_bytes(const CompTuning &t, uint32_t bins)
{
    const size_t tab = t.lut_global ? 0 : (size_t)((bins + 1) / 2) * sizeof(float4);
    const size_t state = (size_t)t.warps_per_block * warp_state_bytes(t.group, t.spl) + cta_len_bytes(t.group, t.spl);
    const size_t res = (size_t)t.warps_per_block * (32 / t.group) * sizeof(double);
    return tab + state + res;
}

bool comp_fit_smem(CompTuning &t, uint32_t bins, bool may_shrink)
{
    while (may_shrink && t.warps_per_block > 4 && comp_smem_bytes(t, bins) > kCompSmemCap) t.warps_per_block -= 4;
    return comp_smem_bytes(t, bins) <= kCompSmemCap;
}

// Measured on B200: L1 at full occupancy 0-9 % below a staged table at full occupancy, and from
// even with one at 5/6 of the warps to +14 % at 2/3 and +40 % and more at 1/4 to 1/2.
bool comp_table_through_l1(const CompTuning &t, uint32_t bins, bool may_shrink)
{
    CompTuning staged = t;
    staged.lut_global = 0;
    const bool fits = comp_fit_smem(staged, bins, may_shrink);
    return !fits || staged.warps_per_block < comp_stage_min_warps(t);
}

uint32_t comp_blocks(const ChainSpec &c, const CompTuning &t)
{
    const uint32_t per_block = t.warps_per_block * (32 / t.group);
    return (c.n_chains + per_block - 1) / per_block;
}

cudaError_t launch_comp_chains(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *fixtab,
                               const float2 *lintab, LutMetaF m, ChainOut *out, double2 *block_partials,
                               cudaStream_t st, LogFixed lf)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    return launch_mode(kModeForward, c, t, init_seg, fixtab, lintab, m, out, block_partials, ma, lf, st);
}

cudaError_t launch_comp_export(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *fixtab,
                               const float2 *lintab, LutMetaF m, const float x0[3], float *exp_pos, double *exp_w,
                               ChainOut *out, cudaStream_t st, LogFixed lf)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    ma.exp_pos = exp_pos;
    ma.exp_w = exp_w;
    ma.x0[0] = x0[0];
    ma.x0[1] = x0[1];
    ma.x0[2] = x0[2];
    return launch_mode(kModeExport, c, t, init_seg, fixtab, lintab, m, out, nullptr, ma, lf, st);
}

cudaError_t launch_comp_adjoint(const ChainSpec &c, const CompTuning &t, const float *init_seg, const float2 *lintab,
                                LutMetaF m, const float4 *dtab, float ref_log10, double *grad_chains, double *grad_out,
                                cudaStream_t st)
{
    ModeArgs ma{};
    ma.log10_abs = log10(c.absorption_factor);
    ma.dtab = dtab;
    ma.ref_log10 = ref_log10;
    ma.grad = grad_chains;
    cudaError_t e = launch_mode(kModeAdjoint, c, t, init_seg, lintab, lintab, m, nullptr, nullptr, ma,
                                LogFixed{0.0, 0.0}, st);
    if (e != cudaSuccess) return e;
    grad_reduce_kernel<<<1, 1024, 0, st>>>(grad_chains, c.n_chains, grad_out);
    return cudaGetLastError();
}

cudaError_t launch_weigh_comp(const float *pos, uint64_t n_paths, uint32_t n_segments, float inv_ds,
                              const float2 *fixtab, const float2 *lintab, int exact_blend, LutMetaF m,
                              double log10_absorption, double *log10w, uint8_t *valid, int32_t *bins, cudaStream_t st,
                              LogFixed lf)
{
    if (n_paths == 0) return cudaSuccess;
    const CompConsts kc = make_consts(inv_ds, m, n_segments, lf);
    const uint64_t blocks = (n_paths * 32 + 255) / 256;
    const bool exact = exact_blend || lf.inv_scale == 0.0;
    const float2 *tab = exact ? lintab : fixtab;
#define TWISTY_W(SS)                                                                                           \
    if (n_segments <= 32u * SS) {                                                                              \
        if (exact)                                                                                             \
            weigh_comp_kernel<SS, true><<<(unsigned)blocks, 256, 0, st>>>(pos, n_paths, n_segments, kc, tab,  \
                                                                          lintab, log10_absorption, log10w, valid, \
                                                                          bins);                                  \
        else                                                                                                   \
            weigh_comp_kernel<SS, false><<<(unsigned)blocks, 256, 0, st>>>(pos, n_paths, n_segments, kc, tab, \
                                                                           lintab, log10_absorption, log10w,     \
                                                                           valid, bins);                          \
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
