// comp_launch.cuh -- the compensated chain kernel and its per-shape launcher, included by the
// translation units that instantiate it (comp_shapes_{a..i}.cu, a few shapes each, so that the
// many template variants compile in parallel) and by chain_comp.cu, which dispatches to them.
#pragma once
#include "comp_body.cuh"

namespace twisty {

// One launch of the chain kernel, as chain_comp.cu's launch_mode resolved it.
struct CompLaunch {
    int mode;
    bool exact, clamp, shift, steep;
    ChainSpec c;
    CompConsts kc;
    CompTuning t;
    const float *init_seg;
    const float2 *tab;
    ChainOut *out;
    double2 *partials;
    ModeArgs ma;
    size_t smem;
    uint32_t blocks;
    cudaStream_t st;
};

// Each returns false when the launch's shape is not among its own, else launches and sets e.
bool launch_comp_shapes_a(const CompLaunch &a, cudaError_t &e);   // 1 x {8, 12}, 4 x {2..17}, 8 x {2, 4}
bool launch_comp_shapes_b(const CompLaunch &a, cudaError_t &e);   // 8 x {8, 9, 12, 16, 17, 32}
bool launch_comp_shapes_c(const CompLaunch &a, cudaError_t &e);   // 16 x {4, 8, 12, 16, 17}
bool launch_comp_shapes_d(const CompLaunch &a, cudaError_t &e);   // 32 x {4, 8, 12, 17}
bool launch_comp_shapes_e(const CompLaunch &a, cudaError_t &e);   // 32 x {16, 24, 32}
bool launch_comp_shapes_f(const CompLaunch &a, cudaError_t &e);   // 16 x 20, 32 x {20, 28}
bool launch_comp_shapes_g(const CompLaunch &a, cudaError_t &e);   // 8 x {20, 24}, 16 x {24, 28, 32}
bool launch_comp_shapes_h(const CompLaunch &a, cudaError_t &e);   // 4 x {20, 24, 28, 32}
bool launch_comp_shapes_i(const CompLaunch &a, cudaError_t &e);   // 1 x {16, 24}, 4 x 12

namespace {

// LUTG: the table is gathered from global memory through L1 (tables too large to stage next to
// the chain state); otherwise each CTA stages it in shared memory first.
template <int G, int SPL, bool EXACT, bool CLAMP, bool SHIFT, int MAXT, int MODE, bool INCR, bool STEEP, bool LUTG>
__global__ void __launch_bounds__(MAXT, 1) comp_chain_kernel(ChainSpec c, CompConsts kc,
                                                             const float *__restrict__ init_seg,
                                                             const float2 *__restrict__ tab_g,
                                                             ChainOut *__restrict__ out,
                                                             double2 *__restrict__ block_partials, ModeArgs ma)
{
    extern __shared__ float4 smem4[];
    const int bins = kc.bins;
    const float2 *s_tab = LUTG ? tab_g : reinterpret_cast<const float2 *>(smem4);
    const int tab_f4 = LUTG ? 0 : (bins + 1) / 2;  // float2 entries, padded to float4
    unsigned char *s_state = reinterpret_cast<unsigned char *>(smem4 + tab_f4);
    const int warps = blockDim.x >> 5;
    using Lay = Layout<G, SPL>;
    float *s_len = reinterpret_cast<float *>(s_state + (size_t)warps * Lay::WARP_BYTES);
    double *s_res = reinterpret_cast<double *>(s_state + (size_t)warps * Lay::WARP_BYTES + cta_len_bytes(G, SPL));
    if (!LUTG) stage_table(smem4, tab_g, bins);
    fill_lengths(s_len, init_seg, c.n_segments, G * SPL);
    __syncthreads();

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q = lane / G, j = lane % G;
    constexpr int CPW = 32 / G;
    const uint32_t chain = (blockIdx.x * warps + warp) * CPW + q;
    unsigned char *wb = s_state + (size_t)warp * Lay::WARP_BYTES;
    const Planes pl{reinterpret_cast<float2 *>(wb), reinterpret_cast<float *>(wb + Lay::XY_BYTES), s_len};
    const double cl = chain_body<G, SPL, EXACT, CLAMP, SHIFT, MODE, INCR, STEEP, LUTG>(c, kc, init_seg, s_tab, pl, q * G,
                                                                                       j, chain, chain < c.n_chains, out,
                                                                                       ma);
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

// ------------------------------------------------------------------------------ launchers
template <int G, int SPL, bool EXACT, bool CLAMP, bool SHIFT, int MODE, bool INCR = false, bool STEEP = false,
          bool LUTG = false>
cudaError_t launch_t(const ChainSpec &c, const CompConsts &kc, int warps, const float *init_seg, const float2 *tab,
                     ChainOut *out, double2 *partials, const ModeArgs &ma, size_t smem, uint32_t blocks, cudaStream_t st)
{
    constexpr int MAXT = comp_max_threads(G, SPL);
    if (warps * 32 > MAXT) return cudaErrorInvalidConfiguration;
    auto kern = comp_chain_kernel<G, SPL, EXACT, CLAMP, SHIFT, MAXT, MODE, INCR, STEEP, LUTG>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (LUTG) {
        // the table is gathered through L1: ask for no more shared memory than the one CTA per SM
        // needs (plus the 1 KB the system reserves per CTA), leaving the rest of the SM's 256 KB
        // of L1/shared storage to L1
        const int pct = (int)std::min<size_t>(100, ((smem + 1024) * 100 + 228 * 1024 - 1) / (228 * 1024));
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
        if (e != cudaSuccess) return e;
    }
    kern<<<blocks, warps * 32, smem, st>>>(c, kc, init_seg, tab, out, partials, ma);
    return cudaGetLastError();
}

// Instantiated variants: forward (fixed/exact x clamp/no clamp, plus an exact+clamp+shift
// variant for receiver-shifted evaluation), export (fixed/exact with clamp), adjoint (exact);
// the fixed-point forward, incremental and export variants again with the steep-bin fallback;
// with the table in global memory (lut_global), the forward variants only.
template <int G, int SPL>
cudaError_t launch_g(int mode, bool exact, bool clamp, bool shift, bool steep, const ChainSpec &c,
                     const CompConsts &kc, const CompTuning &t, const float *init_seg, const float2 *tab,
                     ChainOut *out, double2 *partials, const ModeArgs &ma, size_t smem, uint32_t blocks,
                     cudaStream_t st)
{
    const int w = t.warps_per_block;
    if (t.lut_global) {
        // table through L1: forward passes (fixed point with or without steep bins, exact blend)
        if (mode != kModeForward || shift || c.incr_resync > 1) return cudaErrorInvalidConfiguration;
#define TWISTY_G(E, CL, SP) \
    launch_t<G, SPL, E, CL, false, kModeForward, false, SP, true>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st)
        if (exact) return clamp ? TWISTY_G(true, true, false) : TWISTY_G(true, false, false);
        if (steep) return clamp ? TWISTY_G(false, true, true) : TWISTY_G(false, false, true);
        return clamp ? TWISTY_G(false, true, false) : TWISTY_G(false, false, false);
#undef TWISTY_G
    }
#define TWISTY_L(E, CL, SH, MO) launch_t<G, SPL, E, CL, SH, MO>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st)
#define TWISTY_S(CL, MO, IN) \
    launch_t<G, SPL, false, CL, false, MO, IN, true>(c, kc, w, init_seg, tab, out, partials, ma, smem, blocks, st)
    if (mode == kModeAdjoint) return TWISTY_L(true, true, false, kModeAdjoint);
    if (mode == kModeExport) {
        if (exact) return TWISTY_L(true, true, false, kModeExport);
        return steep ? TWISTY_S(true, kModeExport, false) : TWISTY_L(false, true, false, kModeExport);
    }
    if (shift) return TWISTY_L(true, true, true, kModeForward);
    if (exact) return clamp ? TWISTY_L(true, true, false, kModeForward) : TWISTY_L(true, false, false, kModeForward);
    if (clamp) return steep ? TWISTY_S(true, kModeForward, false) : TWISTY_L(false, true, false, kModeForward);
    if (c.incr_resync > 1)
        return steep ? TWISTY_S(false, kModeForward, true)
                     : launch_t<G, SPL, false, false, false, kModeForward, true>(c, kc, w, init_seg, tab, out, partials,
                                                                                  ma, smem, blocks, st);
    return steep ? TWISTY_S(false, kModeForward, false) : TWISTY_L(false, false, false, kModeForward);
#undef TWISTY_S
#undef TWISTY_L
}


}  // namespace

#define TWISTY_COMP_SHAPE(GG, SS)                                                                           \
    if (a.t.group == GG && a.t.spl == SS) {                                                                 \
        e = launch_g<GG, SS>(a.mode, a.exact, a.clamp, a.shift, a.steep, a.c, a.kc, a.t, a.init_seg, a.tab, a.out, \
                             a.partials, a.ma, a.smem, a.blocks, a.st);                                     \
        return true;                                                                                        \
    }

}  // namespace twisty
