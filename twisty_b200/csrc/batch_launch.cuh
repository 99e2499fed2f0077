// batch_launch.cuh -- the batched persistent kernel and its per-shape launchers, included by
// batch.cu (the host side of the batched form) and by batch_shapes_{a..e}.cu, which instantiate
// the kernel for a few shapes each so that the variants compile in parallel.
#pragma once
#include "comp_body.cuh"

namespace twisty {

// ---------------------------------------------------------------------------------------
// Batched persistent form: many experiments (uneven N, S, mu_s, eps) per launch. Work items
// are (experiment, first chain of a CTA's worth of chains), sorted by cost; persistent CTAs
// pull items from a device counter (atomicAdd), stage that experiment's table in shared
// memory (or read it through L1), and run their chains with chain_body.
// ---------------------------------------------------------------------------------------
struct BatchExp {
    ChainSpec spec;
    CompConsts kc;
    const float2 *tab;
    const float2 *lin;       // linear table (the fallback of steep bins in the fixed-point form)
    const float *init_seg;
    double log10_abs;
    uint32_t out_offset;
    uint32_t pad;
};

// Per-experiment inputs of the batched adjoint replay beyond BatchExp (whose table is then the
// linear table, staged in shared memory): the derivative tables with respect to mu_s and eps
// (launch_deriv_tables layout) and the reference the path weights are scaled by.
struct BatchAdjExp {
    const float4 *dtab;
    float ref_log10;
    uint32_t pad;
};

// Each returns false when the shape is not among its own; else launches (sets e) or reports
// the occupancy (sets occ).
bool batch_shapes_a_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e);   // 1 x {8, 12}, 4 x {2..9}, 8 x {2..17}, 16 x {4, 8, 12, 16, 17}
bool batch_shapes_b_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e);   // 32 x {4, 8, 12, 16, 17, 24, 32}
bool batch_shapes_c_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e);   // 16 x 20, 32 x {20, 28}
bool batch_shapes_d_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e);   // 8 x {20, 24}, 16 x {24, 28, 32}
bool batch_shapes_e_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e);   // 4 x {20, 24, 28, 32}
// The adjoint replay of the same shapes (table staged, exact blend, clamping).
bool batch_shapes_a_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ);
bool batch_shapes_b_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ);
bool batch_shapes_c_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ);
bool batch_shapes_d_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ);
bool batch_shapes_e_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ);
bool batch_shapes_a_occ(const BatchShape &s, size_t smem, int &occ);
bool batch_shapes_b_occ(const BatchShape &s, size_t smem, int &occ);
bool batch_shapes_c_occ(const BatchShape &s, size_t smem, int &occ);
bool batch_shapes_d_occ(const BatchShape &s, size_t smem, int &occ);
bool batch_shapes_e_occ(const BatchShape &s, size_t smem, int &occ);

namespace {

template <int G, int SPL, bool EXACT, bool LUT_SMEM, bool CLAMP, bool STEEP, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) batch_kernel(const BatchExp *__restrict__ exps,
                                                        const uint2 *__restrict__ items, uint32_t n_items,
                                                        uint32_t *__restrict__ counter, ChainOut *__restrict__ out,
                                                        int bins)
{
    extern __shared__ float4 smem4[];
    __shared__ uint32_t s_item;
    const int tab_f4 = LUT_SMEM ? (bins + 1) / 2 : 0;
    unsigned char *s_state = reinterpret_cast<unsigned char *>(smem4 + tab_f4);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q = lane / G, j = lane % G;
    constexpr int CPW = 32 / G;
    using Lay = Layout<G, SPL>;
    unsigned char *wb = s_state + (size_t)warp * Lay::WARP_BYTES;
    float *s_len = reinterpret_cast<float *>(s_state + (size_t)(blockDim.x >> 5) * Lay::WARP_BYTES);
    const Planes st{reinterpret_cast<float2 *>(wb), reinterpret_cast<float *>(wb + Lay::XY_BYTES), s_len};
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items) break;
        const uint2 it = items[item];
        const BatchExp &e = exps[it.x];
        const float2 *tab = e.tab;
        if (LUT_SMEM) {
            stage_table(smem4, e.tab, bins);
            tab = reinterpret_cast<const float2 *>(smem4);
        }
        fill_lengths(s_len, e.init_seg, e.spec.n_segments, G * SPL);
        __syncthreads();
        ModeArgs ma{};
        ma.log10_abs = e.log10_abs;
        ma.lin = e.lin;
        const uint32_t chain = it.y + warp * CPW + q;
        chain_body<G, SPL, EXACT, CLAMP, false, kModeForward, false, STEEP, !LUT_SMEM>(e.spec, e.kc, e.init_seg, tab, st,
                                                                                       q * G, j,
                                                                            chain, chain < e.spec.n_chains,
                                                                            out + e.out_offset, ma);
        __syncthreads();
    }
}

// Adjoint replay of a batch: the forward pass's work items, each CTA staging its experiment's
// linear table and running the chains in the adjoint mode of the chain body (exact blend,
// curvatures recomputed, nothing stored per step); per-chain gradient sums go to
// grad[(out_offset + chain) * 6 ...].
template <int G, int SPL, int MAXT>
__global__ void __launch_bounds__(MAXT, 1) batch_adjoint_kernel(const BatchExp *__restrict__ exps,
                                                                const BatchAdjExp *__restrict__ adj,
                                                                const uint2 *__restrict__ items, uint32_t n_items,
                                                                uint32_t *__restrict__ counter,
                                                                double *__restrict__ grad, int bins)
{
    extern __shared__ float4 smem4[];
    __shared__ uint32_t s_item;
    const int tab_f4 = (bins + 1) / 2;
    unsigned char *s_state = reinterpret_cast<unsigned char *>(smem4 + tab_f4);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t q = lane / G, j = lane % G;
    constexpr int CPW = 32 / G;
    using Lay = Layout<G, SPL>;
    unsigned char *wb = s_state + (size_t)warp * Lay::WARP_BYTES;
    float *s_len = reinterpret_cast<float *>(s_state + (size_t)(blockDim.x >> 5) * Lay::WARP_BYTES);
    const Planes st{reinterpret_cast<float2 *>(wb), reinterpret_cast<float *>(wb + Lay::XY_BYTES), s_len};
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items) break;
        const uint2 it = items[item];
        const BatchExp &e = exps[it.x];
        const BatchAdjExp &a = adj[it.x];
        stage_table(smem4, e.tab, bins);
        fill_lengths(s_len, e.init_seg, e.spec.n_segments, G * SPL);
        __syncthreads();
        ModeArgs ma{};
        ma.log10_abs = e.log10_abs;
        ma.lin = e.lin;
        ma.dtab = a.dtab;
        ma.ref_log10 = a.ref_log10;
        ma.grad = grad + (size_t)e.out_offset * 6;
        const uint32_t chain = it.y + warp * CPW + q;
        chain_body<G, SPL, true, true, false, kModeAdjoint>(e.spec, e.kc, e.init_seg,
                                                            reinterpret_cast<const float2 *>(smem4), st, q * G, j,
                                                            chain, chain < e.spec.n_chains, nullptr, ma);
        __syncthreads();
    }
}

template <int G, int SPL>
cudaError_t batch_adjoint_g(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, int *occ)
{
    constexpr int MAXT = batch_max_threads(G, SPL);
    if (s.warps * 32 > MAXT) return cudaErrorInvalidConfiguration;
    auto kern = batch_adjoint_kernel<G, SPL, MAXT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, s.warps * 32, smem);
    kern<<<grid, s.warps * 32, smem, st>>>(exps, adj, items, n_items, counter, grad, bins);
    return cudaGetLastError();
}

template <int G, int SPL, bool EXACT, bool LS, bool CL, bool SP>
cudaError_t batch_t(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items, uint32_t *counter,
                    ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st)
{
    constexpr int MAXT = batch_max_threads(G, SPL);
    if (s.warps * 32 > MAXT) return cudaErrorInvalidConfiguration;
    auto kern = batch_kernel<G, SPL, EXACT, LS, CL, SP, MAXT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, s.warps * 32, smem, st>>>(exps, items, n_items, counter, out, bins);
    return cudaGetLastError();
}

template <int G, int SPL, bool EXACT, bool LS, bool CL, bool SP>
int batch_occ_t(const BatchShape &s, size_t smem)
{
    constexpr int MAXT = batch_max_threads(G, SPL);
    auto kern = batch_kernel<G, SPL, EXACT, LS, CL, SP, MAXT>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, s.warps * 32, smem) != cudaSuccess) return 0;
    return nb;
}

// Instantiated: exact tables with clamping (table in shared memory or read through L1);
// fixed-point tables with or without clamping, in shared memory with the steep-bin fallback
// or read through L1 without it.
template <int G, int SPL>
int batch_occ_g(const BatchShape &s, size_t smem)
{
    if (s.exact) return s.lut_smem ? batch_occ_t<G, SPL, true, true, true, false>(s, smem)
                                   : batch_occ_t<G, SPL, true, false, true, false>(s, smem);
    if (s.lut_smem != s.steep) return 0;
    if (s.steep) return s.clamp ? batch_occ_t<G, SPL, false, true, true, true>(s, smem)
                                : batch_occ_t<G, SPL, false, true, false, true>(s, smem);
    return s.clamp ? batch_occ_t<G, SPL, false, false, true, false>(s, smem)
                   : batch_occ_t<G, SPL, false, false, false, false>(s, smem);
}

template <int G, int SPL>
cudaError_t batch_g(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items, uint32_t *counter,
                    ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st)
{
#define TWISTY_BT(E, LS, CL, SP) batch_t<G, SPL, E, LS, CL, SP>(s, exps, items, n_items, counter, out, bins, grid, smem, st)
    if (s.exact) return s.lut_smem ? TWISTY_BT(true, true, true, false) : TWISTY_BT(true, false, true, false);
    if (s.lut_smem != s.steep) return cudaErrorInvalidValue;
    if (s.steep) return s.clamp ? TWISTY_BT(false, true, true, true) : TWISTY_BT(false, true, false, true);
    return s.clamp ? TWISTY_BT(false, false, true, false) : TWISTY_BT(false, false, false, false);
#undef TWISTY_BT
}

}  // namespace

#define TWISTY_BATCH_SHAPE_LAUNCH(GG, SS) \
    if (s.group == GG && s.spl == SS) {   \
        e = batch_g<GG, SS>(s, exps, items, n_items, counter, out, bins, grid, smem, st); \
        return true;                       \
    }
#define TWISTY_BATCH_SHAPE_ADJ(GG, SS)                                                                  \
    if (s.group == GG && s.spl == SS) {                                                                 \
        e = batch_adjoint_g<GG, SS>(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, occ); \
        return true;                                                                                    \
    }
#define TWISTY_BATCH_SHAPE_OCC(GG, SS)   \
    if (s.group == GG && s.spl == SS) { \
        occ = batch_occ_g<GG, SS>(s, smem); \
        return true;                     \
    }

}  // namespace twisty
