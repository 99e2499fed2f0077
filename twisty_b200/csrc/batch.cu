// batch.cu -- the host side of the batched persistent form: experiment packing, shape and
// occupancy queries, and the launch, which dispatches to the kernel variants instantiated in
// batch_shapes_{a..e}.cu (batch_launch.cuh holds the kernel; comp_body.cuh the chain body).
#include "batch_launch.cuh"

namespace twisty {

// ------------------------------------------------------------------------- batched form
size_t batch_exp_bytes() { return sizeof(BatchExp); }

void batch_pack_experiments(const BatchExpHost *in, uint32_t n, void *dst)
{
    BatchExp *d = static_cast<BatchExp *>(dst);
    for (uint32_t i = 0; i < n; ++i) {
        BatchExp e{};
        e.spec = in[i].spec;
        e.kc = make_consts(in[i].spec.inv_ds, in[i].meta, in[i].spec.n_segments, in[i].lf);
        e.tab = in[i].tab;
        e.lin = in[i].lin;
        e.init_seg = in[i].init_seg;
        e.log10_abs = log10(in[i].spec.absorption_factor);
        e.out_offset = in[i].out_offset;
        d[i] = e;
    }
}

bool batch_shape_supported(const BatchShape &s, uint32_t n_max, uint32_t k_eff)
{
    // single-run shapes only: no batched variant
    if ((s.group == 8 && s.spl == 32) || (s.group == 1 && (s.spl == 16 || s.spl == 24)) ||
        (s.group == 4 && s.spl == 12)) return false;
    CompTuning t{s.group, s.spl, s.warps, s.exact};
    const int maxt = batch_max_threads(s.group, s.spl);
    return comp_tuning_supported(t, n_max, k_eff) && s.warps * 32 <= maxt;
}

size_t batch_smem_bytes(const BatchShape &s, uint32_t bins)
{
    return (s.lut_smem ? (size_t)((bins + 1) / 2) * sizeof(float4) : 0) +
           (size_t)s.warps * warp_state_bytes(s.group, s.spl) + cta_len_bytes(s.group, s.spl);
}

int batch_chains_per_block(const BatchShape &s) { return s.warps * (32 / s.group); }

int batch_blocks_per_sm(const BatchShape &s, int bins)
{
    const size_t smem = batch_smem_bytes(s, (uint32_t)bins);
    int occ = 0;
    if (batch_shapes_a_occ(s, smem, occ) || batch_shapes_b_occ(s, smem, occ) || batch_shapes_c_occ(s, smem, occ) ||
        batch_shapes_d_occ(s, smem, occ) || batch_shapes_e_occ(s, smem, occ))
        return occ;
    return 0;
}

cudaError_t launch_batch(const BatchShape &s, const void *d_exps, const uint2 *d_items, uint32_t n_items,
                         uint32_t *d_counter, ChainOut *out, int bins, int grid, cudaStream_t st)
{
    const BatchExp *exps = static_cast<const BatchExp *>(d_exps);
    const size_t smem = batch_smem_bytes(s, (uint32_t)bins);
    cudaError_t e = cudaSuccess;
    if (batch_shapes_a_launch(s, exps, d_items, n_items, d_counter, out, bins, grid, smem, st, e) ||
        batch_shapes_b_launch(s, exps, d_items, n_items, d_counter, out, bins, grid, smem, st, e) ||
        batch_shapes_c_launch(s, exps, d_items, n_items, d_counter, out, bins, grid, smem, st, e) ||
        batch_shapes_d_launch(s, exps, d_items, n_items, d_counter, out, bins, grid, smem, st, e) ||
        batch_shapes_e_launch(s, exps, d_items, n_items, d_counter, out, bins, grid, smem, st, e))
        return e;
    return cudaErrorInvalidValue;
}

// --------------------------------------------------------------------- batched adjoint
size_t batch_adj_bytes() { return sizeof(BatchAdjExp); }

void batch_pack_adjoint(const BatchAdjHost *in, uint32_t n, void *dst)
{
    BatchAdjExp *d = static_cast<BatchAdjExp *>(dst);
    for (uint32_t i = 0; i < n; ++i) d[i] = BatchAdjExp{in[i].dtab, in[i].ref_log10, 0u};
}

namespace {
bool adjoint_dispatch(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                      uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                      cudaStream_t st, cudaError_t &e, int *occ)
{
    return batch_shapes_a_adjoint(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, e, occ) ||
           batch_shapes_b_adjoint(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, e, occ) ||
           batch_shapes_c_adjoint(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, e, occ) ||
           batch_shapes_d_adjoint(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, e, occ) ||
           batch_shapes_e_adjoint(s, exps, adj, items, n_items, counter, grad, bins, grid, smem, st, e, occ);
}
}  // namespace

int batch_adjoint_blocks_per_sm(const BatchShape &s, int bins)
{
    BatchShape t = s;
    t.lut_smem = 1;
    const size_t smem = batch_smem_bytes(t, (uint32_t)bins);
    int occ = 0;
    cudaError_t e = cudaSuccess;
    if (!adjoint_dispatch(t, nullptr, nullptr, nullptr, 0, nullptr, nullptr, bins, 0, smem, nullptr, e, &occ) ||
        e != cudaSuccess)
        return 0;
    return occ;
}

cudaError_t launch_batch_adjoint(const BatchShape &s, const void *d_exps, const void *d_adj, const uint2 *d_items,
                                 uint32_t n_items, uint32_t *d_counter, double *grad, int bins, int grid,
                                 cudaStream_t st)
{
    BatchShape t = s;
    t.lut_smem = 1;
    const size_t smem = batch_smem_bytes(t, (uint32_t)bins);
    cudaError_t e = cudaSuccess;
    if (adjoint_dispatch(t, static_cast<const BatchExp *>(d_exps), static_cast<const BatchAdjExp *>(d_adj), d_items,
                         n_items, d_counter, grad, bins, grid, smem, st, e, nullptr))
        return e;
    return cudaErrorInvalidValue;
}

}  // namespace twisty
