// batch_shapes_d.cu -- batched kernel variants for the shapes 8 x 20, 8 x 24, 16 x 24, 16 x 28,
// 16 x 32 (lanes per chain x segments per lane).
#include "batch_launch.cuh"

namespace twisty {

bool batch_shapes_d_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e)
{
    TWISTY_BATCH_SHAPE_LAUNCH(8, 20)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 24)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 24)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 28)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 32)
    return false;
}

bool batch_shapes_d_occ(const BatchShape &s, size_t smem, int &occ)
{
    TWISTY_BATCH_SHAPE_OCC(8, 20)
    TWISTY_BATCH_SHAPE_OCC(8, 24)
    TWISTY_BATCH_SHAPE_OCC(16, 24)
    TWISTY_BATCH_SHAPE_OCC(16, 28)
    TWISTY_BATCH_SHAPE_OCC(16, 32)
    return false;
}

bool batch_shapes_d_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ)
{
    TWISTY_BATCH_SHAPE_ADJ(8, 20)
    TWISTY_BATCH_SHAPE_ADJ(8, 24)
    TWISTY_BATCH_SHAPE_ADJ(16, 24)
    TWISTY_BATCH_SHAPE_ADJ(16, 28)
    TWISTY_BATCH_SHAPE_ADJ(16, 32)
    return false;
}

}  // namespace twisty
