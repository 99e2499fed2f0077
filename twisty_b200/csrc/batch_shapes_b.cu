// batch_shapes_b.cu -- batched kernel variants for the shapes 32 x 4, 32 x 8, 32 x 12, 32 x 16, 32 x 17, 32 x 24, 32 x 32
// (lanes per chain x segments per lane).
#include "batch_launch.cuh"

namespace twisty {

bool batch_shapes_b_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e)
{
    TWISTY_BATCH_SHAPE_LAUNCH(32, 4)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 8)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 12)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 17)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 16)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 24)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 32)
    return false;
}

bool batch_shapes_b_occ(const BatchShape &s, size_t smem, int &occ)
{
    TWISTY_BATCH_SHAPE_OCC(32, 4)
    TWISTY_BATCH_SHAPE_OCC(32, 8)
    TWISTY_BATCH_SHAPE_OCC(32, 12)
    TWISTY_BATCH_SHAPE_OCC(32, 17)
    TWISTY_BATCH_SHAPE_OCC(32, 16)
    TWISTY_BATCH_SHAPE_OCC(32, 24)
    TWISTY_BATCH_SHAPE_OCC(32, 32)
    return false;
}

bool batch_shapes_b_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ)
{
    TWISTY_BATCH_SHAPE_ADJ(32, 4)
    TWISTY_BATCH_SHAPE_ADJ(32, 8)
    TWISTY_BATCH_SHAPE_ADJ(32, 12)
    TWISTY_BATCH_SHAPE_ADJ(32, 17)
    TWISTY_BATCH_SHAPE_ADJ(32, 16)
    TWISTY_BATCH_SHAPE_ADJ(32, 24)
    TWISTY_BATCH_SHAPE_ADJ(32, 32)
    return false;
}

}  // namespace twisty
