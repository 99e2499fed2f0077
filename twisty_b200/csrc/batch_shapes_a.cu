// batch_shapes_a.cu -- batched kernel variants for the shapes 1 x 8, 1 x 12, 4 x 2, 4 x 3, 4 x 4, 4 x 5, 4 x 8, 4 x 9, 4 x 16, 4 x 17, 8 x 2, 8 x 4, 8 x 8, 8 x 9, 8 x 12, 8 x 16, 8 x 17, 16 x 4, 16 x 8, 16 x 12, 16 x 16, 16 x 17
// (lanes per chain x segments per lane).
#include "batch_launch.cuh"

namespace twisty {

bool batch_shapes_a_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e)
{
    TWISTY_BATCH_SHAPE_LAUNCH(4, 4)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 8)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 2)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 3)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 5)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 9)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 16)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 17)
    TWISTY_BATCH_SHAPE_LAUNCH(1, 8)
    TWISTY_BATCH_SHAPE_LAUNCH(1, 12)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 9)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 17)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 17)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 2)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 4)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 8)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 12)
    TWISTY_BATCH_SHAPE_LAUNCH(8, 16)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 4)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 8)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 12)
    TWISTY_BATCH_SHAPE_LAUNCH(16, 16)
    return false;
}

bool batch_shapes_a_occ(const BatchShape &s, size_t smem, int &occ)
{
    TWISTY_BATCH_SHAPE_OCC(4, 4)
    TWISTY_BATCH_SHAPE_OCC(4, 8)
    TWISTY_BATCH_SHAPE_OCC(4, 2)
    TWISTY_BATCH_SHAPE_OCC(4, 3)
    TWISTY_BATCH_SHAPE_OCC(4, 5)
    TWISTY_BATCH_SHAPE_OCC(4, 9)
    TWISTY_BATCH_SHAPE_OCC(4, 16)
    TWISTY_BATCH_SHAPE_OCC(4, 17)
    TWISTY_BATCH_SHAPE_OCC(1, 8)
    TWISTY_BATCH_SHAPE_OCC(1, 12)
    TWISTY_BATCH_SHAPE_OCC(8, 9)
    TWISTY_BATCH_SHAPE_OCC(8, 17)
    TWISTY_BATCH_SHAPE_OCC(16, 17)
    TWISTY_BATCH_SHAPE_OCC(8, 2)
    TWISTY_BATCH_SHAPE_OCC(8, 4)
    TWISTY_BATCH_SHAPE_OCC(8, 8)
    TWISTY_BATCH_SHAPE_OCC(8, 12)
    TWISTY_BATCH_SHAPE_OCC(8, 16)
    TWISTY_BATCH_SHAPE_OCC(16, 4)
    TWISTY_BATCH_SHAPE_OCC(16, 8)
    TWISTY_BATCH_SHAPE_OCC(16, 12)
    TWISTY_BATCH_SHAPE_OCC(16, 16)
    return false;
}

bool batch_shapes_a_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ)
{
    TWISTY_BATCH_SHAPE_ADJ(4, 4)
    TWISTY_BATCH_SHAPE_ADJ(4, 8)
    TWISTY_BATCH_SHAPE_ADJ(4, 2)
    TWISTY_BATCH_SHAPE_ADJ(4, 3)
    TWISTY_BATCH_SHAPE_ADJ(4, 5)
    TWISTY_BATCH_SHAPE_ADJ(4, 9)
    TWISTY_BATCH_SHAPE_ADJ(4, 16)
    TWISTY_BATCH_SHAPE_ADJ(4, 17)
    TWISTY_BATCH_SHAPE_ADJ(1, 8)
    TWISTY_BATCH_SHAPE_ADJ(1, 12)
    TWISTY_BATCH_SHAPE_ADJ(8, 9)
    TWISTY_BATCH_SHAPE_ADJ(8, 17)
    TWISTY_BATCH_SHAPE_ADJ(16, 17)
    TWISTY_BATCH_SHAPE_ADJ(8, 2)
    TWISTY_BATCH_SHAPE_ADJ(8, 4)
    TWISTY_BATCH_SHAPE_ADJ(8, 8)
    TWISTY_BATCH_SHAPE_ADJ(8, 12)
    TWISTY_BATCH_SHAPE_ADJ(8, 16)
    TWISTY_BATCH_SHAPE_ADJ(16, 4)
    TWISTY_BATCH_SHAPE_ADJ(16, 8)
    TWISTY_BATCH_SHAPE_ADJ(16, 12)
    TWISTY_BATCH_SHAPE_ADJ(16, 16)
    return false;
}

}  // namespace twisty
