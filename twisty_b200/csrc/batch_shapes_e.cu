// batch_shapes_e.cu -- batched kernel variants for the shapes 4 x 20, 4 x 24, 4 x 28, 4 x 32
// (lanes per chain x segments per lane).
#include "batch_launch.cuh"

namespace twisty {

bool batch_shapes_e_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e)
{
    TWISTY_BATCH_SHAPE_LAUNCH(4, 20)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 24)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 28)
    TWISTY_BATCH_SHAPE_LAUNCH(4, 32)
    return false;
}

bool batch_shapes_e_occ(const BatchShape &s, size_t smem, int &occ)
{
    TWISTY_BATCH_SHAPE_OCC(4, 20)
    TWISTY_BATCH_SHAPE_OCC(4, 24)
    TWISTY_BATCH_SHAPE_OCC(4, 28)
    TWISTY_BATCH_SHAPE_OCC(4, 32)
    return false;
}

bool batch_shapes_e_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ)
{
    TWISTY_BATCH_SHAPE_ADJ(4, 20)
    TWISTY_BATCH_SHAPE_ADJ(4, 24)
    TWISTY_BATCH_SHAPE_ADJ(4, 28)
    TWISTY_BATCH_SHAPE_ADJ(4, 32)
    return false;
}

}  // namespace twisty
