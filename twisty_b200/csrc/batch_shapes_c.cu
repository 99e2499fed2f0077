// batch_shapes_c.cu -- batched kernel variants for the shapes 16 x 20, 32 x 20, 32 x 28
// (lanes per chain x segments per lane).
#include "batch_launch.cuh"

namespace twisty {

bool batch_shapes_c_launch(const BatchShape &s, const BatchExp *exps, const uint2 *items, uint32_t n_items,
                           uint32_t *counter, ChainOut *out, int bins, int grid, size_t smem, cudaStream_t st,
                           cudaError_t &e)
{
    TWISTY_BATCH_SHAPE_LAUNCH(16, 20)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 20)
    TWISTY_BATCH_SHAPE_LAUNCH(32, 28)
    return false;
}

bool batch_shapes_c_occ(const BatchShape &s, size_t smem, int &occ)
{
    TWISTY_BATCH_SHAPE_OCC(16, 20)
    TWISTY_BATCH_SHAPE_OCC(32, 20)
    TWISTY_BATCH_SHAPE_OCC(32, 28)
    return false;
}

bool batch_shapes_c_adjoint(const BatchShape &s, const BatchExp *exps, const BatchAdjExp *adj, const uint2 *items,
                            uint32_t n_items, uint32_t *counter, double *grad, int bins, int grid, size_t smem,
                            cudaStream_t st, cudaError_t &e, int *occ)
{
    TWISTY_BATCH_SHAPE_ADJ(16, 20)
    TWISTY_BATCH_SHAPE_ADJ(32, 20)
    TWISTY_BATCH_SHAPE_ADJ(32, 28)
    return false;
}

}  // namespace twisty
