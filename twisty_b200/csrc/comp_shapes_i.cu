// comp_shapes_i.cu -- compensated chain kernel variants for the one-lane shapes 1 x 16, 1 x 24
// and for 4 x 12 (lanes per chain x segments per lane): single-run shapes of N = 13..24 and
// 37..48, which the batched kernels do not have.
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_i(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(1, 16)
    TWISTY_COMP_SHAPE(1, 24)
    TWISTY_COMP_SHAPE(4, 12)
    return false;
}

}  // namespace twisty
