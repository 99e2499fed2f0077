// comp_shapes_f.cu -- compensated chain kernel variants for the shapes 16 x 20, 32 x 20, 32 x 28
// (lanes per chain x segments per lane): the N between 16 x 17 and 32 x 12, 32 x 17 and 32 x 24,
// 32 x 24 and 32 x 32 with less padding.
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_f(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(16, 20)
    TWISTY_COMP_SHAPE(32, 20)
    TWISTY_COMP_SHAPE(32, 28)
    return false;
}

}  // namespace twisty
