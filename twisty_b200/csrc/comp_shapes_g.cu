// comp_shapes_g.cu -- compensated chain kernel variants for the shapes 8 x 20, 8 x 24, 16 x 24,
// 16 x 28, 16 x 32 (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_g(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(8, 20)
    TWISTY_COMP_SHAPE(8, 24)
    TWISTY_COMP_SHAPE(16, 24)
    TWISTY_COMP_SHAPE(16, 28)
    TWISTY_COMP_SHAPE(16, 32)
    return false;
}

}  // namespace twisty
