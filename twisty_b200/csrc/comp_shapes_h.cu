// comp_shapes_h.cu -- compensated chain kernel variants for the shapes 4 x 20, 4 x 24, 4 x 28,
// 4 x 32 (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_h(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(4, 20)
    TWISTY_COMP_SHAPE(4, 24)
    TWISTY_COMP_SHAPE(4, 28)
    TWISTY_COMP_SHAPE(4, 32)
    return false;
}

}  // namespace twisty
