// comp_shapes_e.cu -- compensated chain kernel variants for the shapes 32 x 16, 32 x 24, 32 x 32
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_e(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(32, 16)
    TWISTY_COMP_SHAPE(32, 24)
    TWISTY_COMP_SHAPE(32, 32)
    return false;
}

}  // namespace twisty
