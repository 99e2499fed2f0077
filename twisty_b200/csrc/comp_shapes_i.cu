// comp_shapes_i.cu -- compensated chain kernel variants for the one-lane shapes 1 x 16, 1 x 24
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_i(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(1, 16)
    TWISTY_COMP_SHAPE(1, 24)
    return false;
}

}  // namespace twisty
