// comp_shapes_d.cu -- compensated chain kernel variants for the shapes 32 x 4, 32 x 8, 32 x 12, 32 x 17
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_d(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(32, 4)
    TWISTY_COMP_SHAPE(32, 8)
    TWISTY_COMP_SHAPE(32, 12)
    TWISTY_COMP_SHAPE(32, 17)
    return false;
}

}  // namespace twisty
