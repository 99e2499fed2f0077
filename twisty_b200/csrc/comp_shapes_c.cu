// comp_shapes_c.cu -- compensated chain kernel variants for the shapes 16 x 4, 16 x 8, 16 x 12, 16 x 16, 16 x 17
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_c(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(16, 4)
    TWISTY_COMP_SHAPE(16, 8)
    TWISTY_COMP_SHAPE(16, 12)
    TWISTY_COMP_SHAPE(16, 16)
    TWISTY_COMP_SHAPE(16, 17)
    return false;
}

}  // namespace twisty
