// comp_shapes_b.cu -- compensated chain kernel variants for the shapes 8 x 8, 8 x 9, 8 x 12, 8 x 16, 8 x 17, 8 x 32
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_b(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(8, 8)
    TWISTY_COMP_SHAPE(8, 12)
    TWISTY_COMP_SHAPE(8, 16)
    TWISTY_COMP_SHAPE(8, 9)
    TWISTY_COMP_SHAPE(8, 17)
    TWISTY_COMP_SHAPE(8, 32)
    return false;
}

}  // namespace twisty
