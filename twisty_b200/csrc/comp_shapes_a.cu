// comp_shapes_a.cu -- compensated chain kernel variants for the shapes 1 x 8, 1 x 12, 4 x 2, 4 x 3, 4 x 4, 4 x 5, 4 x 8, 4 x 9, 4 x 16, 4 x 17, 8 x 2, 8 x 4
// (lanes per chain x segments per lane).
#include "comp_launch.cuh"

namespace twisty {

bool launch_comp_shapes_a(const CompLaunch &a, cudaError_t &e)
{
    TWISTY_COMP_SHAPE(4, 4)
    TWISTY_COMP_SHAPE(4, 8)
    TWISTY_COMP_SHAPE(4, 2)
    TWISTY_COMP_SHAPE(4, 3)
    TWISTY_COMP_SHAPE(4, 5)
    TWISTY_COMP_SHAPE(4, 9)
    TWISTY_COMP_SHAPE(4, 16)
    TWISTY_COMP_SHAPE(4, 17)
    TWISTY_COMP_SHAPE(1, 8)
    TWISTY_COMP_SHAPE(1, 12)
    TWISTY_COMP_SHAPE(8, 2)
    TWISTY_COMP_SHAPE(8, 4)
    return false;
}

}  // namespace twisty
