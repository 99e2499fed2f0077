// Test-infrastructure shim (see FMath/Vector3.h): the reference includes this header
// but the compiled hot-path sources use no Matrix3x3 member.
#pragma once
#include "Vector3.h"
namespace Farlor {
struct Matrix3x3 {
    float m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
};
}  // namespace Farlor
