// Test-infrastructure shim (see FMath/Vector3.h).
#pragma once
#include "Matrix3x3.h"
#include "Vector3.h"
