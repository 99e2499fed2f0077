// Test-infrastructure shim (see openvdb/openvdb.h).
#pragma once
#include "../openvdb.h"
namespace openvdb {
namespace tools {
struct BoxSampler {
    template <class TreeT, class PointT>
    static float sample(const TreeT &, const PointT &) { return 0.0f; }
};
}  // namespace tools
}  // namespace openvdb
