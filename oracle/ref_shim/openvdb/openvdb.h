// Test-infrastructure shim: type-only stand-ins for the OpenVDB symbols named by the
// position-dependent weighter (Twisty/PathWeighters.cpp:216-241), which is outside the
// hot path and never called by the runner. Every member returns a neutral value.
#pragma once
#include <memory>
namespace openvdb {
struct Vec3d {
    double v[3];
    Vec3d(double a = 0, double b = 0, double c = 0) : v{a, b, c} {}
};
typedef Vec3d Vec3R;
struct Coord {};
struct FloatTree {};
struct FloatGrid {
    typedef std::shared_ptr<FloatGrid> Ptr;
    typedef float ValueType;
    struct Accessor {};
    Accessor getAccessor() { return Accessor(); }
    Vec3d worldToIndex(const Vec3d &p) const { return p; }
    const FloatTree &tree() const { return m_tree; }
    FloatTree m_tree;
};
inline void initialize() {}
}  // namespace openvdb
