// Test-infrastructure shim: a minimal stand-in for Farlor::Vector3 from the
// un-vendored, unpinned FMath dependency (github.com/BrennenTaylor/FMath, fetched
// without a GIT_TAG by the reference's dependencies/CMakeLists.txt:10-13).
// Only used to compile the reference sources into the oracle pin (oracle/_ref).
//
// This file FIXES the arithmetic at that boundary (the "pinned definition"):
//   Dot        = x*x' + y*y' + z*z'   evaluated left to right, no FMA contraction
//   Magnitude  = sqrtf(Dot(self))
//   Normalized = self * (1.0f / sqrtf(Dot(self)))   (the same operation order as the
//                reference's own _CudaSafe tangent code, Twisty/CurvePerturbUtils.cpp:209-214)
#pragma once
#include <array>
#include <cmath>
#include <ostream>

namespace Farlor {
struct Vector3 {
    union {
        std::array<float, 3> m_data;
        struct {
            float x, y, z;
        };
    };
    Vector3() : m_data{0.0f, 0.0f, 0.0f} {}
    Vector3(float a, float b, float c) : m_data{a, b, c} {}
    Vector3(const Vector3 &o) : m_data(o.m_data) {}
    Vector3 &operator=(const Vector3 &o) { m_data = o.m_data; return *this; }

    Vector3 operator+(const Vector3 &o) const { return Vector3(x + o.x, y + o.y, z + o.z); }
    Vector3 operator-(const Vector3 &o) const { return Vector3(x - o.x, y - o.y, z - o.z); }
    Vector3 operator-() const { return Vector3(-x, -y, -z); }
    Vector3 operator*(float s) const { return Vector3(x * s, y * s, z * s); }
    Vector3 &operator+=(const Vector3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    Vector3 &operator-=(const Vector3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    Vector3 &operator*=(float s) { x *= s; y *= s; z *= s; return *this; }

    float Dot(const Vector3 &o) const { return x * o.x + y * o.y + z * o.z; }
    Vector3 Cross(const Vector3 &o) const
    {
        return Vector3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    float SqrMagnitude() const { return Dot(*this); }
    float Magnitude() const { return std::sqrt(SqrMagnitude()); }
    Vector3 Normalized() const
    {
        const float inv = 1.0f / std::sqrt(SqrMagnitude());
        return (*this) * inv;
    }
    void Normalize() { *this = Normalized(); }
};
inline Vector3 operator*(float s, const Vector3 &v) { return v * s; }
inline std::ostream &operator<<(std::ostream &os, const Vector3 &v)
{
    return os << "(" << v.x << ", " << v.y << ", " << v.z << ")";
}
}  // namespace Farlor
