// Stand-in for the absent bitloop framework header <bitloop/core/types.h>.
// Only what UniformCPU needs to compile: plain 2-vectors and a byte buffer.
#pragma once
#include <cstdint>
#include <vector>

namespace bl
{
template <typename T> struct Vec2
{
    T x{};
    T y{};
    bool operator==(const Vec2&) const = default;
};

using DVec2 = Vec2<double>;
using FVec2 = Vec2<float>;
using IVec2 = Vec2<int>;
using bytebuf = std::vector<std::uint8_t>;
}
