// Core types, identical to the reference's include/velographx/types.hpp:5-7.
#pragma once
#include <cstdint>

namespace velographx {
using VertexId = std::uint32_t;
using EdgeOffset = std::uint64_t;
inline constexpr std::uint32_t kUnreachable = UINT32_MAX;
}  // namespace velographx
