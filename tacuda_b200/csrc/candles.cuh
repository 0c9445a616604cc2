// Candlestick engine (placeholder until the pattern set lands).
#pragma once
#include "families.cuh"

namespace tb {
constexpr int kCdlHalo = 16;
template <int K>
__device__ void cdl_round(const Ctx<K>&, const Job&) {}
}  // namespace tb
namespace tb {
namespace sp { struct Driver; struct Stage; struct Line; }
}
