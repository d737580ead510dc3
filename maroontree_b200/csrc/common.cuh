// Small integer helpers shared by the device headers.
#pragma once
#include <stdint.h>

namespace mtd {
__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return max(lo, min(v, hi)); }
__device__ __forceinline__ uint32_t uabs(int32_t v) { return v < 0 ? 0u - (uint32_t)v : (uint32_t)v; }
}  // namespace mtd
