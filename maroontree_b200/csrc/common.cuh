// Small integer helpers shared by the device headers, satd_sad_proxy and
// cfl_pred_pixel.
#pragma once
#include <stdint.h>

namespace mtd {
__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return max(lo, min(v, hi)); }
__device__ __forceinline__ uint32_t uabs(int32_t v) { return v < 0 ? 0u - (uint32_t)v : (uint32_t)v; }

// cfl_pred_pixel (src/intrapred.rs:1194-1199).
__device__ __forceinline__ int32_t cfl_pred_pixel(int32_t dc, int32_t ac, int32_t alpha, int32_t maxv) {
  const int32_t diff = alpha * ac;
  const int32_t mag = (abs(diff) + 32) >> 6;
  return min(max(dc + (diff < 0 ? -mag : mag), 0), maxv);
}

// satd_sad_proxy_scalar (src/rd_sse.rs:1143-1176): SAD + (SATD >> 2) of
// src - pred over 4x4 tiles, with the samples past the displayed window
// (vw x vh from the block origin) taken as the prediction.
template <int N>
__device__ uint64_t satd_sad_proxy(const uint16_t* __restrict__ src, int stride, int px, int py,
                                   const int16_t* __restrict__ pred, int vw, int vh) {
  uint64_t sad = 0, satd = 0;
#pragma unroll 1
  for (int tile = 0; tile < (N / 4) * (N / 4); tile++) {
    const int ty = (tile / (N / 4)) * 4, tx = (tile % (N / 4)) * 4;
    int32_t r[4][4];
#pragma unroll
    for (int y = 0; y < 4; y++) {
      int32_t d[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const bool vis = tx + x < vw && ty + y < vh;
        d[x] = vis ? (int32_t)src[(size_t)(py + ty + y) * stride + px + tx + x] - pred[(ty + y) * N + tx + x] : 0;
        sad += uabs(d[x]);
      }
      const int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], h = d[1] - d[3];
      r[y][0] = e + g;
      r[y][1] = f + h;
      r[y][2] = f - h;
      r[y][3] = e - g;
    }
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int32_t e = r[0][x] + r[2][x], f = r[0][x] - r[2][x], g = r[1][x] + r[3][x], h = r[1][x] - r[3][x];
      satd += (uint64_t)uabs(e + g) + uabs(f + h) + uabs(f - h) + uabs(e - g);
    }
  }
  return sad + (satd >> 2);
}
}  // namespace mtd
