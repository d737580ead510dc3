// Device decision distortion of one reconstructed block (sse_recon,
// src/rd_sse.rs:449-475): the plain SSE of clamp(pred + resid) against the
// displayed part of the source, or the scaled 4x4-DCT weighted SSE
// (weighted_dist, src/rd_sse.rs:244-271) in the pinned AVX2 order
// (src/avx/rd.rs:767-848): 8-lane accumulators per row-transform index k over
// the 8-wide tile pairs in (row, column) order, the lane-pair / k reduction,
// the 4-wide tail tiles into the 4 sums, then (s0 + s2) + (s1 + s3).  The error
// is formed on the fly from the source, prediction and residual.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace mtd {

// The weighted-SSE 4x4 DCT basis and weights (src/rd_sse.rs:1400-1430).
constexpr float kWsseRawMean = 0.4625f;
__constant__ float kWsseD[4][4] = {{0.5f, 0.5f, 0.5f, 0.5f},
                               {0.6532815f, 0.27059805f, -0.27059805f, -0.6532815f},
                               {0.5f, -0.5f, -0.5f, 0.5f},
                               {0.27059805f, -0.6532815f, 0.6532815f, -0.27059805f}};
__constant__ float kWsseW[4][4] = {
    {1.8f / kWsseRawMean, 1.0f / kWsseRawMean, 0.4f / kWsseRawMean, 0.2f / kWsseRawMean},
    {1.0f / kWsseRawMean, 0.8f / kWsseRawMean, 0.2f / kWsseRawMean, 0.2f / kWsseRawMean},
    {0.4f / kWsseRawMean, 0.2f / kWsseRawMean, 0.2f / kWsseRawMean, 0.2f / kWsseRawMean},
    {0.2f / kWsseRawMean, 0.2f / kWsseRawMean, 0.2f / kWsseRawMean, 0.2f / kWsseRawMean},
};

template <typename P, typename Q>
struct ErrBlock {
  const uint16_t* src;  // block origin in the source plane
  int stride;
  const P* pred;  // packed w-wide
  const Q* resid;  // packed w-wide, or NULL (zero)
  int w, vw, vh, maxv;
  __device__ __forceinline__ int32_t at(int x, int y) const {
    if (x >= vw || y >= vh) return 0;
    const int i = y * w + x;
    return (int32_t)src[(size_t)y * stride + x] - clampi((int32_t)pred[i] + (resid ? (int32_t)resid[i] : 0), 0, maxv);
  }
};

// weighted_sse of the pw x ph error (multiples of 4) in the AVX2 order.
template <typename E>
__device__ float weighted_sse(const E& e, int pw, int ph) {
  float total[4][8];
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int ln = 0; ln < 8; ln++) total[k][ln] = 0.0f;
  const int pairs = pw / 8 * 8;
  for (int r0 = 0; r0 < ph; r0 += 4)
    for (int c0 = 0; c0 < pairs; c0 += 8) {
      float rows[4][8];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int ln = 0; ln < 8; ln++) rows[i][ln] = (float)e.at(c0 + ln, r0 + i);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float t[8];
#pragma unroll
        for (int ln = 0; ln < 8; ln++) {
          float v = __fmul_rn(rows[0][ln], kWsseD[k][0]);
          v = __fmaf_rn(rows[1][ln], kWsseD[k][1], v);
          v = __fmaf_rn(rows[2][ln], kWsseD[k][2], v);
          v = __fmaf_rn(rows[3][ln], kWsseD[k][3], v);
          t[ln] = v;
        }
#pragma unroll
        for (int ln = 0; ln < 8; ln++) {
          const int hb = ln & 4, l = ln & 3;
          float c = __fmul_rn(kWsseD[l][0], t[hb + 0]);
          c = __fmaf_rn(kWsseD[l][1], t[hb + 1], c);
          c = __fmaf_rn(kWsseD[l][2], t[hb + 2], c);
          c = __fmaf_rn(kWsseD[l][3], t[hb + 3], c);
          total[k][ln] = __fmaf_rn(__fmul_rn(kWsseW[k][l], c), c, total[k][ln]);
        }
      }
    }
  float sum[4];
#pragma unroll
  for (int l = 0; l < 4; l++) {
    const float a = __fadd_rn(__fadd_rn(total[0][l], total[0][4 + l]), __fadd_rn(total[1][l], total[1][4 + l]));
    sum[l] = __fadd_rn(a, __fadd_rn(__fadd_rn(total[2][l], total[2][4 + l]), __fadd_rn(total[3][l], total[3][4 + l])));
  }
  if (pairs < pw) {
    const int c0 = pairs;
    for (int r0 = 0; r0 < ph; r0 += 4) {
      float rows[4][4];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int ln = 0; ln < 4; ln++) rows[i][ln] = (float)e.at(c0 + ln, r0 + i);
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float t[4];
#pragma unroll
        for (int ln = 0; ln < 4; ln++) {
          float v = __fmul_rn(rows[0][ln], kWsseD[k][0]);
          v = __fmaf_rn(rows[1][ln], kWsseD[k][1], v);
          v = __fmaf_rn(rows[2][ln], kWsseD[k][2], v);
          v = __fmaf_rn(rows[3][ln], kWsseD[k][3], v);
          t[ln] = v;
        }
#pragma unroll
        for (int l = 0; l < 4; l++) {
          float c = __fmul_rn(kWsseD[l][0], t[0]);
          c = __fmaf_rn(kWsseD[l][1], t[1], c);
          c = __fmaf_rn(kWsseD[l][2], t[2], c);
          c = __fmaf_rn(kWsseD[l][3], t[3], c);
          sum[l] = __fmaf_rn(__fmul_rn(kWsseW[k][l], c), c, sum[l]);
        }
      }
    }
  }
  return __fadd_rn(__fadd_rn(sum[0], sum[2]), __fadd_rn(sum[1], sum[3]));
}

// sse_recon of one block from its error view: 0 for a block outside the
// displayed plane, round(weighted_sse * scale) (half away from zero) over the
// displayed part padded to whole 4x4 tiles when scale > 0, else the plain SSE.
template <typename E>
__device__ long long sse_recon_block(const E& e, float scale) {
  if (e.vw <= 0 || e.vh <= 0) return 0;
  if (scale > 0.0f) {
    const int pw = (e.vw + 3) & ~3, ph = (e.vh + 3) & ~3;
    const float d = weighted_sse(e, pw, ph);
    return __float2ll_rz(roundf(__fmul_rn(d, scale)));
  }
  long long s = 0;
  for (int y = 0; y < e.vh; y++)
    for (int x = 0; x < e.vw; x++) {
      const long long v = e.at(x, y);
      s += v * v;
    }
  return s;
}

}  // namespace mtd
