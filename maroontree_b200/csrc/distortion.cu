// Decision distortion of reconstructed blocks (sse_recon, src/rd_sse.rs:449-475):
// the plain SSE of clamp(pred + resid) against the displayed part of the
// source, or the scaled 4x4-DCT weighted SSE (weighted_dist,
// src/rd_sse.rs:244-271) in the pinned AVX2 order (src/avx/rd.rs:767-848):
// 8-lane accumulators per row-transform index k over the 8-wide tile pairs in
// (row, column) order, the lane-pair / k reduction, the 4-wide tail tiles into
// the 4 sums, then (s0 + s2) + (s1 + s3).  One thread per block; the error is
// formed on the fly from the source, prediction and residual.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"

namespace {

using mtd::clampi;

// The weighted-SSE 4x4 DCT basis and weights (src/rd_sse.rs:1400-1430).
constexpr float kRawMean = 0.4625f;
__constant__ float kD[4][4] = {{0.5f, 0.5f, 0.5f, 0.5f},
                               {0.6532815f, 0.27059805f, -0.27059805f, -0.6532815f},
                               {0.5f, -0.5f, -0.5f, 0.5f},
                               {0.27059805f, -0.6532815f, 0.6532815f, -0.27059805f}};
__constant__ float kW[4][4] = {
    {1.8f / kRawMean, 1.0f / kRawMean, 0.4f / kRawMean, 0.2f / kRawMean},
    {1.0f / kRawMean, 0.8f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
    {0.4f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
    {0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
};

struct ErrBlock {
  const uint16_t* src;  // block origin in the source plane
  int stride;
  const int32_t* pred;  // packed w-wide
  const int32_t* resid;
  int w, vw, vh, maxv;
  __device__ __forceinline__ int32_t at(int x, int y) const {
    if (x >= vw || y >= vh) return 0;
    const int i = y * w + x;
    return (int32_t)src[(size_t)y * stride + x] - clampi(pred[i] + (resid ? resid[i] : 0), 0, maxv);
  }
};

// weighted_sse of the pw x ph error (multiples of 4) in the AVX2 order.
__device__ float weighted_sse(const ErrBlock& e, int pw, int ph) {
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
          float v = __fmul_rn(rows[0][ln], kD[k][0]);
          v = __fmaf_rn(rows[1][ln], kD[k][1], v);
          v = __fmaf_rn(rows[2][ln], kD[k][2], v);
          v = __fmaf_rn(rows[3][ln], kD[k][3], v);
          t[ln] = v;
        }
#pragma unroll
        for (int ln = 0; ln < 8; ln++) {
          const int hb = ln & 4, l = ln & 3;
          float c = __fmul_rn(kD[l][0], t[hb + 0]);
          c = __fmaf_rn(kD[l][1], t[hb + 1], c);
          c = __fmaf_rn(kD[l][2], t[hb + 2], c);
          c = __fmaf_rn(kD[l][3], t[hb + 3], c);
          total[k][ln] = __fmaf_rn(__fmul_rn(kW[k][l], c), c, total[k][ln]);
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
          float v = __fmul_rn(rows[0][ln], kD[k][0]);
          v = __fmaf_rn(rows[1][ln], kD[k][1], v);
          v = __fmaf_rn(rows[2][ln], kD[k][2], v);
          v = __fmaf_rn(rows[3][ln], kD[k][3], v);
          t[ln] = v;
        }
#pragma unroll
        for (int l = 0; l < 4; l++) {
          float c = __fmul_rn(kD[l][0], t[0]);
          c = __fmaf_rn(kD[l][1], t[1], c);
          c = __fmaf_rn(kD[l][2], t[2], c);
          c = __fmaf_rn(kD[l][3], t[3], c);
          sum[l] = __fmaf_rn(__fmul_rn(kW[k][l], c), c, sum[l]);
        }
      }
    }
  }
  return __fadd_rn(__fadd_rn(sum[0], sum[2]), __fadd_rn(sum[1], sum[3]));
}

__global__ void __launch_bounds__(128) sse_recon_kernel(const uint16_t* __restrict__ src, int stride, int vis_w,
                                                        int vis_h, int maxv, const uint16_t* __restrict__ pos,
                                                        const int32_t* __restrict__ pred,
                                                        const int32_t* __restrict__ resid, int n, int w, int h,
                                                        float scale, long long* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int px = pos[2 * b], py = pos[2 * b + 1];
  ErrBlock e;
  e.src = src + (size_t)py * stride + px;
  e.stride = stride;
  e.pred = pred + (size_t)b * w * h;
  e.resid = resid ? resid + (size_t)b * w * h : nullptr;
  e.w = w;
  e.vw = min(max(vis_w - px, 0), w);
  e.vh = min(max(vis_h - py, 0), h);
  e.maxv = maxv;
  if (e.vw == 0 || e.vh == 0) {
    out[b] = 0;
    return;
  }
  if (scale > 0.0f) {
    const int pw = (e.vw + 3) & ~3, ph = (e.vh + 3) & ~3;
    const float d = weighted_sse(e, pw, ph);
    out[b] = __float2ll_rz(roundf(__fmul_rn(d, scale)));
  } else {
    long long s = 0;
    for (int y = 0; y < e.vh; y++)
      for (int x = 0; x < e.vw; x++) {
        const long long v = e.at(x, y);
        s += v * v;
      }
    out[b] = s;
  }
}

int check(int32_t stride, int32_t vis_w, int32_t vis_h, int32_t bd, int32_t n, int32_t w, int32_t h,
          float scale) {
  if (n < 0 || stride <= 0 || vis_w < 0 || vis_h < 0) return MT_ERR_INVALID_INPUT;
  if (w <= 0 || h <= 0 || (w & 3) || (h & 3) || w > 64 || h > 64) return MT_ERR_INVALID_INPUT;
  if (bd != 8 && bd != 10 && bd != 12) return MT_ERR_UNSUPPORTED;
  if (!(scale >= 0.0f)) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int mt_sse_recon_device(const uint16_t* d_src, int32_t stride, int32_t vis_w, int32_t vis_h, int32_t bd,
                        const uint16_t* d_pos, const int32_t* d_pred, const int32_t* d_resid, int32_t n, int32_t w,
                        int32_t h, float wsse_scale, int64_t* d_out, void* stream) {
  int rc = check(stride, vis_w, vis_h, bd, n, w, h, wsse_scale);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_pos || !d_pred || !d_out) return MT_ERR_INVALID_INPUT;
  sse_recon_kernel<<<(n + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_src, stride, vis_w, vis_h, (1 << bd) - 1, d_pos, d_pred, d_resid, n, w, h, wsse_scale,
      reinterpret_cast<long long*>(d_out));
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_sse_recon(const uint16_t* src, int32_t stride, int32_t plane_h, int32_t vis_w, int32_t vis_h, int32_t bd,
                 const uint16_t* pos, const int32_t* pred, const int32_t* resid, int32_t n, int32_t w, int32_t h,
                 float wsse_scale, int64_t* out) {
  int rc = check(stride, vis_w, vis_h, bd, n, w, h, wsse_scale);
  if (rc != MT_OK) return rc;
  if (plane_h <= 0) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  if (!src || !pos || !pred || !out) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)stride * plane_h * 2, nb = (size_t)n * w * h * 4;
  const size_t o_src = 0, o_pos = up256(plane), o_pred = o_pos + up256((size_t)n * 4), o_res = o_pred + up256(nb),
               o_out = o_res + up256(resid ? nb : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_out + up256((size_t)n * 8)) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_pos, pos, (size_t)n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_pred, pred, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && resid) e = cudaMemcpy(d + o_res, resid, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_sse_recon_device(reinterpret_cast<const uint16_t*>(d + o_src), stride, vis_w, vis_h, bd,
                             reinterpret_cast<const uint16_t*>(d + o_pos), reinterpret_cast<const int32_t*>(d + o_pred),
                             resid ? reinterpret_cast<const int32_t*>(d + o_res) : nullptr, n, w, h, wsse_scale,
                             reinterpret_cast<int64_t*>(d + o_out), nullptr);
    if (rc == MT_OK) e = cudaMemcpy(out, d + o_out, (size_t)n * 8, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
