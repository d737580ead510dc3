// Batched decision distortion of reconstructed blocks (sse_recon,
// src/rd_sse.rs:449-475): one thread per block, the plain or weighted SSE of
// wsse.cuh.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"
#include "wsse.cuh"

namespace {

__global__ void __launch_bounds__(128) sse_recon_kernel(const uint16_t* __restrict__ src, int stride, int vis_w,
                                                        int vis_h, int maxv, const uint16_t* __restrict__ pos,
                                                        const int32_t* __restrict__ pred,
                                                        const int32_t* __restrict__ resid, int n, int w, int h,
                                                        float scale, long long* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int px = pos[2 * b], py = pos[2 * b + 1];
  mtd::ErrBlock<int32_t, int32_t> e;
  e.src = src + (size_t)py * stride + px;
  e.stride = stride;
  e.pred = pred + (size_t)b * w * h;
  e.resid = resid ? resid + (size_t)b * w * h : nullptr;
  e.w = w;
  e.vw = min(max(vis_w - px, 0), w);
  e.vh = min(max(vis_h - py, 0), h);
  e.maxv = maxv;
  out[b] = mtd::sse_recon_block(e, scale);
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
