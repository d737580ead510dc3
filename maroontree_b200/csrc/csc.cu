// Colour conversion + padding: interleaved 8-bit RGB -> the coder's padded
// u16 Y/Cb/Cr planes in one pass.  Q13 BT.601 full-range coefficients of the
// reference (src/encoder.rs:113-127, :403-409); 4:2:0 chroma averages the four
// unrounded Q13 values of each 2x2 quad with the last row/column repeated
// (src/encoder.rs:560-604); every plane is edge-padded to a multiple of 8
// (src/dispatch.rs:113-131, :180-215): padded[y][x] = plane[min(y,h-1)][min(x,w-1)].
// One thread writes one padded output sample (luma) or one chroma pair, so
// every store is coalesced; the RGB reads are served from L2 after the first
// touch of each row.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"

namespace {

constexpr int kQ = 13;
constexpr int kHalf = 1 << (kQ - 1);

__device__ __forceinline__ int32_t clamp255(int32_t v) { return max(0, min(v, 255)); }

__device__ __forceinline__ void load_rgb(const uint8_t* __restrict__ rgb, int w, int x, int y, int32_t& r, int32_t& g,
                                         int32_t& b) {
  const uint8_t* p = rgb + ((size_t)y * w + x) * 3;
  r = p[0];
  g = p[1];
  b = p[2];
}

__global__ void luma_kernel(const uint8_t* __restrict__ rgb, int w, int h, int pw, int ph, uint16_t* __restrict__ y) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (x >= pw || row >= ph) return;
  int32_t r, g, b;
  load_rgb(rgb, w, min(x, w - 1), min(row, h - 1), r, g, b);
  y[(size_t)row * pw + x] = (uint16_t)clamp255((2449 * r + 4809 * g + 934 * b + kHalf) >> kQ);
}

// Full-resolution chroma (4:4:4).
__global__ void chroma444_kernel(const uint8_t* __restrict__ rgb, int w, int h, int pw, int ph,
                                 uint16_t* __restrict__ cb, uint16_t* __restrict__ cr) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = blockIdx.y;
  if (x >= pw || row >= ph) return;
  int32_t r, g, b;
  load_rgb(rgb, w, min(x, w - 1), min(row, h - 1), r, g, b);
  const int32_t off = 128 << kQ;
  const size_t o = (size_t)row * pw + x;
  cb[o] = (uint16_t)clamp255((-1382 * r - 2714 * g + 4096 * b + off + kHalf) >> kQ);
  cr[o] = (uint16_t)clamp255((4096 * r - 3430 * g - 666 * b + off + kHalf) >> kQ);
}

// 4:2:0 chroma: the unrounded Q13 chroma of the 2x2 quad (last row/column of
// the source repeated), summed, +2^14, >> 15.
__global__ void chroma420_kernel(const uint8_t* __restrict__ rgb, int w, int h, int pcw, int pch,
                                 uint16_t* __restrict__ cb, uint16_t* __restrict__ cr) {
  const int cx = blockIdx.x * blockDim.x + threadIdx.x;
  const int cy = blockIdx.y;
  if (cx >= pcw || cy >= pch) return;
  const int cw = (w + 1) >> 1, ch = (h + 1) >> 1;
  const int sx = min(cx, cw - 1), sy = min(cy, ch - 1);
  const int x0 = 2 * sx, x1 = min(2 * sx + 1, w - 1);
  const int y0 = 2 * sy, y1 = min(2 * sy + 1, h - 1);
  const int32_t off = 128 << kQ;
  int32_t sb = 0, sr = 0;
  const int xs[2] = {x0, x1}, ys[2] = {y0, y1};
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int i = 0; i < 2; i++) {
      int32_t r, g, b;
      load_rgb(rgb, w, xs[i], ys[j], r, g, b);
      sb += -1382 * r - 2714 * g + 4096 * b + off;
      sr += 4096 * r - 3430 * g - 666 * b + off;
    }
  const size_t o = (size_t)cy * pcw + cx;
  cb[o] = (uint16_t)clamp255((sb + (1 << (kQ + 1))) >> (kQ + 2));
  cr[o] = (uint16_t)clamp255((sr + (1 << (kQ + 1))) >> (kQ + 2));
}

int csc_check(int32_t w, int32_t h, int32_t sub) {
  if (w <= 0 || h <= 0 || w > 16383 || h > 16383) return MT_ERR_INVALID_INPUT;
  if (sub != 0 && sub != 2) return MT_ERR_UNSUPPORTED;
  return MT_OK;
}

}  // namespace

extern "C" {

int mt_padded_plane_dims(int32_t w, int32_t h, int32_t sub, int32_t* pw, int32_t* ph, int32_t* pcw, int32_t* pch) {
  int rc = csc_check(w, h, sub);
  if (rc != MT_OK) return rc;
  const int32_t aw = (w + 7) & ~7, ah = (h + 7) & ~7;
  if (pw) *pw = aw;
  if (ph) *ph = ah;
  if (pcw) *pcw = sub == 2 ? aw >> 1 : aw;
  if (pch) *pch = sub == 2 ? ah >> 1 : ah;
  return MT_OK;
}

int mt_csc_rgb8_device(const uint8_t* d_rgb, int32_t w, int32_t h, int32_t sub, uint16_t* d_y, uint16_t* d_cb,
                       uint16_t* d_cr, void* stream) {
  int32_t pw, ph, pcw, pch;
  int rc = mt_padded_plane_dims(w, h, sub, &pw, &ph, &pcw, &pch);
  if (rc != MT_OK) return rc;
  if (!d_rgb || !d_y || !d_cb || !d_cr) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int T = 256;
  luma_kernel<<<dim3((pw + T - 1) / T, ph), T, 0, st>>>(d_rgb, w, h, pw, ph, d_y);
  if (sub == 2)
    chroma420_kernel<<<dim3((pcw + T - 1) / T, pch), T, 0, st>>>(d_rgb, w, h, pcw, pch, d_cb, d_cr);
  else
    chroma444_kernel<<<dim3((pcw + T - 1) / T, pch), T, 0, st>>>(d_rgb, w, h, pcw, pch, d_cb, d_cr);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_csc_rgb8(const uint8_t* rgb, int32_t w, int32_t h, int32_t sub, uint16_t* y, uint16_t* cb, uint16_t* cr) {
  int32_t pw, ph, pcw, pch;
  int rc = mt_padded_plane_dims(w, h, sub, &pw, &ph, &pcw, &pch);
  if (rc != MT_OK) return rc;
  if (!rgb || !y || !cb || !cr) return MT_ERR_INVALID_INPUT;
  const size_t n_rgb = (size_t)w * h * 3, n_y = (size_t)pw * ph, n_c = (size_t)pcw * pch;
  uint8_t* d = nullptr;
  const size_t off_y = (n_rgb + 255) & ~(size_t)255;
  const size_t off_cb = off_y + ((n_y * 2 + 255) & ~(size_t)255);
  const size_t off_cr = off_cb + ((n_c * 2 + 255) & ~(size_t)255);
  const size_t total = off_cr + n_c * 2;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d, rgb, n_rgb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_csc_rgb8_device(d, w, h, sub, (uint16_t*)(d + off_y), (uint16_t*)(d + off_cb), (uint16_t*)(d + off_cr),
                            nullptr);
    if (rc == MT_OK) {
      e = cudaMemcpy(y, d + off_y, n_y * 2, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess) e = cudaMemcpy(cb, d + off_cb, n_c * 2, cudaMemcpyDeviceToHost);
      if (e == cudaSuccess) e = cudaMemcpy(cr, d + off_cr, n_c * 2, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
