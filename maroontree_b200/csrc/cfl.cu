// Chroma-from-luma alpha search over a batch of chroma blocks
// (cfl_ac_sub / cfl_ac_444 and cfl_best_alpha, src/intrapred.rs:1112-1258).
//
// One warp per block, four blocks per CTA.  The lanes stride over the block's
// samples: the AC (luma sums scaled to the <<3 range) goes to the warp's
// shared-memory slice, the block sum, num / den and every candidate's SSE are
// 64-bit integer sums reduced across the warp -- integers, so the reduction
// order cannot change them.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"

namespace {

using namespace mtd;

constexpr int kCflWarps = 4;
constexpr int kCflMaxSamples = 32 * 32;

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(32 * kCflWarps) cfl_kernel(
    const uint16_t* __restrict__ luma, int luma_stride, const uint16_t* __restrict__ src_u,
    const uint16_t* __restrict__ src_v, int chroma_stride, int sub_x, int sub_y, int lcw, int lch, int vis_cw,
    int vis_ch, int maxv, const mt_cfl_block* __restrict__ blocks, int n, int8_t* __restrict__ alpha,
    int32_t* __restrict__ ac_out) {
  __shared__ int32_t s_ac[kCflWarps][kCflMaxSamples];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kCflWarps + warp;
  if (b >= n) return;  // whole warps leave together
  const int cw = 1 << lcw, ch = 1 << lch, ns = cw * ch, log2sz = lcw + lch;
  const mt_cfl_block bk = blocks[b];
  const int cx = bk.cx, cy = bk.cy;
  const int shift = 1 + (sub_y ? 0 : 1) + (sub_x ? 0 : 1);
  const uint16_t* l = luma + (size_t)(cy << sub_y) * luma_stride + (cx << sub_x);
  int32_t* ac = s_ac[warp];
  long long sum = 0;
  for (int i = lane; i < ns; i += 32) {
    const int y = i >> lcw, x = i & (cw - 1);
    const uint16_t* p = l + (size_t)(y << sub_y) * luma_stride + (x << sub_x);
    int32_t s = p[0];
    if (sub_x) s += p[1];
    if (sub_y) {
      s += p[luma_stride];
      if (sub_x) s += p[luma_stride + 1];
    }
    s <<= shift;
    ac[i] = s;
    sum += s;
  }
  sum = warp_sum64(sum) + ((1LL << log2sz) >> 1);
  const int32_t mean = (int32_t)(sum >> log2sz);
  for (int i = lane; i < ns; i += 32) {
    const int32_t v = ac[i] - mean;
    ac[i] = v;
    if (ac_out) ac_out[(size_t)b * ns + i] = v;
  }
  __syncwarp();
  const int vw = min(max(vis_cw - cx, 0), cw), vh = min(max(vis_ch - cy, 0), ch);
  for (int pl = 0; pl < 2; pl++) {
    const uint16_t* s = (pl ? src_v : src_u) + (size_t)cy * chroma_stride + cx;
    const int32_t dc = bk.dc[pl];
    long long num = 0, den = 0;
    for (int i = lane; i < ns; i += 32) {
      const int y = i >> lcw, x = i & (cw - 1);
      if (x < vw && y < vh) {
        const long long a = ac[i];
        num += (long long)((int32_t)s[(size_t)y * chroma_stride + x] - dc) * a;
        den += a * a;
      }
    }
    num = warp_sum64(num);
    den = warp_sum64(den);
    int best_a = 0;
    if (den != 0) {
      const long long sg = num > 0 ? 1 : (num < 0 ? -1 : 0);
      long long a0 = (64 * num + (den >> 1) * sg) / den;
      a0 = a0 < -16 ? -16 : (a0 > 16 ? 16 : a0);
      long long best_e = 0x7fffffffffffffffLL;
      for (int cand = (int)a0 - 3; cand <= (int)a0 + 3; cand++) {
        if (cand < -16 || cand > 16) continue;
        long long e = 0;
        for (int i = lane; i < ns; i += 32) {
          const int y = i >> lcw, x = i & (cw - 1);
          if (x < vw && y < vh) {
            const long long d = (int32_t)s[(size_t)y * chroma_stride + x] - cfl_pred_pixel(dc, ac[i], cand, maxv);
            e += d * d;
          }
        }
        e = warp_sum64(e);
        if (e < best_e) {
          best_e = e;
          best_a = cand;
        }
      }
    }
    if (lane == 0) alpha[2 * b + pl] = (int8_t)best_a;
  }
}

int log2_dim(int v) {
  switch (v) {
    case 4: return 2;
    case 8: return 3;
    case 16: return 4;
    case 32: return 5;
  }
  return -1;
}

int check(int32_t luma_stride, int32_t chroma_stride, int32_t sub_x, int32_t sub_y, int32_t cw, int32_t ch,
          int32_t vis_cw, int32_t vis_ch, int32_t bd, int32_t n) {
  if (n < 0 || luma_stride <= 0 || chroma_stride <= 0 || vis_cw < 0 || vis_ch < 0) return MT_ERR_INVALID_INPUT;
  if (log2_dim(cw) < 0 || log2_dim(ch) < 0) return MT_ERR_INVALID_INPUT;
  if (sub_x < 0 || sub_x > 1 || sub_y < 0 || sub_y > 1 || (sub_y && !sub_x)) return MT_ERR_UNSUPPORTED;
  if (bd != 8 && bd != 10 && bd != 12) return MT_ERR_UNSUPPORTED;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int mt_cfl_alpha_device(const uint16_t* d_luma, int32_t luma_stride, const uint16_t* d_src_u, const uint16_t* d_src_v,
                        int32_t chroma_stride, int32_t sub_x, int32_t sub_y, int32_t cw, int32_t ch, int32_t vis_cw,
                        int32_t vis_ch, int32_t bd, const mt_cfl_block* d_blocks, int32_t n, int8_t* d_alpha,
                        int32_t* d_ac, void* stream) {
  const int rc = check(luma_stride, chroma_stride, sub_x, sub_y, cw, ch, vis_cw, vis_ch, bd, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_luma || !d_src_u || !d_src_v || !d_blocks || !d_alpha) return MT_ERR_INVALID_INPUT;
  const int vcw = vis_cw > 0 ? vis_cw : 0x7fffffff, vch = vis_ch > 0 ? vis_ch : 0x7fffffff;
  cfl_kernel<<<(unsigned)((n + kCflWarps - 1) / kCflWarps), 32 * kCflWarps, 0,
               reinterpret_cast<cudaStream_t>(stream)>>>(d_luma, luma_stride, d_src_u, d_src_v, chroma_stride, sub_x,
                                                         sub_y, log2_dim(cw), log2_dim(ch), vcw, vch, (1 << bd) - 1,
                                                         d_blocks, n, d_alpha, d_ac);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_cfl_alpha(const uint16_t* luma, int32_t luma_stride, int32_t luma_h, const uint16_t* src_u,
                 const uint16_t* src_v, int32_t chroma_stride, int32_t chroma_h, int32_t sub_x, int32_t sub_y,
                 int32_t cw, int32_t ch, int32_t vis_cw, int32_t vis_ch, int32_t bd, const mt_cfl_block* blocks,
                 int32_t n, int8_t* alpha, int32_t* ac) {
  int rc = check(luma_stride, chroma_stride, sub_x, sub_y, cw, ch, vis_cw, vis_ch, bd, n);
  if (rc != MT_OK) return rc;
  if (luma_h <= 0 || chroma_h <= 0) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  if (!luma || !src_u || !src_v || !blocks || !alpha) return MT_ERR_INVALID_INPUT;
  // every block's luma and chroma samples must lie inside the planes
  for (int32_t b = 0; b < n; b++) {
    if ((blocks[b].cx + cw) << sub_x > luma_stride || (blocks[b].cy + ch) << sub_y > luma_h) return MT_ERR_INVALID_INPUT;
    if (blocks[b].cx + cw > chroma_stride || blocks[b].cy + ch > chroma_h) return MT_ERR_INVALID_INPUT;
  }
  const size_t lp = (size_t)luma_stride * luma_h * 2, cp = (size_t)chroma_stride * chroma_h * 2;
  const size_t o_l = 0, o_u = up256(lp), o_v = o_u + up256(cp), o_b = o_v + up256(cp);
  const size_t o_a = o_b + up256((size_t)n * sizeof(mt_cfl_block)), o_ac = o_a + up256((size_t)n * 2);
  const size_t total = o_ac + (ac ? up256((size_t)n * cw * ch * 4) : 0);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, total) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_l, luma, lp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_u, src_u, cp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_v, src_v, cp, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_b, blocks, (size_t)n * sizeof(mt_cfl_block), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_cfl_alpha_device(reinterpret_cast<const uint16_t*>(d + o_l), luma_stride,
                             reinterpret_cast<const uint16_t*>(d + o_u), reinterpret_cast<const uint16_t*>(d + o_v),
                             chroma_stride, sub_x, sub_y, cw, ch, vis_cw, vis_ch, bd,
                             reinterpret_cast<const mt_cfl_block*>(d + o_b), n, reinterpret_cast<int8_t*>(d + o_a),
                             ac ? reinterpret_cast<int32_t*>(d + o_ac) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(alpha, d + o_a, (size_t)n * 2, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && ac) e = cudaMemcpy(ac, d + o_ac, (size_t)n * cw * ch * 4, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
