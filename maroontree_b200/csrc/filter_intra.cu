// Recursive filter-intra prediction and the Slow search's filter-intra
// shortlist ranking (rank_filter_intra_modes, src/coder/superblock.rs:356-400)
// over a batch of blocks.
//
// fi_score_kernel: thread t predicts mode t / n of block t % n (mode-major, so
// a warp runs one tap set over 32 blocks) into a per-thread (h+1) x (w+1)
// int16 grid -- row 0 the above edge, column 0 the left edge -- filling 4x2
// cells in raster order, each from the seven samples above and to its left
// (filter_intra_predict_impl / scalar_filter_intra_cells,
// src/intrapred.rs:473-565), then scores it with satd_sad_proxy
// (src/rd_sse.rs:1143-1176).  fi_sort_kernel orders each block's five
// (score, mode) pairs.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"
#include "common.cuh"

namespace {

using mtd::uabs;

constexpr int kFiModes = MT_FILTER_INTRA_MODES;
__constant__ int8_t kFiTaps[5 * 8 * 7] = {MT_INTRA_FILTER_TAPS_LIST};

__global__ void __launch_bounds__(128) fi_score_kernel(const uint16_t* __restrict__ src,
                                                       const uint16_t* __restrict__ rec, int stride, int fw, int fh,
                                                       int vis_w, int vis_h, int bd, int w, int h,
                                                       const uint16_t* __restrict__ pos, int n,
                                                       unsigned long long* __restrict__ scores,
                                                       int16_t* __restrict__ preds) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int m = (int)(t / n), b = (int)(t - (long long)m * n);
  if (m >= kFiModes) return;
  const int px = pos[2 * b], py = pos[2 * b + 1];
  if (px + w > fw || py + h > fh) {
    scores[(size_t)b * kFiModes + m] = ~0ull;
    return;
  }
  int16_t g[33 * 33];
  const int gs = w + 1;  // grid stride
  const int32_t base = 1 << (bd - 1), mx = (1 << bd) - 1;
  const bool top = py > 0, left = px > 0;
  const uint16_t* up = rec + (size_t)(py - 1) * stride + px;  // read only when top
  const uint16_t* lf = rec + (size_t)py * stride + px - 1;    // read only when left
  g[0] = (int16_t)(top ? (left ? up[-1] : up[0]) : (left ? lf[0] : base));
  for (int x = 0; x < w; x++) g[1 + x] = (int16_t)(top ? up[x] : (left ? lf[0] : base - 1));
  for (int y = 0; y < h; y++) g[(y + 1) * gs] = (int16_t)(left ? lf[(size_t)y * stride] : (top ? up[0] : base + 1));
  const int8_t* taps = kFiTaps + m * 56;
  for (int r = 1; r <= h; r += 2)
    for (int c = 1; c <= w; c += 4) {
      const int16_t* a = g + (r - 1) * gs + c - 1;
      const int32_t p0 = a[0], p1 = a[1], p2 = a[2], p3 = a[3], p4 = a[4];
      const int32_t p5 = g[r * gs + c - 1], p6 = g[(r + 1) * gs + c - 1];
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const int8_t* f = taps + k * 7;
        const int32_t sum = f[0] * p0 + f[1] * p1 + f[2] * p2 + f[3] * p3 + f[4] * p4 + f[5] * p5 + f[6] * p6;
        g[(r + (k >> 2)) * gs + c + (k & 3)] = (int16_t)mtd::clampi((sum + 8) >> 4, 0, mx);
      }
    }
  if (preds) {
    int16_t* o = preds + ((size_t)b * kFiModes + m) * w * h;
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) o[y * w + x] = g[(y + 1) * gs + x + 1];
  }
  // satd_sad_proxy with the samples past the displayed window taken as the
  // prediction.
  const int vw = (vis_w > 0 ? vis_w : fw) - px, vh = (vis_h > 0 ? vis_h : fh) - py;
  unsigned long long sad = 0, satd = 0;
  for (int ty = 0; ty < h; ty += 4)
    for (int tx = 0; tx < w; tx += 4) {
      int32_t rr[4][4];
#pragma unroll
      for (int y = 0; y < 4; y++) {
        int32_t d[4];
#pragma unroll
        for (int x = 0; x < 4; x++) {
          const bool vis = tx + x < vw && ty + y < vh;
          d[x] = vis ? (int32_t)src[(size_t)(py + ty + y) * stride + px + tx + x] - g[(ty + y + 1) * gs + tx + x + 1]
                     : 0;
          sad += uabs(d[x]);
        }
        const int32_t e = d[0] + d[2], f = d[0] - d[2], gg = d[1] + d[3], hh = d[1] - d[3];
        rr[y][0] = e + gg;
        rr[y][1] = f + hh;
        rr[y][2] = f - hh;
        rr[y][3] = e - gg;
      }
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int32_t e = rr[0][x] + rr[2][x], f = rr[0][x] - rr[2][x], gg = rr[1][x] + rr[3][x],
                      hh = rr[1][x] - rr[3][x];
        satd += (unsigned long long)uabs(e + gg) + uabs(f + hh) + uabs(f - hh) + uabs(e - gg);
      }
    }
  scores[(size_t)b * kFiModes + m] = sad + (satd >> 2);
}

// Per block: sort the five (score, mode order) pairs ascending (insertion sort
// on the exact integer key, ties to the lower mode).
__global__ void fi_sort_kernel(unsigned long long* __restrict__ scores, uint8_t* __restrict__ modes, int n) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  unsigned long long s[kFiModes];
  int m[kFiModes];
#pragma unroll
  for (int k = 0; k < kFiModes; k++) {
    s[k] = scores[(size_t)b * kFiModes + k];
    m[k] = k;
  }
  if (s[0] == ~0ull) {
#pragma unroll
    for (int k = 0; k < kFiModes; k++) modes[(size_t)b * kFiModes + k] = 255;
    return;
  }
  for (int i = 1; i < kFiModes; i++) {
    const unsigned long long vs = s[i];
    const int vm = m[i];
    int j = i - 1;
    while (j >= 0 && (s[j] > vs || (s[j] == vs && m[j] > vm))) {
      s[j + 1] = s[j];
      m[j + 1] = m[j];
      j--;
    }
    s[j + 1] = vs;
    m[j + 1] = vm;
  }
  for (int k = 0; k < kFiModes; k++) {
    scores[(size_t)b * kFiModes + k] = s[k];
    modes[(size_t)b * kFiModes + k] = (uint8_t)m[k];
  }
}

bool dim_ok(int v) { return v == 4 || v == 8 || v == 16 || v == 32; }

int check(int32_t stride, int32_t fw, int32_t fh, int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h,
          int32_t n) {
  if (n < 0 || fw <= 0 || fh <= 0 || stride < fw || vis_w < 0 || vis_h < 0) return MT_ERR_INVALID_INPUT;
  if (!dim_ok(w) || !dim_ok(h)) return MT_ERR_INVALID_INPUT;
  if (bd != 8 && bd != 10 && bd != 12) return MT_ERR_UNSUPPORTED;
  if ((long long)n * kFiModes > 0x7fffffffLL) return MT_ERR_TOO_LARGE;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int mt_filter_intra_beam_device(const uint16_t* d_src, const uint16_t* d_recon, int32_t stride, int32_t frame_w,
                                int32_t frame_h, int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h,
                                const uint16_t* d_pos, int32_t n, uint64_t* d_scores, uint8_t* d_modes,
                                int16_t* d_preds, void* stream) {
  const int rc = check(stride, frame_w, frame_h, vis_w, vis_h, bd, w, h, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_recon || !d_pos || !d_scores || !d_modes) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long* sc = reinterpret_cast<unsigned long long*>(d_scores);
  const long long total = (long long)n * kFiModes;
  fi_score_kernel<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(d_src, d_recon, stride, frame_w, frame_h, vis_w,
                                                                   vis_h, bd, w, h, d_pos, n, sc, d_preds);
  fi_sort_kernel<<<(n + 127) / 128, 128, 0, st>>>(sc, d_modes, n);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_filter_intra_beam(const uint16_t* src, const uint16_t* recon, int32_t stride, int32_t frame_w, int32_t frame_h,
                         int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h, const uint16_t* pos,
                         int32_t n, uint64_t* scores, uint8_t* modes, int16_t* preds) {
  int rc = check(stride, frame_w, frame_h, vis_w, vis_h, bd, w, h, n);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !recon || !pos || !modes) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)stride * frame_h * 2, nsc = (size_t)n * kFiModes;
  const size_t npred = preds ? nsc * w * h * 2 : 0;
  const size_t o_src = 0, o_rec = up256(plane), o_pos = o_rec + up256(plane), o_sc = o_pos + up256((size_t)n * 4);
  const size_t o_md = o_sc + up256(nsc * 8), o_pr = o_md + up256(nsc);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_pr + up256(npred)) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_pos, pos, (size_t)n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_filter_intra_beam_device(reinterpret_cast<const uint16_t*>(d + o_src),
                                     reinterpret_cast<const uint16_t*>(d + o_rec), stride, frame_w, frame_h, vis_w,
                                     vis_h, bd, w, h, reinterpret_cast<const uint16_t*>(d + o_pos), n,
                                     reinterpret_cast<uint64_t*>(d + o_sc), d + o_md,
                                     preds ? reinterpret_cast<int16_t*>(d + o_pr) : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(modes, d + o_md, nsc, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && scores) e = cudaMemcpy(scores, d + o_sc, nsc * 8, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && preds) e = cudaMemcpy(preds, d + o_pr, npred, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
