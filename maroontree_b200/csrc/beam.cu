// The proxy's mode beam (proxy_mode_beam, src/coder/partition_search.rs:187-238):
// every block's 11 nd_modes predicted and scored by satd_sad_proxy, then sorted
// by (score, mode).
//
// beam_score_kernel: thread t takes mode t / nblocks and block t % nblocks, so
// a warp predicts one mode over 32 blocks (one code path); the prediction and
// the 4x4 Hadamard tiles stay in registers / a small per-thread array.
// beam_sort_kernel: one thread per block sorts its 11 (score, mode) pairs in
// place (insertion sort; scores are exact integers, ties go to the lower mode
// as the reference's sort by the (score, mode) key).
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "common.cuh"
#include "intrapred.cuh"

namespace {

using namespace mtd;

using mtd::clampi;
using mtd::uabs;

constexpr int kBeamModes = MT_BEAM_MODES;
// ND_LUMA_MODES (src/intrapred.rs:1712-1724).
__constant__ uint8_t kNdModes[kBeamModes] = {MT_DC_PRED,    MT_V_PRED,      MT_H_PRED,    MT_D45_PRED,
                                             MT_D135_PRED,  MT_D113_PRED,   MT_D157_PRED, MT_D203_PRED,
                                             MT_D67_PRED,   MT_SMOOTH_PRED, MT_PAETH_PRED};

template <int N>
__global__ void __launch_bounds__(128) beam_score_kernel(const uint16_t* __restrict__ src,
                                                         const uint16_t* __restrict__ rec, const mt_chain_params p,
                                                         const mt_block8* __restrict__ blocks, int nblocks,
                                                         unsigned long long* __restrict__ scores) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = (int)(t / nblocks), b = (int)(t - (long long)k * nblocks);
  if (k >= kBeamModes) return;
  const mt_block8 bk = blocks[b];
  if (bk.px + N > p.frame_w || bk.py + N > p.frame_h) {
    scores[(size_t)b * kBeamModes + k] = ~0ull;
    return;
  }
  int16_t pred[N * N];
  int32_t scratch[3 * mtd::edge_cap<N>()];
  mtd::predict_sq<N>(rec, p.stride, p.frame_w, p.frame_h, bk.px, bk.py, kNdModes[k], 0, bk.flags & 1,
                     (bk.flags >> 1) & 1, (bk.flags >> 2) & 1, p.bd, pred, scratch);
  const int vw = (p.vis_w > 0 ? p.vis_w : p.frame_w) - bk.px, vh = (p.vis_h > 0 ? p.vis_h : p.frame_h) - bk.py;
  scores[(size_t)b * kBeamModes + k] = satd_sad_proxy<N>(src, p.stride, bk.px, bk.py, pred, vw, vh);
}

__global__ void beam_sort_kernel(unsigned long long* __restrict__ scores, uint8_t* __restrict__ modes, int nblocks) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  unsigned long long s[kBeamModes];
  int m[kBeamModes];
#pragma unroll
  for (int k = 0; k < kBeamModes; k++) {
    s[k] = scores[(size_t)b * kBeamModes + k];
    m[k] = kNdModes[k];
  }
  if (s[0] == ~0ull) {  // block outside the frame
#pragma unroll
    for (int k = 0; k < kBeamModes; k++) modes[(size_t)b * kBeamModes + k] = 255;
    return;
  }
  for (int i = 1; i < kBeamModes; i++) {
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
  for (int k = 0; k < kBeamModes; k++) {
    scores[(size_t)b * kBeamModes + k] = s[k];
    modes[(size_t)b * kBeamModes + k] = (uint8_t)m[k];
  }
}

int check(const mt_chain_params* p, int32_t nblocks) {
  if (!p || nblocks < 0) return MT_ERR_INVALID_INPUT;
  if ((p->tx_size != 4 && p->tx_size != 8 && p->tx_size != 16) || p->bd != 8) return MT_ERR_UNSUPPORTED;
  if (p->frame_w <= 0 || p->frame_h <= 0 || p->stride < p->frame_w) return MT_ERR_INVALID_INPUT;
  if ((long long)nblocks * kBeamModes > 0x7fffffffLL) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

int mt_mode_beam_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                        const mt_block8* d_blocks, int32_t nblocks, uint64_t* d_scores, uint8_t* d_modes,
                        void* stream) {
  int rc = check(prm, nblocks);
  if (rc != MT_OK) return rc;
  if (nblocks == 0) return MT_OK;
  if (!d_src || !d_recon || !d_blocks || !d_scores || !d_modes) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long* sc = reinterpret_cast<unsigned long long*>(d_scores);
  const long long total = (long long)nblocks * kBeamModes;
  const unsigned grid = (unsigned)((total + 127) / 128);
  switch (prm->tx_size) {
    case 4: beam_score_kernel<4><<<grid, 128, 0, st>>>(d_src, d_recon, *prm, d_blocks, nblocks, sc); break;
    case 8: beam_score_kernel<8><<<grid, 128, 0, st>>>(d_src, d_recon, *prm, d_blocks, nblocks, sc); break;
    default: beam_score_kernel<16><<<grid, 128, 0, st>>>(d_src, d_recon, *prm, d_blocks, nblocks, sc); break;
  }
  beam_sort_kernel<<<(nblocks + 127) / 128, 128, 0, st>>>(sc, d_modes, nblocks);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_mode_beam(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_block8* blocks,
                 int32_t nblocks, uint64_t* scores, uint8_t* modes) {
  int rc = check(prm, nblocks);
  if (rc != MT_OK) return rc;
  if (nblocks == 0) return MT_OK;
  if (!src || !recon || !blocks || !modes) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)prm->stride * prm->frame_h * sizeof(uint16_t);
  const size_t nsc = (size_t)nblocks * kBeamModes;
  const size_t o_src = 0, o_rec = up256(plane), o_blk = o_rec + up256(plane);
  const size_t o_sc = o_blk + up256((size_t)nblocks * sizeof(mt_block8)), o_md = o_sc + up256(nsc * 8);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_md + up256(nsc)) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_src, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_rec, recon, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_blk, blocks, (size_t)nblocks * sizeof(mt_block8), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_mode_beam_device(reinterpret_cast<const uint16_t*>(d + o_src), reinterpret_cast<const uint16_t*>(d + o_rec),
                             prm, reinterpret_cast<const mt_block8*>(d + o_blk), nblocks,
                             reinterpret_cast<uint64_t*>(d + o_sc), d + o_md, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(modes, d + o_md, nsc, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && scores) e = cudaMemcpy(scores, d + o_sc, nsc * 8, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
