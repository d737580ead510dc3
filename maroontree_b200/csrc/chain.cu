// Kernels of the batched 8x8 luma candidate chain.
//
//  * chain8_kernel: an arbitrary candidate list.  The launcher first buckets
//    the candidates by (transform type, mode, angle delta) into a permutation
//    (counting sort, 3 small kernels) so that each warp runs one code path.
//  * level8_kernel: one whole RDO level -- every (block, combo) pair of a block
//    list and a combo list (mode, angle delta, transform type), enumerated so a
//    warp holds one combo over 32 consecutive blocks -- with the per-block
//    argmin under the reference's comparison (strict <, first in evaluation
//    order wins) folded in through a 64-bit atomicMin on (cost bits, combo).
//  * stage kernels (forward, inverse, trellis, prediction) for the
//    kernel-level entry points.
#include <cuda_runtime.h>
#include <stdint.h>

#include "chain16.cuh"
#include "chain4.cuh"
#include "chain8.cuh"

namespace mtd {

struct ChainArgs {
  mt_chain_params p;
  mt_quant q;
  float trellis_lambda;  // scaled_trellis_lambda(dc_q, ac_q, lambda0), computed on the host
  int has_qm;
};

constexpr int kThreads = 128;
// Minimum resident CTAs per SM requested from the register allocator.
#ifndef MT_CHAIN_MIN_BLOCKS
#define MT_CHAIN_MIN_BLOCKS 3
#endif
constexpr int kMinBlocks = MT_CHAIN_MIN_BLOCKS;
constexpr int kBuckets = 1024;
constexpr int kLevelMaxCombos = MT_LEVEL_MAX_COMBOS;

__device__ __forceinline__ int bucket_of(const mt_candidate& c) {
  const int t = min((int)c.tx_type, 7), m = min((int)c.mode, 15), d = min(max(c.angle_delta + 3, 0), 7);
  return (t * 16 + m) * 8 + d;
}

__global__ void bucket_count_kernel(const mt_candidate* __restrict__ cands, int n, int* __restrict__ hist) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&hist[bucket_of(cands[i])], 1);
}
// Exclusive scan of the 1024 bucket counts into the scatter cursors (one CTA).
__global__ void bucket_scan_kernel(const int* __restrict__ hist, int* __restrict__ cursor) {
  __shared__ int s[kBuckets];
  const int t = threadIdx.x;  // 1024 threads
  s[t] = hist[t];
  __syncthreads();
  for (int off = 1; off < kBuckets; off <<= 1) {
    const int v = t >= off ? s[t - off] : 0;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  cursor[t] = s[t] - hist[t];
}
__global__ void bucket_scatter_kernel(const mt_candidate* __restrict__ cands, int n, int* __restrict__ cursor,
                                      int* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[atomicAdd(&cursor[bucket_of(cands[i])], 1)] = i;
}

__device__ __forceinline__ void stage_tables(const mt_coef_costs* __restrict__ costs, const uint8_t* __restrict__ qm_row,
                                             int has_qm, mt_coef_costs& sC, uint8_t* sQm, float* sQs, float* sLut) {
  const float* g = reinterpret_cast<const float*>(costs);
  float* s = reinterpret_cast<float*>(&sC);
  for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
  if (threadIdx.x < 64) {
    const int w = has_qm ? qm_row[threadIdx.x] : 32;
    sQm[threadIdx.x] = (uint8_t)w;
    sQs[threadIdx.x] = fwd_qm_scale(w);
    sLut[threadIdx.x] = kCoefRateLut[threadIdx.x];
  }
  __syncthreads();
}

__device__ __forceinline__ void store_blocks(Work8& w, int32_t maxv, int32_t* lv_out, int32_t* rec_out, size_t slot) {
  const int16_t* cf = w.cf();
  const int16_t* pred = w.pred();
  const int16_t* rr = w.rr();
  if (lv_out) {
    int4* o = reinterpret_cast<int4*>(lv_out + slot * 64);
#pragma unroll
    for (int i = 0; i < 16; i++) o[i] = make_int4(cf[4 * i], cf[4 * i + 1], cf[4 * i + 2], cf[4 * i + 3]);
  }
  if (rec_out) {
    int4* o = reinterpret_cast<int4*>(rec_out + slot * 64);
#pragma unroll
    for (int i = 0; i < 16; i++)
      o[i] = make_int4(clampi(pred[4 * i] + rr[4 * i], 0, maxv), clampi(pred[4 * i + 1] + rr[4 * i + 1], 0, maxv),
                       clampi(pred[4 * i + 2] + rr[4 * i + 2], 0, maxv),
                       clampi(pred[4 * i + 3] + rr[4 * i + 3], 0, maxv));
  }
}

template <bool VIS>
__global__ void __launch_bounds__(kThreads, kMinBlocks) chain8_kernel(const uint16_t* __restrict__ src,
                                                          const uint16_t* __restrict__ rec, ChainArgs a,
                                                          const uint8_t* __restrict__ qm_row,
                                                          const mt_coef_costs* __restrict__ costs,
                                                          const mt_candidate* __restrict__ cands,
                                                          const int* __restrict__ perm, int n,
                                                          mt_candidate_result* __restrict__ res,
                                                          int32_t* __restrict__ lv_out, int32_t* __restrict__ rec_out) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  __shared__ float sLut[64];
  stage_tables(costs, qm_row, a.has_qm, sC, sQm, sQs, sLut);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int idx = perm ? perm[t] : t;
  const mt_candidate cd = cands[idx];
  if (!cand_ok(cd, a.p.frame_w, a.p.frame_h)) {
    mt_candidate_result bad = {};
    bad.eob = MT_EOB_INVALID;
    res[idx] = bad;
    return;
  }
  int32_t store[kWork8Words];
  Work8 w{store};
  mt_candidate_result r;
  chain8_one<VIS>(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
  res[idx] = r;
  store_blocks(w, (1 << a.p.bd) - 1, lv_out, rec_out, (size_t)idx);
}

// A level runs in three kernels.  Consecutive combos that share (mode, angle
// delta) form a run; the prediction depends on the run only, so
//   level8_runs_kernel  finds the runs (one thread),
//   level8_pred_kernel  predicts each (run, block) once into an 8-bit buffer
//                       (64 B per item, L2-resident for a 1080p level),
//   level8_kernel       evaluates the rest of every candidate chain: thread t
//                       takes combo t / nblocks and block t % nblocks, so a
//                       warp -- and nearly the whole device at any moment --
//                       runs one transform type's code path over 32
//                       consecutive blocks; the per-block argmin folds in
//                       through a 64-bit atomicMin on (cost bits, combo).
struct LevelRuns {
  int nruns;
  int16_t start[kLevelMaxCombos + 1];  // run r covers combos [start[r], start[r + 1])
  int16_t run_of[kLevelMaxCombos];
};

__global__ void level8_runs_kernel(const mt_combo* __restrict__ combos, int ncombos, LevelRuns* __restrict__ runs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int nr = 0;
  for (int c = 0; c < ncombos; c++) {
    if (c == 0 || combos[c].mode != combos[c - 1].mode || combos[c].angle_delta != combos[c - 1].angle_delta)
      runs->start[nr++] = (int16_t)c;
    runs->run_of[c] = (int16_t)(nr - 1);
  }
  runs->start[nr] = (int16_t)ncombos;
  runs->nruns = nr;
}

__device__ __forceinline__ mt_candidate level_candidate(const mt_block8& bk, const mt_combo& cb) {
  mt_candidate cd;
  cd.px = bk.px;
  cd.py = bk.py;
  cd.mode = cb.mode;
  cd.angle_delta = cb.angle_delta;
  cd.tx_type = cb.tx_type;
  cd.flags = (uint8_t)((bk.flags & ~MT_CAND_NO_TRELLIS) | ((cb.flags & MT_COMBO_NO_TRELLIS) ? MT_CAND_NO_TRELLIS : 0));
  cd.dcs_ctx = bk.dcs_ctx;
  cd.skip_ctx = bk.skip_ctx;
  cd.reserved = 0;
  cd.mode_bits = cb.mode <= MT_PAETH_PRED ? bk.mode_bits[cb.mode] : 0.0f;
  cd.extra_bits = cb.bits;
  return cd;
}

// One (run, block) prediction per thread; items past the run count exit.
__global__ void __launch_bounds__(kThreads) level8_pred_kernel(const uint16_t* __restrict__ rec, ChainArgs a,
                                                               const mt_block8* __restrict__ blocks, int nblocks,
                                                               const mt_combo* __restrict__ combos,
                                                               const LevelRuns* __restrict__ runs,
                                                               uint4* __restrict__ preds) {
  const long long wi = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (wi >= (long long)runs->nruns * nblocks) return;
  const int r = (int)(wi / nblocks), b = (int)(wi - (long long)r * nblocks);
  mt_candidate cd = level_candidate(blocks[b], combos[runs->start[r]]);
  cd.tx_type = 0;  // every check but the transform type's
  if (!cand_ok(cd, a.p.frame_w, a.p.frame_h)) return;
  int32_t store[kWork8Words];
  Work8 w{store};
  chain8_predict(rec, a.p, cd, w);
  const int16_t* pr = w.pred();
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int o = k * 16 + j * 4;
      v[j] = (uint32_t)(uint8_t)pr[o] | ((uint32_t)(uint8_t)pr[o + 1] << 8) | ((uint32_t)(uint8_t)pr[o + 2] << 16) |
             ((uint32_t)(uint8_t)pr[o + 3] << 24);
    }
    preds[wi * 4 + k] = make_uint4(v[0], v[1], v[2], v[3]);
  }
}

template <bool VIS>
__global__ void __launch_bounds__(kThreads, kMinBlocks) level8_kernel(const uint16_t* __restrict__ src, ChainArgs a,
                                                          const uint8_t* __restrict__ qm_row,
                                                          const mt_coef_costs* __restrict__ costs,
                                                          const mt_block8* __restrict__ blocks, int nblocks,
                                                          const mt_combo* __restrict__ combos, int ncombos,
                                                          const LevelRuns* __restrict__ runs,
                                                          const uint4* __restrict__ preds,
                                                          mt_candidate_result* __restrict__ res,
                                                          unsigned long long* __restrict__ best_key) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[64];
  __shared__ float sQs[64];
  __shared__ float sLut[64];
  stage_tables(costs, qm_row, a.has_qm, sC, sQm, sQs, sLut);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(t / nblocks), b = (int)(t - (long long)c * nblocks);
  if (c >= ncombos) return;
  const mt_candidate cd = level_candidate(blocks[b], combos[c]);
  const size_t slot = (size_t)c * nblocks + b;
  if (!cand_ok(cd, a.p.frame_w, a.p.frame_h)) {
    mt_candidate_result bad = {};
    bad.eob = MT_EOB_INVALID;
    res[slot] = bad;
    return;
  }
  int32_t store[kWork8Words];
  Work8 w{store};
  {
    const uint4* pp = preds + ((size_t)runs->run_of[c] * nblocks + b) * 4;
    int16_t* pr = w.pred();
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint4 q = pp[k];
      const uint32_t v[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
        for (int i = 0; i < 4; i++) pr[k * 16 + j * 4 + i] = (int16_t)((v[j] >> (8 * i)) & 0xff);
    }
  }
  mt_candidate_result r;
  chain8_tx<VIS>(src, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
  res[slot] = r;
  // Costs are non-negative finite floats, so their bit patterns order like
  // the values; ties go to the lower combo index (evaluated first in the
  // reference's loop).
  const unsigned long long key = ((unsigned long long)__float_as_uint(r.cost) << 32) | (unsigned)c;
  atomicMin(&best_key[b], key);
}

// The batched 4x4 level: thread t takes combo t / nblocks and block t % nblocks
// (a warp runs one combo over 32 consecutive blocks); prediction per
// candidate (a 4x4 prediction is a few dozen operations).
// 8 resident CTAs per SM requested (80 registers): measured 5 % faster than
// the register allocator's free choice.
template <bool VIS>
__global__ void __launch_bounds__(kThreads, 8) level4_kernel(const uint16_t* __restrict__ src,
                                                          const uint16_t* __restrict__ rec, ChainArgs a,
                                                          const uint8_t* __restrict__ qm_row,
                                                          const mt_coef_costs* __restrict__ costs,
                                                          const mt_block8* __restrict__ blocks, int nblocks,
                                                          const mt_combo* __restrict__ combos, int ncombos,
                                                          mt_candidate_result* __restrict__ res,
                                                          unsigned long long* __restrict__ best_key) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[16];
  __shared__ float sQs[16];
  __shared__ float sLut[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sC);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    if (threadIdx.x < 16) {
      const int w = a.has_qm ? qm_row[threadIdx.x] : 32;
      sQm[threadIdx.x] = (uint8_t)w;
      sQs[threadIdx.x] = fwd_qm_scale(w);
    }
    if (threadIdx.x < 64) sLut[threadIdx.x] = kCoefRateLut[threadIdx.x];
    __syncthreads();
  }
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(t / nblocks), b = (int)(t - (long long)c * nblocks);
  if (c >= ncombos) return;
  const mt_candidate cd = level_candidate(blocks[b], combos[c]);
  const size_t slot = (size_t)c * nblocks + b;
  if (!cand4_ok(cd, a.p.frame_w, a.p.frame_h)) {
    mt_candidate_result bad = {};
    bad.eob = MT_EOB_INVALID;
    res[slot] = bad;
    return;
  }
  int32_t store[kWork4Words];
  Work4 w{store};
  mt_candidate_result r;
  chain4_one<VIS>(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
  res[slot] = r;
  const unsigned long long key = ((unsigned long long)__float_as_uint(r.cost) << 32) | (unsigned)c;
  atomicMin(&best_key[b], key);
}

// The batched 16x16 level: thread t takes combo t / nblocks and block t %
// nblocks, the whole chain per thread (prediction included) in a 3.6 KB
// per-thread arena; the 256 QM weights and their forward scales are staged in
// shared memory.
// Full occupancy requested (16 CTAs of 128 threads, 32 registers): the kernel
// waits on its local-memory arena, and more resident warps hide that better
// (2.61 -> 2.26 ms on the 1080p level; a cap of 2-4 CTAs was slower).
template <bool VIS>
__global__ void __launch_bounds__(kThreads, 16) level16_kernel(const uint16_t* __restrict__ src,
                                                           const uint16_t* __restrict__ rec, ChainArgs a,
                                                           const uint8_t* __restrict__ qm_row,
                                                           const mt_coef_costs* __restrict__ costs,
                                                           const mt_block8* __restrict__ blocks, int nblocks,
                                                           const mt_combo* __restrict__ combos, int ncombos,
                                                           mt_candidate_result* __restrict__ res,
                                                           unsigned long long* __restrict__ best_key) {
  __shared__ mt_coef_costs sC;
  __shared__ uint8_t sQm[256];
  __shared__ float sQs[256];
  __shared__ float sLut[64];
  {
    const float* g = reinterpret_cast<const float*>(costs);
    float* s = reinterpret_cast<float*>(&sC);
    for (int i = threadIdx.x; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) s[i] = g[i];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
      const int w = a.has_qm ? qm_row[i] : 32;
      sQm[i] = (uint8_t)w;
      sQs[i] = fwd_qm_scale(w);
    }
    if (threadIdx.x < 64) sLut[threadIdx.x] = kCoefRateLut[threadIdx.x];
    __syncthreads();
  }
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int c = (int)(t / nblocks), b = (int)(t - (long long)c * nblocks);
  if (c >= ncombos) return;
  const mt_candidate cd = level_candidate(blocks[b], combos[c]);
  const size_t slot = (size_t)c * nblocks + b;
  if (!cand16_ok(cd, a.p.frame_w, a.p.frame_h)) {
    mt_candidate_result bad = {};
    bad.eob = MT_EOB_INVALID;
    res[slot] = bad;
    return;
  }
  int32_t store[kWork16Words];
  Work16 w{store};
  mt_candidate_result r;
  chain16_one<VIS>(src, rec, a.p, a.q, a.trellis_lambda, a.has_qm ? sQm : nullptr, sQs, sLut, sC, cd, r, w);
  res[slot] = r;
  const unsigned long long key = ((unsigned long long)__float_as_uint(r.cost) << 32) | (unsigned)c;
  atomicMin(&best_key[b], key);
}

__global__ void level8_finalize_kernel(const unsigned long long* __restrict__ best_key, int nblocks,
                                       const mt_candidate_result* __restrict__ res, mt_block_best* __restrict__ best) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const unsigned long long k = best_key[b];
  mt_block_best o = {};
  if (k == ~0ull) {
    o.combo = -1;
    o.eob = MT_EOB_INVALID;
  } else {
    const int c = (int)(k & 0xffffffffu);
    const mt_candidate_result r = res[(size_t)c * nblocks + b];
    o.combo = c;
    o.cost = r.cost;
    o.distortion = r.distortion;
    o.bits = r.bits;
    o.satd = r.satd;
    o.eob = r.eob;
  }
  best[b] = o;
}

// Standalone stage kernels, one block per thread.
__global__ void fwd8_kernel(const int32_t* __restrict__ resid, const uint8_t* __restrict__ types, int n, mt_quant q,
                            const uint8_t* __restrict__ qm_row, int32_t* __restrict__ levels,
                            float* __restrict__ targets) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int32_t store[kWork8Words + 64];
  Work8 w{store};
  int32_t* r = w.w + 64;   // int32 residual at [64, 128)
  int32_t* cf = w.w + 128; // int32 levels at [128, 192)
  float* tf = w.tf();
  for (int i = 0; i < 64; i++) r[i] = resid[(size_t)idx * 64 + i];
  const int tx = types[idx];
  fwd8x8(r, tx, q, cf, tf, store + kWork8Words);
  if (qm_row && (tx == MT_TX_DCT_DCT || tx >= MT_TX_ADST_ADST)) {
    float qs[64];
    for (int i = 0; i < 64; i++) qs[i] = fwd_qm_scale(qm_row[i]);
    apply_qm(cf, tf, qs, 64);
  }
  for (int i = 0; i < 64; i++) {
    levels[(size_t)idx * 64 + i] = cf[i];
    targets[(size_t)idx * 64 + i] = tf[i];
  }
}
__global__ void inv8_kernel(const int32_t* __restrict__ levels, const uint8_t* __restrict__ types, int n, mt_quant q,
                            const uint8_t* __restrict__ qm_row, int32_t* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int32_t store[kWork8Words + 64];
  Work8 w{store};
  int32_t* cf = w.w;        // int32 levels at [0, 64)
  int32_t* o = w.w + 64;    // int32 output at [64, 128)
  for (int i = 0; i < 64; i++) cf[i] = levels[(size_t)idx * 64 + i];
  inv8x8(cf, types[idx], q, qm_row, o, store + kWork8Words);
  for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = o[i];
}
__global__ void trellis8_kernel(int32_t* __restrict__ levels, const float* __restrict__ targets, int n, float dc_q,
                                float ac_q, float lambda) {
  __shared__ float sLut[64];
  for (int i = threadIdx.x; i < 64; i += blockDim.x) sLut[i] = kCoefRateLut[i];
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  int32_t store[kWork8Words];
  Work8 w{store};
  int32_t* cf = w.w + 132;  // int32 levels at [132, 196)
  float* tf = w.tf();
  for (int i = 0; i < 64; i++) {
    cf[i] = levels[(size_t)idx * 64 + i];
    tf[i] = targets[(size_t)idx * 64 + i];
  }
  trellis8(cf, tf, w.suf(), dc_q, ac_q, lambda, sLut);
  for (int i = 0; i < 64; i++) levels[(size_t)idx * 64 + i] = cf[i];
}
__global__ void pred8_kernel(const uint16_t* __restrict__ rec, mt_chain_params p, const mt_candidate* __restrict__ cands,
                             int n, int32_t* __restrict__ out) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const mt_candidate cd = cands[idx];
  int32_t store[kWork8Words];
  Work8 w{store};
  int16_t* pr = w.pred();
  if (!cand_ok(cd, p.frame_w, p.frame_h)) {
    for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = 0;
    return;
  }
  predict8(rec, p.stride, p.frame_w, p.frame_h, cd.px, cd.py, cd.mode, cd.angle_delta, cd.flags & 1,
           (cd.flags >> 1) & 1, (cd.flags >> 2) & 1, p.bd, pr, w.edges());
  for (int i = 0; i < 64; i++) out[(size_t)idx * 64 + i] = pr[i];
}

}  // namespace mtd

// Host launchers used by the C ABI (capi.cu).
namespace {
// The displayed frame is smaller than the coded one: the distortion masks
// samples past it (a separate instantiation, so coded-size frames pay nothing).
bool clipped(const mt_chain_params& p) {
  return (p.vis_w > 0 && p.vis_w < p.frame_w) || (p.vis_h > 0 && p.vis_h < p.frame_h);
}
}  // namespace

namespace mth {
static mtd::ChainArgs make_args(const mt_chain_params& p, const mt_quant& q, float tl, const uint8_t* qm) {
  mtd::ChainArgs a;
  a.p = p;
  a.q = q;
  a.trellis_lambda = tl;
  a.has_qm = qm != nullptr;
  return a;
}

size_t chain8_scratch_bytes(int n) { return (size_t)2 * mtd::kBuckets * sizeof(int) + (size_t)n * sizeof(int); }

cudaError_t launch_chain8(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_candidate* cands, int n, mt_candidate_result* res, int32_t* lv, int32_t* ro,
                          void* scratch, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (n + mtd::kThreads - 1) / mtd::kThreads;
  int* perm = nullptr;
  if (scratch) {
    int* hist = static_cast<int*>(scratch);
    int* cursor = hist + mtd::kBuckets;
    perm = cursor + mtd::kBuckets;
    cudaError_t e = cudaMemsetAsync(hist, 0, mtd::kBuckets * sizeof(int), st);
    if (e != cudaSuccess) return e;
    mtd::bucket_count_kernel<<<blocks, mtd::kThreads, 0, st>>>(cands, n, hist);
    mtd::bucket_scan_kernel<<<1, mtd::kBuckets, 0, st>>>(hist, cursor);
    mtd::bucket_scatter_kernel<<<blocks, mtd::kThreads, 0, st>>>(cands, n, cursor, perm);
  }
  if (clipped(p))
    mtd::chain8_kernel<true><<<blocks, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row), qm_row,
                                                       costs, cands, perm, n, res, lv, ro);
  else
    mtd::chain8_kernel<false><<<blocks, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row), qm_row,
                                                       costs, cands, perm, n, res, lv, ro);
  return cudaGetLastError();
}

// Working storage of a level: argmin keys, the run table, the predictions.
struct LevelLayout {
  size_t keys, runs, preds, total;
};
LevelLayout level_layout(int nblocks, int ncombos) {
  auto up = [](size_t v) { return (v + 255) & ~(size_t)255; };
  LevelLayout L;
  L.keys = 0;
  L.runs = up((size_t)nblocks * 8);
  L.preds = L.runs + up(sizeof(mtd::LevelRuns));
  L.total = L.preds + (size_t)nblocks * ncombos * 64;
  return L;
}

size_t level8_scratch_bytes(int nblocks, int ncombos) {
  if (nblocks <= 0 || ncombos <= 0) return 0;
  return level_layout(nblocks, ncombos).total;
}

cudaError_t launch_level8(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                          mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st) {
  if (nblocks <= 0 || ncombos <= 0) return cudaSuccess;
  const LevelLayout L = level_layout(nblocks, ncombos);
  uint8_t* s = static_cast<uint8_t*>(scratch);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(s + L.keys);
  mtd::LevelRuns* runs = reinterpret_cast<mtd::LevelRuns*>(s + L.runs);
  uint4* preds = reinterpret_cast<uint4*>(s + L.preds);
  cudaError_t e = cudaMemsetAsync(keys, 0xff, (size_t)nblocks * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const mtd::ChainArgs args = make_args(p, q, trellis_lambda, qm_row);
  const long long total = (long long)nblocks * ncombos;
  const long long grid = (total + mtd::kThreads - 1) / mtd::kThreads;
  mtd::level8_runs_kernel<<<1, 32, 0, st>>>(combos, ncombos, runs);
  // At most ncombos runs: pred CTAs past the run count exit at once.
  mtd::level8_pred_kernel<<<(unsigned)grid, mtd::kThreads, 0, st>>>(rec, args, blocks, nblocks, combos, runs, preds);
  if (clipped(p))
    mtd::level8_kernel<true><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, args, qm_row, costs, blocks, nblocks, combos,
                                                               ncombos, runs, preds, res, keys);
  else
    mtd::level8_kernel<false><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, args, qm_row, costs, blocks, nblocks, combos,
                                                               ncombos, runs, preds, res, keys);
  mtd::level8_finalize_kernel<<<(nblocks + 255) / 256, 256, 0, st>>>(keys, nblocks, res, best);
  return cudaGetLastError();
}

cudaError_t launch_level4(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                          float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                          const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                          mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st) {
  if (nblocks <= 0 || ncombos <= 0) return cudaSuccess;
  unsigned long long* keys = static_cast<unsigned long long*>(scratch);
  cudaError_t e = cudaMemsetAsync(keys, 0xff, (size_t)nblocks * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const long long total = (long long)nblocks * ncombos;
  const long long grid = (total + mtd::kThreads - 1) / mtd::kThreads;
  if (clipped(p))
    mtd::level4_kernel<true><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row),
                                                               qm_row, costs, blocks, nblocks, combos, ncombos, res,
                                                               keys);
  else
    mtd::level4_kernel<false><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row),
                                                               qm_row, costs, blocks, nblocks, combos, ncombos, res,
                                                               keys);
  mtd::level8_finalize_kernel<<<(nblocks + 255) / 256, 256, 0, st>>>(keys, nblocks, res, best);
  return cudaGetLastError();
}

cudaError_t launch_level16(const uint16_t* src, const uint16_t* rec, const mt_chain_params& p, const mt_quant& q,
                           float trellis_lambda, const uint8_t* qm_row, const mt_coef_costs* costs,
                           const mt_block8* blocks, int nblocks, const mt_combo* combos, int ncombos,
                           mt_candidate_result* res, void* scratch, mt_block_best* best, cudaStream_t st) {
  if (nblocks <= 0 || ncombos <= 0) return cudaSuccess;
  unsigned long long* keys = static_cast<unsigned long long*>(scratch);
  cudaError_t e = cudaMemsetAsync(keys, 0xff, (size_t)nblocks * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const long long total = (long long)nblocks * ncombos;
  const long long grid = (total + mtd::kThreads - 1) / mtd::kThreads;
  if (clipped(p))
    mtd::level16_kernel<true><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row),
                                                                qm_row, costs, blocks, nblocks, combos, ncombos, res,
                                                                keys);
  else
    mtd::level16_kernel<false><<<(unsigned)grid, mtd::kThreads, 0, st>>>(src, rec, make_args(p, q, trellis_lambda, qm_row),
                                                                qm_row, costs, blocks, nblocks, combos, ncombos, res,
                                                                keys);
  mtd::level8_finalize_kernel<<<(nblocks + 255) / 256, 256, 0, st>>>(keys, nblocks, res, best);
  return cudaGetLastError();
}

cudaError_t launch_fwd8(const int32_t* resid, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* levels, float* targets, cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::fwd8_kernel<<<blocks, 128, 0, st>>>(resid, types, n, q, qm, levels, targets);
  return cudaGetLastError();
}
cudaError_t launch_inv8(const int32_t* levels, const uint8_t* types, int n, const mt_quant& q, const uint8_t* qm,
                        int32_t* out, cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::inv8_kernel<<<blocks, 128, 0, st>>>(levels, types, n, q, qm, out);
  return cudaGetLastError();
}
cudaError_t launch_trellis8(int32_t* levels, const float* targets, int n, float dc_q, float ac_q, float lambda,
                            cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::trellis8_kernel<<<blocks, 128, 0, st>>>(levels, targets, n, dc_q, ac_q, lambda);
  return cudaGetLastError();
}
cudaError_t launch_pred8(const uint16_t* rec, const mt_chain_params& p, const mt_candidate* cands, int n, int32_t* out,
                         cudaStream_t st) {
  const int blocks = (n + 127) / 128;
  if (blocks > 0) mtd::pred8_kernel<<<blocks, 128, 0, st>>>(rec, p, cands, n, out);
  return cudaGetLastError();
}
}  // namespace mth
