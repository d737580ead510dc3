// Screen-content frame gate (screen_frame_gate, src/coder/screen_gate.rs:64-273).
//
// Block pass (sg_block16_kernel, one warp per 16x16 luma block, 8 blocks per
// CTA): each lane holds 8 samples (one row half); the distinct-value count is
// the popcount of a per-warp shared bitset of the 4096 possible values
// (block_color_histogram, src/coder/palette.rs:651-690, with its > 64 / < 2
// cut-offs), the span a warp min/max.  Each lane also holds one row of one
// aligned 8x8 sub-block, so the window hash (hash8, src/coder/block64.rs:177-188:
// c = sum r_j * HQ^(7-j) mod 2^32 over the 8 row hashes) is a 3-step shuffle
// sum.  The repeats among the non-flat hashes are counted by inserting them in
// an open-addressing set (64-bit CAS); repeats = inserts - new keys, which is the
// reference's `!seen.insert(h)` count whatever the insertion order.
//
// Copy stage (when the pre-screen passes; the host reads four counters):
// sg_index_kernel hashes every 8x8 window on the chroma-parity grid into a
// 64-bit key (hash << 32 | y << 16 | x); the keys are sorted (bitonic: one
// 2048-key shared-memory sort per CTA, then global merge steps with the
// shared-memory tail), and a bucket table over the top 16 hash bits indexes
// them.  Equal hashes are then in raster order of origins, which is the order
// in which the reference's bucketed index (LossyIbcIndex::build /
// candidates, src/coder/block64.rs:190-329) offers candidates, so the first
// three earlier exact copies are the same.  sg_gain_kernel (one warp per 16x16
// block) forms the gradient-energy mass, walks those candidates (exact 8x8
// compare and the 16x16 SSE are warp-cooperative) and the photo-like count;
// gain / photo / copies are integer atomics (order-free).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"

namespace {

constexpr uint32_t kHp = 0x9E3779B1u, kHq = 0x85EBCA77u;
constexpr int kSortChunk = 2048;  // keys per CTA of the shared-memory sort
constexpr int kBuckets = 1 << 16;

constexpr uint32_t hq_pow(int e) {
  uint32_t r = 1;
  for (int i = 0; i < e; i++) r *= kHq;
  return r;
}
__constant__ uint32_t cHqPow[8] = {hq_pow(7), hq_pow(6), hq_pow(5), hq_pow(4),
                                   hq_pow(3), hq_pow(2), hq_pow(1), hq_pow(0)};

__device__ __forceinline__ uint32_t ibc_mix(uint32_t h) {
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  return h ^ (h >> 16);
}

__device__ __forceinline__ uint32_t row_hash8(const uint16_t* v) {
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) r = r * kHp + ((uint32_t)v[i] + 1u);
  return r;
}

__device__ __forceinline__ void load8(const uint16_t* p, uint16_t* v) {
  const uint4 q = *reinterpret_cast<const uint4*>(p);
  const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    v[2 * i] = (uint16_t)(w[i] & 0xffffu);
    v[2 * i + 1] = (uint16_t)(w[i] >> 16);
  }
}

// Sum / and / min / max over the 8 lanes of one 8x8 sub-block (lanes that
// differ in bits 1..3: the sub-block's 8 rows).
__device__ __forceinline__ uint32_t sub_sum(uint32_t v) {
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  return v;
}
__device__ __forceinline__ int sub_min(int v) {
  v = min(v, __shfl_xor_sync(0xffffffffu, v, 2));
  v = min(v, __shfl_xor_sync(0xffffffffu, v, 4));
  return min(v, __shfl_xor_sync(0xffffffffu, v, 8));
}
__device__ __forceinline__ int sub_max(int v) {
  v = max(v, __shfl_xor_sync(0xffffffffu, v, 2));
  v = max(v, __shfl_xor_sync(0xffffffffu, v, 4));
  return max(v, __shfl_xor_sync(0xffffffffu, v, 8));
}
__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Counters in the scratch (all integer, order-free).
enum { kFew16, kLenient16, kNonflat, kDistinct, kGain, kPhoto, kCopied, kNCounters };

struct Geom {
  int w8, h8, n16x, n16y, span_min;
  int step_x, step_y, nwx, nwy;  // index grid
  uint32_t set_mask;              // hash-set slots - 1
  uint32_t n_keys, n_pad;
  unsigned long long dv_cost;
};

// Insert into the open-addressing set; true when h was not there yet.  The set
// has at least twice as many slots as keys, so a free slot is always reached.
__device__ bool set_insert(unsigned long long* __restrict__ tab, uint32_t mask, uint32_t h) {
  const unsigned long long key = (1ull << 32) | h;
  uint32_t i = h & mask;
  for (uint32_t probe = 0; probe <= mask; probe++) {
    const unsigned long long prev = atomicCAS(&tab[i], 0ull, key);
    if (prev == 0ull) return true;
    if (prev == key) return false;
    i = (i + 1) & mask;
  }
  return false;
}

__global__ void __launch_bounds__(256) sg_block16_kernel(const uint16_t* __restrict__ luma, const Geom g,
                                                         uint8_t* __restrict__ few, unsigned long long* __restrict__ set,
                                                         unsigned long long* __restrict__ counters) {
  __shared__ uint32_t s_bits[8][128];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * 8 + warp;
  if (blk >= g.n16x * g.n16y) return;
  const int row16 = blk / g.n16x, col16 = blk - row16 * g.n16x;
  const int r = lane >> 1, half = lane & 1;
  const int px = col16 * 16, py = row16 * 16;
  uint16_t v[8];
  load8(luma + (size_t)(py + r) * g.w8 + px + half * 8, v);
  // distinct values of the 16x16 block
  uint32_t* bits = s_bits[warp];
#pragma unroll
  for (int k = 0; k < 4; k++) bits[lane * 4 + k] = 0u;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 8; i++) atomicOr(&bits[(v[i] >> 5) & 127], 1u << (v[i] & 31));
  __syncwarp();
  int cnt = 0, lo = 1 << 30, hi = -1;
#pragma unroll
  for (int k = 0; k < 4; k++) cnt += __popc(bits[lane * 4 + k]);
#pragma unroll
  for (int i = 0; i < 8; i++) {
    lo = min(lo, (int)v[i]);
    hi = max(hi, (int)v[i]);
  }
  cnt = warp_sum(cnt);
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const bool hist = cnt >= 2 && cnt <= 64 && hi - lo >= g.span_min;
  const bool is_few = hist && cnt <= 8, is_len = hist && cnt <= 16;
  // the four aligned 8x8 sub-blocks: hash and flatness
  const uint32_t c = sub_sum(row_hash8(v) * cHqPow[r & 7]);
  const uint16_t first = (uint16_t)__shfl_sync(0xffffffffu, (uint32_t)v[0], ((r & 8) << 1) | half);
  bool same = true;
#pragma unroll
  for (int i = 0; i < 8; i++) same &= v[i] == first;
  const uint32_t flat = sub_sum(same ? 0u : 1u) == 0u;
  int nonflat = 0, fresh = 0;
  if ((r & 7) == 0 && !flat) {
    nonflat = 1;
    fresh = set_insert(set, g.set_mask, ibc_mix(c)) ? 1 : 0;
  }
  nonflat = warp_sum(nonflat);
  fresh = warp_sum(fresh);
  if (lane == 0) {
    few[blk] = is_few;
    if (is_few) atomicAdd(&counters[kFew16], 1ull);
    if (is_len) atomicAdd(&counters[kLenient16], 1ull);
    if (nonflat) atomicAdd(&counters[kNonflat], (unsigned long long)nonflat);
    if (fresh) atomicAdd(&counters[kDistinct], (unsigned long long)fresh);
  }
}

// Every window on the chroma-parity grid: key = hash << 32 | y << 16 | x; the
// padding up to the sort size takes the largest key.
__global__ void sg_index_kernel(const uint16_t* __restrict__ luma, const Geom g, unsigned long long* __restrict__ keys) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n_pad) return;
  if (i >= g.n_keys) {
    keys[i] = ~0ull;
    return;
  }
  const uint32_t wy = i / g.nwx, wx = i - wy * g.nwx;
  const int x = wx * g.step_x, y = wy * g.step_y;
  uint32_t cc = 0;
  for (int j = 0; j < 8; j++) {
    const uint16_t* row = luma + (size_t)(y + j) * g.w8 + x;
    uint32_t rr = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) rr = rr * kHp + ((uint32_t)row[k] + 1u);
    cc = cc * kHq + rr;
  }
  keys[i] = ((unsigned long long)ibc_mix(cc) << 32) | ((uint32_t)y << 16) | (uint32_t)x;
}

__device__ __forceinline__ void cmp_swap(unsigned long long& a, unsigned long long& b, bool asc) {
  if ((a > b) == asc) {
    const unsigned long long t = a;
    a = b;
    b = t;
  }
}

// Bitonic steps inside one 2048-key chunk: the whole sort up to k = 2048
// (merge_k == 0), or the j < 2048 steps of the merge of size merge_k.
__global__ void __launch_bounds__(1024) sg_sort_local_kernel(unsigned long long* __restrict__ keys, uint32_t merge_k) {
  __shared__ unsigned long long s[kSortChunk];
  const uint32_t t = threadIdx.x, base = blockIdx.x * kSortChunk;
  s[t] = keys[base + t];
  s[t + 1024] = keys[base + t + 1024];
  __syncthreads();
  const uint32_t k0 = merge_k ? merge_k : 2u, k1 = merge_k ? merge_k : (uint32_t)kSortChunk;
  for (uint32_t k = k0; k <= k1; k <<= 1) {
    for (uint32_t j = min(k, (uint32_t)kSortChunk) >> 1; j > 0; j >>= 1) {
      const uint32_t i = 2 * t - (t & (j - 1));
      const bool asc = ((base + i) & k) == 0;
      cmp_swap(s[i], s[i + j], asc);
      __syncthreads();
    }
  }
  keys[base + t] = s[t];
  keys[base + t + 1024] = s[t + 1024];
}

__global__ void sg_sort_global_kernel(unsigned long long* __restrict__ keys, uint32_t n_pad, uint32_t k, uint32_t j) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_pad / 2) return;
  const uint32_t i = 2 * t - (t & (j - 1));
  unsigned long long a = keys[i], b = keys[i + j];
  const unsigned long long a0 = a;
  cmp_swap(a, b, (i & k) == 0);
  if (a != a0) {
    keys[i] = a;
    keys[i + j] = b;
  }
}

// start[b] = first sorted key whose top 16 hash bits are >= b, b in [0, 65536].
__global__ void sg_bucket_kernel(const unsigned long long* __restrict__ keys, uint32_t n, uint32_t* __restrict__ start) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = (int)(keys[i] >> 48);
  const int prev = i == 0 ? -1 : (int)(keys[i - 1] >> 48);
  for (int bb = prev + 1; bb <= b; bb++) start[bb] = i;
  if (i == n - 1)
    for (int bb = b + 1; bb <= kBuckets; bb++) start[bb] = n;
}

__global__ void __launch_bounds__(256) sg_gain_kernel(const uint16_t* __restrict__ luma, const Geom g,
                                                      const uint8_t* __restrict__ few,
                                                      const unsigned long long* __restrict__ keys,
                                                      const uint32_t* __restrict__ start,
                                                      unsigned long long* __restrict__ counters) {
  __shared__ uint32_t s_bits[8][4][128];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int blk = blockIdx.x * 8 + warp;
  if (blk >= g.n16x * g.n16y) return;
  const int row16 = blk / g.n16x, col16 = blk - row16 * g.n16x;
  const int r = lane >> 1, half = lane & 1, sub = ((r >> 3) << 1) | half;
  const int px = col16 * 16, py = row16 * 16;
  const int w8 = g.w8;
  uint16_t v[8];
  load8(luma + (size_t)(py + r) * w8 + px + half * 8, v);
  // sad8 of this lane's sub-block row: horizontal steps, and the step from the
  // row above inside the sub-block.
  uint32_t e = 0;
#pragma unroll
  for (int i = 0; i < 7; i++) {
    const int d = (int)v[i] - (int)v[i + 1];
    e += (uint32_t)(d * d);
  }
  uint16_t up[8];
#pragma unroll
  for (int i = 0; i < 8; i++) up[i] = (uint16_t)__shfl_up_sync(0xffffffffu, (uint32_t)v[i], 2);
  if ((r & 7) != 0)
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int d = (int)v[i] - (int)up[i];
      e += (uint32_t)(d * d);
    }
  const uint32_t sad_sub = sub_sum(e);  // <= 112 * 4095^2 < 2^32
  const unsigned long long mass =
      warp_sum64((r & 7) == 0 ? (unsigned long long)sad_sub : 0ull);
  if (mass == 0) return;
  const uint32_t hsub = ibc_mix(sub_sum(row_hash8(v) * cHqPow[r & 7]));
  unsigned long long best = ~0ull;
  for (int k = 0; k < 4 && best != 0; k++) {
    const int sx = px + (k & 1) * 8, sy = py + (k >> 1) * 8;
    const uint32_t want = __shfl_sync(0xffffffffu, hsub, ((k >> 1) << 4) | (k & 1));
    // candidates: equal hashes in raster order of origin, origin rows <= sy
    uint32_t lo = start[want >> 16], hi = start[(want >> 16) + 1];
    const unsigned long long key0 = (unsigned long long)want << 32;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (keys[mid] < key0) lo = mid + 1;
      else hi = mid;
    }
    int taken = 0;
    for (uint32_t q = lo; q < g.n_keys && taken < 3; q++) {
      const unsigned long long kk = keys[q];
      if ((uint32_t)(kk >> 32) != want) break;
      const int ay = (int)((kk >> 16) & 0xffffu), ax = (int)(kk & 0xffffu);
      if (ay > sy) break;
      const bool earlier = ay + 8 <= sy || (ay <= sy && ax + 8 <= sx);
      if (!earlier) continue;
      {  // exact 8x8 copy: two samples per lane
        const int rr = lane >> 2, cc = (lane & 3) * 2;
        const uint16_t* pa = luma + (size_t)(ay + rr) * w8 + ax + cc;
        const uint16_t* pb = luma + (size_t)(sy + rr) * w8 + sx + cc;
        if (!__all_sync(0xffffffffu, pa[0] == pb[0] && pa[1] == pb[1])) continue;
      }
      taken++;
      if (px + ax < sx || py + ay < sy) continue;
      const int rx = px + ax - sx, ry = py + ay - sy;
      if (rx + 16 > w8 || ry + 16 > g.h8 || (ry + 16 > py && rx + 16 > px && ry < py + 16 && rx < px + 16)) continue;
      const uint16_t* pr = luma + (size_t)(ry + r) * w8 + rx + half * 8;
      unsigned long long res = 0;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const long long d = (long long)v[i] - (long long)pr[i];
        res += (unsigned long long)(d * d);
      }
      res = warp_sum64(res);
      best = min(best, res);
      if (best == 0) break;
    }
  }
  unsigned long long gv = 0;
  if (best != ~0ull) {
    gv = mass > best ? mass - best : 0ull;
    gv = gv > g.dv_cost ? gv - g.dv_cost : 0ull;
  }
  if (gv > 0) {
    if (lane == 0) {
      atomicAdd(&counters[kGain], gv);
      atomicAdd(&counters[kCopied], 1ull);
    }
    return;
  }
  if (few[blk]) return;
  // photo-like 8x8s: not a text fragment (2..12 values spanning span_min) and textured
  uint32_t* bits = s_bits[warp][sub];
#pragma unroll
  for (int k = 0; k < 16; k++) bits[(r & 7) * 16 + k] = 0u;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 8; i++) atomicOr(&bits[(v[i] >> 5) & 127], 1u << (v[i] & 31));
  __syncwarp();
  int cnt = 0, mn = 1 << 30, mx = -1;
#pragma unroll
  for (int k = 0; k < 16; k++) cnt += __popc(bits[(r & 7) * 16 + k]);
#pragma unroll
  for (int i = 0; i < 8; i++) {
    mn = min(mn, (int)v[i]);
    mx = max(mx, (int)v[i]);
  }
  cnt = (int)sub_sum((uint32_t)cnt);
  mn = sub_min(mn);
  mx = sub_max(mx);
  const bool text = cnt >= 2 && cnt <= 12 && mx - mn >= g.span_min;
  const int photo = warp_sum(((r & 7) == 0 && !text && sad_sub > 0) ? 1 : 0);
  if (lane == 0 && photo) atomicAdd(&counters[kPhoto], (unsigned long long)photo);
}

struct Layout {
  size_t few, counters, set, keys, start, total;
};

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

int make_geom(const mt_screen_gate_params* p, Geom* g) {
  if (!p) return MT_ERR_INVALID_INPUT;
  if (p->w8 <= 0 || p->h8 <= 0 || (p->w8 & 7) || (p->h8 & 7) || p->w8 > 16384 || p->h8 > 16384)
    return MT_ERR_INVALID_INPUT;
  if (p->sub_x < 0 || p->sub_x > 1 || p->sub_y < 0 || p->sub_y > 1) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8 && p->bd != 10 && p->bd != 12) return MT_ERR_UNSUPPORTED;
  if (p->base_q_idx < 0 || p->base_q_idx > 255) return MT_ERR_INVALID_INPUT;
  memset(g, 0, sizeof(*g));
  g->w8 = p->w8;
  g->h8 = p->h8;
  g->n16x = p->w8 / 16;
  g->n16y = p->h8 / 16;
  g->span_min = 64 << (p->bd - 8);
  g->step_x = 1 << p->sub_x;
  g->step_y = 1 << p->sub_y;
  if (p->w8 >= 16 && p->h8 >= 16) {
    g->nwx = (p->w8 - 7 + g->step_x - 1) / g->step_x;
    g->nwy = (p->h8 - 7 + g->step_y - 1) / g->step_y;
  }
  const uint64_t nk = (uint64_t)g->nwx * g->nwy;
  if (nk > MT_SCREEN_MAX_WINDOWS) return MT_ERR_TOO_LARGE;
  g->n_keys = (uint32_t)nk;
  uint32_t np = kSortChunk;
  while (np < g->n_keys) np <<= 1;
  g->n_pad = np;
  uint32_t slots = 1024;
  while (slots < 2u * 4u * (uint32_t)(g->n16x * g->n16y)) slots <<= 1;
  g->set_mask = slots - 1;
  const float acq = (float)(p->bd == 10 ? MT_AC_QLOOKUP_10 : (p->bd == 12 ? MT_AC_QLOOKUP_12 : MT_AC_QLOOKUP_8))
      [p->base_q_idx];
  // (ibc_gate_dv * ac_q^2) as u64 (src/coder/screen_gate.rs:168); ibc_gate_dv = 1.
  const float dvf = 1.0f * (acq * acq);
  g->dv_cost = (unsigned long long)dvf;
  return MT_OK;
}

Layout make_layout(const Geom& g) {
  Layout L;
  L.few = 0;
  L.counters = up256((size_t)g.n16x * g.n16y);
  L.set = L.counters + up256(kNCounters * 8);
  L.keys = L.set + up256(((size_t)g.set_mask + 1) * 8);
  L.start = L.keys + up256((size_t)g.n_pad * 8);
  L.total = L.start + up256((size_t)(kBuckets + 1) * 4);
  return L;
}

// loop_filter_levels(q, sub).0 with lf_level_scale 1 (src/obu.rs:314).
int lf_level_y(int q) { return std::min(std::max((int)roundf((float)(q / 8) * 1.0f), 0), 40); }

}  // namespace

extern "C" {

size_t mt_screen_gate_scratch_bytes(const mt_screen_gate_params* prm) {
  Geom g;
  if (make_geom(prm, &g) != MT_OK) return 0;
  return make_layout(g).total;
}

int mt_screen_gate_device(const uint16_t* d_luma, const mt_screen_gate_params* prm, void* d_scratch,
                          mt_screen_gate_result* out, void* stream) {
  Geom g;
  int rc = make_geom(prm, &g);
  if (rc != MT_OK) return rc;
  if (!d_luma || !d_scratch || !out) return MT_ERR_INVALID_INPUT;
  if (reinterpret_cast<uintptr_t>(d_luma) & 15) return MT_ERR_INVALID_INPUT;
  memset(out, 0, sizeof(*out));
  if (g.w8 / 8 < 2 || g.h8 / 8 < 2) return MT_OK;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const Layout L = make_layout(g);
  uint8_t* s = static_cast<uint8_t*>(d_scratch);
  uint8_t* few = s + L.few;
  unsigned long long* counters = reinterpret_cast<unsigned long long*>(s + L.counters);
  unsigned long long* set = reinterpret_cast<unsigned long long*>(s + L.set);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(s + L.keys);
  uint32_t* start = reinterpret_cast<uint32_t*>(s + L.start);
  if (cudaMemsetAsync(s + L.counters, 0, L.keys - L.counters, st) != cudaSuccess) return MT_ERR_DEVICE;
  const int n16 = g.n16x * g.n16y;
  unsigned long long h[kNCounters] = {0};
  if (n16 > 0) {
    sg_block16_kernel<<<(n16 + 7) / 8, 256, 0, st>>>(d_luma, g, few, set, counters);
    if (cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MT_ERR_DEVICE;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MT_ERR_DEVICE;
  }
  const uint32_t t16 = (uint32_t)std::max(n16, 1);
  const float total16 = (float)t16;
  out->blocks16 = (uint32_t)n16;
  out->few16 = (uint32_t)h[kFew16];
  out->lenient16 = (uint32_t)h[kLenient16];
  out->nonflat8 = (uint32_t)h[kNonflat];
  out->dup8 = (uint32_t)(h[kNonflat] - h[kDistinct]);
  out->few_colour = (float)out->few16 / total16 >= 0.10f;
  const float dup8 = (float)out->dup8 / (4.0f * total16);
  const float lenient_share = (float)out->lenient16 / total16;
  if (lenient_share < 0.02f && dup8 < 0.02f) return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
  out->copy_stage = 1;
  if (g.n_keys > 0) {
    sg_index_kernel<<<(g.n_pad + 255) / 256, 256, 0, st>>>(d_luma, g, keys);
    sg_sort_local_kernel<<<g.n_pad / kSortChunk, 1024, 0, st>>>(keys, 0u);
    for (uint32_t k = 2 * kSortChunk; k <= g.n_pad; k <<= 1) {
      for (uint32_t j = k >> 1; j >= (uint32_t)kSortChunk; j >>= 1)
        sg_sort_global_kernel<<<(g.n_pad / 2 + 255) / 256, 256, 0, st>>>(keys, g.n_pad, k, j);
      sg_sort_local_kernel<<<g.n_pad / kSortChunk, 1024, 0, st>>>(keys, k);
    }
    sg_bucket_kernel<<<(g.n_keys + 255) / 256, 256, 0, st>>>(keys, g.n_keys, start);
  } else {
    // An empty index: every bucket is empty.
    if (cudaMemsetAsync(start, 0, (size_t)(kBuckets + 1) * 4, st) != cudaSuccess) return MT_ERR_DEVICE;
  }
  if (n16 > 0) sg_gain_kernel<<<(n16 + 7) / 8, 256, 0, st>>>(d_luma, g, few, keys, start, counters);
  if (cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MT_ERR_DEVICE;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MT_ERR_DEVICE;
  out->gain = h[kGain];
  out->photo = h[kPhoto];
  out->copied = (uint32_t)h[kCopied];
  // The deblocking the copies cost scales with the quantiser step, and is 0
  // once the q-law switches the filter off (screen_gate.rs:255-271).
  const double acd = (double)(prm->bd == 10 ? MT_AC_QLOOKUP_10 : (prm->bd == 12 ? MT_AC_QLOOKUP_12 : MT_AC_QLOOKUP_8))
      [prm->base_q_idx];
  const double loss = lf_level_y(prm->base_q_idx) > 0 ? (double)32.0f * (double)out->photo * acd : 0.0;
  out->ibc_pays = out->copied >= 4 && (double)out->gain > loss;
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_screen_gate(const uint16_t* luma, const mt_screen_gate_params* prm, mt_screen_gate_result* out) {
  Geom g;
  int rc = make_geom(prm, &g);
  if (rc != MT_OK) return rc;
  if (!luma || !out) return MT_ERR_INVALID_INPUT;
  const size_t ny = (size_t)g.w8 * g.h8 * 2;
  const size_t scratch = make_layout(g).total;
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, up256(ny) + scratch) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d, luma, ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) rc = mt_screen_gate_device(reinterpret_cast<const uint16_t*>(d), prm, d + up256(ny), out, nullptr);
  cudaFree(d);
  if (e != cudaSuccess) return MT_ERR_DEVICE;
  return rc;
}

}  // extern "C"
