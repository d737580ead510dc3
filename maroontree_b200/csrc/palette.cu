// Lossy luma palette candidates over a batch of blocks (src/coder/palette.rs).
//
// pal_centers_kernel: one warp per block.  block_color_histogram (:651-706)
// as a 4096-bit shared bitset (atomicOr per sample; the distinct values come
// out ascending from a popcount prefix over the words) plus per-value counts
// (atomicAdd at the value's rank, exact integers); then the fourteen centre
// sets: dp_palette_center_sets (:805-869, the interval DP over prefix sums,
// lanes over the interval end j, first minimal start on ties), the exact
// distinct values when colours == distinct (:728-737), and
// top_palette_centers (:708-726, rank by count desc / value asc).
//
// pal_map_kernel: one thread per (slot, block), slot-major so a warp runs one
// palette size over 32 blocks.  lossy_luma_palette_from_centers
// (:1218-1265): viterbi_map_core (:1078-1172; the transition bits of
// palette_color_ctx_nb, :980-1021, tabulated once per CTA in shared memory) or
// luma_nearest_indices (src/kmeans.rs:71-101) + smooth_palette_map
// (:1173-1216); then palette_index_bits (:1911-1925) in its diagonal order.
// Float arithmetic is explicit round-to-nearest in the reference's order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "leaf8.cuh"

namespace {

using mtd::arena_launch_shape;
using mtd::arena_stride;
using mtd::smem_arena;

constexpr int kSlots = MT_PALETTE_SLOTS;
constexpr int kWarps = 4;

struct PalShared {
  uint32_t bits[128];  // one bit per sample value, bd <= 12
  int32_t wpre[128];   // distinct values before each word
  int32_t vals[64];
  uint32_t cnt[64];
  int32_t rank[64];    // position in (count desc, value asc)
  long long pw[65], p1[65], p2[65];
  long long f[8][65];
  uint8_t arg[8][65];
};

__device__ __forceinline__ long long iv_center(const PalShared& s, int i, int j) {
  const long long w = s.pw[j] - s.pw[i];
  return (s.p1[j] - s.p1[i] + w / 2) / w;
}

__device__ __forceinline__ long long iv_cost(const PalShared& s, int i, int j) {
  const long long w = s.pw[j] - s.pw[i], s1 = s.p1[j] - s.p1[i], s2 = s.p2[j] - s.p2[i];
  const long long c = (s1 + w / 2) / w;
  return s2 - 2 * c * s1 + c * c * w;
}

__global__ void __launch_bounds__(32 * kWarps) pal_centers_kernel(const uint16_t* __restrict__ src, int stride,
                                                                   int fw, int fh, int bd, int w, int h,
                                                                   const uint16_t* __restrict__ pos, int n,
                                                                   mt_palette_cand* __restrict__ cands) {
  __shared__ PalShared sh[kWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = blockIdx.x * kWarps + warp;
  if (b >= n) return;  // warp-uniform
  PalShared& s = sh[warp];
  const int px = pos[2 * b], py = pos[2 * b + 1];
  const int maxv = (1 << bd) - 1;
  bool ok = px + w <= fw && py + h <= fh;
  int H = 0;
  if (ok) {
    for (int i = lane; i < 128; i += 32) s.bits[i] = 0u;
    __syncwarp();
    bool bad = false;
    for (int i = lane; i < w * h; i += 32) {
      const int v = src[(size_t)(py + i / w) * stride + px + i % w];
      if (v > maxv) bad = true;
      else atomicOr(&s.bits[v >> 5], 1u << (v & 31));
    }
    ok = !__any_sync(0xffffffffu, bad);
    __syncwarp();
    // distinct values: lane owns words 4 lane .. 4 lane + 3
    int c = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) c += __popc(s.bits[4 * lane + k]);
    int incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int o = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += o;
    }
    H = __shfl_sync(0xffffffffu, incl, 31);
    if (ok && H >= 2 && H <= 64) {
      int at = incl - c;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int wd = 4 * lane + k;
        s.wpre[wd] = at;
        uint32_t m = s.bits[wd];
        while (m) {
          const int bit = __ffs(m) - 1;
          s.vals[at++] = wd * 32 + bit;
          m &= m - 1;
        }
      }
      for (int i = lane; i < 64; i += 32) s.cnt[i] = 0u;
      __syncwarp();
      for (int i = lane; i < w * h; i += 32) {
        const int v = src[(size_t)(py + i / w) * stride + px + i % w];
        atomicAdd(&s.cnt[s.wpre[v >> 5] + __popc(s.bits[v >> 5] & ((1u << (v & 31)) - 1u))], 1u);
      }
      __syncwarp();
      if (lane == 0) {
        s.pw[0] = s.p1[0] = s.p2[0] = 0;
        for (int i = 0; i < H; i++) {
          const long long v = s.vals[i], cc = s.cnt[i];
          s.pw[i + 1] = s.pw[i] + cc;
          s.p1[i + 1] = s.p1[i] + cc * v;
          s.p2[i + 1] = s.p2[i] + cc * v * v;
        }
      }
      for (int e = lane; e < H; e += 32) {
        int r = 0;
        for (int j = 0; j < H; j++)
          r += s.cnt[j] > s.cnt[e] || (s.cnt[j] == s.cnt[e] && s.vals[j] < s.vals[e]);
        s.rank[e] = r;
      }
      __syncwarp();
      // F(0, j) = C(0, j); F(k, j) = min over i in k..j-1 of F(k-1, i) + C(i, j)
      for (int j = 1 + lane; j <= H; j += 32) s.f[0][j] = iv_cost(s, 0, j);
      __syncwarp();
      const int kmax = min(8, H);
      for (int k = 1; k < kmax; k++) {
        for (int j = k + 1 + lane; j <= H; j += 32) {
          long long best = 0x7fffffffffffffffLL;
          int bi = k;
          for (int i = k; i < j; i++) {
            const long long cst = s.f[k - 1][i] + iv_cost(s, i, j);
            if (cst < best) {
              best = cst;
              bi = i;
            }
          }
          s.f[k][j] = best;
          s.arg[k][j] = (uint8_t)bi;
        }
        __syncwarp();
      }
    }
  }
  if (!ok || H < 2 || H > 64) H = 0;
  if (lane >= kSlots) return;
  mt_palette_cand cd;
#pragma unroll
  for (int k = 0; k < 8; k++) cd.colors[k] = 0;
  cd.n_colors = 0;
  cd.sel = 0;
  cd.hist_len = (uint8_t)H;
  cd.reserved = 0;
  cd.index_bits = 0.0f;
  const int slot = lane;
  if (H > 0) {
    if (slot < 7) {
      const int nc = slot + 2;
      cd.sel = (uint8_t)nc;
      if (nc <= H) {
        cd.n_colors = (uint8_t)nc;
        if (nc == H) {
          for (int k = 0; k < nc; k++) cd.colors[k] = (int16_t)s.vals[k];
        } else {
          int bounds[9];
          bounds[nc] = H;
          for (int k = nc - 1; k >= 1; k--) bounds[k] = s.arg[k][bounds[k + 1]];
          bounds[0] = 0;
          for (int k = 0; k < nc; k++) cd.colors[k] = (int16_t)iv_center(s, bounds[k], bounds[k + 1]);
        }
      }
    } else {
      const int nc = slot - 5;
      cd.sel = (uint8_t)(nc + 8);
      if (nc < H) {
        cd.n_colors = (uint8_t)nc;
        int k = 0;
        for (int e = 0; e < H; e++)
          if (s.rank[e] < nc) cd.colors[k++] = (int16_t)s.vals[e];
      }
    }
  }
  cands[(size_t)b * kSlots + slot] = cd;
}

// palette_color_ctx_nb (palette.rs:980-1021): l / u < 0 = absent.
__device__ __forceinline__ void color_ctx_nb(int l, int u, int ul, int cur, int& ctx, int& sym) {
  int n, r0, r1 = 0, r2 = 0;
  if (l >= 0 && u >= 0) {
    if (l == u) {
      if (l == ul) {
        n = 1; ctx = 4; r0 = l;
      } else {
        n = 2; ctx = 3; r0 = l; r1 = ul;
      }
    } else if (l == ul) {
      n = 2; ctx = 2; r0 = l; r1 = u;
    } else if (u == ul) {
      n = 2; ctx = 2; r0 = u; r1 = l;
    } else {
      n = 3; ctx = 1; r0 = min(l, u); r1 = max(l, u); r2 = ul;
    }
  } else if (l >= 0 || u >= 0) {
    n = 1; ctx = 0; r0 = l >= 0 ? l : u;
  } else {
    ctx = 0;
    sym = cur;
    return;
  }
  if (cur == r0) sym = 0;
  else if (n >= 2 && cur == r1) sym = 1;
  else if (n >= 3 && cur == r2) sym = 2;
  else {
    int below = r0 < cur;
    if (n >= 2) below += r1 < cur;
    if (n >= 3) below += r2 < cur;
    sym = n + cur - below;
  }
}

// dirty_log2f (src/util.rs:63-78) with f_fmlaf unfused (the default x86_64
// build has no FMA target feature).
__device__ float dirty_log2f(float d) {
  uint32_t ix = __float_as_uint(d);
  ix += 0x3f800000u - 0x3f3504f3u;
  const int e = (int)(ix >> 23) - 0x7f;
  ix = (ix & 0x007fffffu) + 0x3f3504f3u;
  const float a = __uint_as_float(ix);
  const float x = __fdiv_rn(__fsub_rn(a, 1.0f), __fadd_rn(a, 1.0f));
  const float x2 = __fmul_rn(x, x);
  float u = 0.4121985850084821691e+0f;
  u = __fadd_rn(__fmul_rn(u, x2), 0.5770780163490337802e+0f);
  u = __fadd_rn(__fmul_rn(u, x2), 0.9617966939259845749e+0f);
  const float inner = __fadd_rn(__fmul_rn(x, 0.2885390081777926802e+1f), (float)e);
  return __fadd_rn(__fmul_rn(__fmul_rn(x2, x), u), inner);
}

__global__ void __launch_bounds__(128) pal_map_kernel(const uint16_t* __restrict__ src, int stride, int w, int h,
                                                       const uint16_t* __restrict__ pos, int n,
                                                       const mt_palette_opts opt,
                                                       mt_palette_cand* __restrict__ cands,
                                                       uint8_t* __restrict__ maps) {
  // The weighted transition bits lam x costs[ctx][sym] depend on the slot's
  // palette size alone, so the CTA tabulates them once for the (at most two)
  // slots its threads start in: [u][ul][j][i] interior, then top[j][i] (first
  // row) and col[u][i] (first column), as viterbi_map_core does per block.
  // Threads of a third slot (n < 64) price on the fly: the same products.
  constexpr int kTab = 4096 + 128;
  __shared__ float sTr[2][kTab];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int slot = (int)(t / n), b = (int)(t - (long long)slot * n);
  const int slot0 = (int)(((long long)blockIdx.x * blockDim.x) / n);
  const float lam = opt.viterbi_lambda;
  if (lam > 0.0f) {
    for (int e = threadIdx.x; e < 2 * kTab; e += blockDim.x) {
      const int k = e / kTab, r = e - k * kTab, s = slot0 + k;
      if (s >= kSlots) continue;
      const int ns = s < 7 ? s + 2 : s - 5;
      int ctx = 0, sym = 0, i;
      bool in;
      if (r < 4096) {
        const int u = r >> 9, ul = (r >> 6) & 7, j = (r >> 3) & 7;
        i = r & 7;
        in = u < ns && ul < ns && j < ns && i < ns;
        if (in) color_ctx_nb(j, u, ul, i, ctx, sym);
      } else if (r < 4096 + 64) {
        const int j = (r - 4096) >> 3;
        i = r & 7;
        in = j < ns && i < ns;
        if (in) color_ctx_nb(j, -1, 0, i, ctx, sym);
      } else {
        const int u = (r - 4160) >> 3;
        i = r & 7;
        in = u < ns && i < ns;
        if (in) color_ctx_nb(-1, u, 0, i, ctx, sym);
      }
      sTr[k][r] = in ? __fmul_rn(lam, opt.color_costs[ns - 2][ctx][sym]) : 0.0f;
    }
    __syncthreads();
  }
  if (slot >= kSlots) return;
  const float* tab = slot - slot0 < 2 ? sTr[slot - slot0] : nullptr;
  mt_palette_cand& cd = cands[(size_t)b * kSlots + slot];
  uint8_t* map = maps + ((size_t)b * kSlots + slot) * w * h;
  const int nc = cd.n_colors;
  if (nc == 0) {
    for (int i = 0; i < w * h; i++) map[i] = 0;
    return;
  }
  int32_t c[8];
#pragma unroll
  for (int k = 0; k < 8; k++) c[k] = cd.colors[k];
  const int px = pos[2 * b], py = pos[2 * b + 1];
  const uint16_t* blk = src + (size_t)py * stride + px;
  const float(*costs)[8] = opt.color_costs[nc - 2];
  if (lam > 0.0f) {
    uint8_t back[64 * 8];
    float prev[8], cur[8];
#pragma unroll
    for (int i = 0; i < 8; i++) prev[i] = cur[i] = 0.0f;
    for (int y = 0; y < h; y++) {
      for (int x = 0; x < w; x++) {
        const int v = blk[(size_t)y * stride + x];
        float dist[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const float e = (float)(v - c[i]);
          dist[i] = __fmul_rn(e, e);
        }
        if (x == 0) {
          if (y > 0) {
            const int u = map[(y - 1) * w];
#pragma unroll
            for (int i = 0; i < 8; i++) {
              if (i >= nc) break;
              float tc;
              if (tab) {
                tc = tab[4160 + u * 8 + i];
              } else {
                int ctx, sym;
                color_ctx_nb(-1, u, 0, i, ctx, sym);
                tc = __fmul_rn(lam, costs[ctx][sym]);
              }
              cur[i] = __fadd_rn(dist[i], tc);
            }
          } else {
#pragma unroll
            for (int i = 0; i < 8; i++) cur[i] = dist[i];
          }
        } else {
          const int u = y > 0 ? map[(y - 1) * w + x] : -1;
          const int ul = y > 0 ? map[(y - 1) * w + x - 1] : 0;
          const float* tr = tab ? (y > 0 ? tab + (u * 8 + ul) * 64 : tab + 4096) : nullptr;
          // states are unrolled to 8 and cut at nc so prev / cur / dist stay
          // in registers
#pragma unroll
          for (int i = 0; i < 8; i++) {
            if (i >= nc) break;
            float best = __int_as_float(0x7f800000);
            int arg = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
              if (j >= nc) break;
              float tc;
              if (tr) {
                tc = tr[j * 8 + i];
              } else {
                int ctx, sym;
                color_ctx_nb(j, u, ul, i, ctx, sym);
                tc = __fmul_rn(lam, costs[ctx][sym]);
              }
              const float cc = __fadd_rn(prev[j], tc);
              if (cc < best) {
                best = cc;
                arg = j;
              }
            }
            cur[i] = __fadd_rn(best, dist[i]);
            back[x * 8 + i] = (uint8_t)arg;
          }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) prev[i] = cur[i];
      }
      int bi = 0;
      float bc = __int_as_float(0x7f800000);
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i < nc && prev[i] < bc) {
          bc = prev[i];
          bi = i;
        }
      for (int x = w - 1; x >= 0; x--) {
        map[y * w + x] = (uint8_t)bi;
        if (x > 0) bi = back[x * 8 + bi];
      }
    }
  } else {
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++) {
        const int v = blk[(size_t)y * stride + x];
        long long bd = 0x7fffffffffffffffLL;
        int bi = 0;
        for (int i = 0; i < nc; i++) {
          const long long d = (long long)(v - c[i]) * (v - c[i]);
          if (d < bd) {
            bd = d;
            bi = i;
          }
        }
        map[y * w + x] = (uint8_t)bi;
      }
    if (opt.smooth_t > 0 && nc > 1)
      for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
          const int v = blk[(size_t)y * stride + x];
          const int i0 = map[y * w + x];
          const int d0 = abs(v - c[i0]);
          if (opt.smooth_guard && d0 == 0) continue;
          int best = i0, best_d = d0 + opt.smooth_t;
          if (x > 0) {
            const int l = map[y * w + x - 1];
            const int d = abs(v - c[l]);
            if (l != i0 && d <= best_d) {
              best = l;
              best_d = d;
            }
          }
          if (y > 0) {
            const int u = map[(y - 1) * w + x];
            const int d = abs(v - c[u]);
            if (u != i0 && u != best && d < best_d) best = u;
          }
          map[y * w + x] = (uint8_t)best;
        }
  }
  // palette_index_bits: the first entry uniform, the rest on the diagonals
  float bits = dirty_log2f((float)nc);
  for (int dg = 1; dg < w + h - 1; dg++) {
    const int first_x = min(dg, w - 1), last_x = max(dg - (h - 1), 0);
    for (int x = first_x; x >= last_x; x--) {
      const int y = dg - x;
      const int l = x > 0 ? map[y * w + x - 1] : -1;
      const int u = y > 0 ? map[(y - 1) * w + x] : -1;
      const int ul = (x > 0 && y > 0) ? map[(y - 1) * w + x - 1] : 0;
      int ctx, sym;
      color_ctx_nb(l, u, ul, map[y * w + x], ctx, sym);
      bits = __fadd_rn(bits, costs[ctx][sym]);
    }
  }
  cd.index_bits = bits;
}

bool dim_ok(int v) { return v == 4 || v == 8 || v == 16 || v == 32 || v == 64; }

int check(int32_t stride, int32_t fw, int32_t fh, int32_t bd, int32_t w, int32_t h, int32_t n,
          const mt_palette_opts* opts) {
  if (!opts || n < 0 || fw <= 0 || fh <= 0 || stride < fw || !dim_ok(w) || !dim_ok(h)) return MT_ERR_INVALID_INPUT;
  if (bd != 8 && bd != 10 && bd != 12) return MT_ERR_UNSUPPORTED;
  if (opts->smooth_t < 0 || !(opts->viterbi_lambda >= 0.0f)) return MT_ERR_INVALID_INPUT;
  if ((long long)n * kSlots > 0x7fffffffLL) return MT_ERR_TOO_LARGE;
  return MT_OK;
}

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

// ---- UV palette candidates (exact_uv_palette, uv_pair_histogram,
// lossy_uv_palette_from_hist, src/coder/palette.rs:199-431; the index map by
// viterbi_uv_palette_map, :1053-1076, or uv_nearest_indices,
// src/kmeans.rs:37-68) ----
//
// One thread per block.  The (U, V) pairs are sorted as u << 16 | v keys (the
// reference's lexicographic pair order) with a Shell sort in local memory,
// counted into the histogram, then the exact palette (2..8 distinct pairs:
// the histogram itself) or the four lossy candidates; each candidate's map
// is written straight to its slot.

constexpr int kUvMaxSamples = 32 * 32;

// The histogram is compacted into the sorted keys in place (entry e's key in
// key[e], its count in cnt[e]).  Each thread's copy sits in the CTA's dynamic
// shared memory (1.5 KB for blocks up to 16x16, 6 KB up to 32x32), which keeps
// the per-thread local allocation under 1 KB.  The kernel's time goes to each
// thread's serial work, not to this scratch: the 8-colour Viterbi derives n^2
// palette contexts per sample, and a warp's lanes diverge between exact and
// lossy blocks.
template <int MAXS>
struct UvPalScratch {
  uint32_t key[MAXS];
  uint16_t cnt[MAXS];
};

__device__ __forceinline__ int32_t key_u(uint32_t k) { return (int32_t)(k >> 16); }
__device__ __forceinline__ int32_t key_v(uint32_t k) { return (int32_t)(k & 0xffffu); }

// lossy_uv_palette_from_hist's centres (ascending keys); false: None.
__device__ bool uv_lossy_centers(const uint32_t* hk, const uint16_t* hc, int hn, int colors, bool top,
                                 uint32_t* out) {
  if (hn < 2 || colors > hn) return false;
  if (colors == hn) {
    for (int i = 0; i < colors; i++) out[i] = hk[i];
    return true;  // already ascending
  }
  if (top) {
    // the `colors` most frequent pairs, count descending then pair ascending
    int n = 0;
    while (n < colors) {
      int best = -1;
      for (int i = 0; i < hn; i++) {
        bool used = false;
        for (int k = 0; k < n; k++) used |= out[k] == hk[i];
        if (used) continue;
        if (best < 0 || hc[i] > hc[best]) best = i;  // ties keep the smaller pair (earlier in the sorted list)
      }
      out[n++] = hk[best];
    }
  } else {
    unsigned long long total = 0;
    for (int i = 0; i < hn; i++) total += hc[i];
    uint32_t init[8];
    int m = 0;
    for (int i = 0; i < colors; i++) {
      const uint32_t target = (uint32_t)((unsigned long long)(2 * i + 1) * total / (unsigned long long)(2 * colors));
      uint32_t acc = 0, pick = hk[hn - 1];
      for (int e = 0; e < hn; e++) {
        acc += hc[e];
        if (acc > target) {
          pick = hk[e];
          break;
        }
      }
      if (m == 0 || init[m - 1] != pick) init[m++] = pick;  // dedup of consecutive equal starts
    }
    if (m != colors) return false;
    for (int it = 0; it < 8; it++) {
      long long su[8] = {}, sv[8] = {}, cnt[8] = {};
      for (int e = 0; e < hn; e++) {
        const int32_t u = key_u(hk[e]), v = key_v(hk[e]);
        int best = 0;
        long long bd = 0x7fffffffffffffffLL;
        for (int i = 0; i < m; i++) {
          const long long du = u - key_u(init[i]), dv = v - key_v(init[i]);
          const long long d = du * du + dv * dv;
          if (d < bd) {
            bd = d;
            best = i;
          }
        }
        su[best] += (long long)u * hc[e];
        sv[best] += (long long)v * hc[e];
        cnt[best] += hc[e];
      }
      for (int i = 0; i < m; i++)
        if (cnt[i] != 0)
          init[i] = ((uint32_t)((su[i] + cnt[i] / 2) / cnt[i]) << 16) | (uint32_t)((sv[i] + cnt[i] / 2) / cnt[i]);
      // sort (at most eight) and drop consecutive duplicates
      for (int a = 1; a < m; a++) {
        const uint32_t x = init[a];
        int b = a - 1;
        while (b >= 0 && init[b] > x) {
          init[b + 1] = init[b];
          b--;
        }
        init[b + 1] = x;
      }
      int k = 0;
      for (int i = 0; i < m; i++)
        if (k == 0 || init[k - 1] != init[i]) init[k++] = init[i];
      m = k;
      if (m != colors) return false;
    }
    for (int i = 0; i < colors; i++) out[i] = init[i];
  }
  for (int a = 1; a < colors; a++) {  // centres.sort_unstable()
    const uint32_t x = out[a];
    int b = a - 1;
    while (b >= 0 && out[b] > x) {
      out[b + 1] = out[b];
      b--;
    }
    out[b + 1] = x;
  }
  return true;
}

template <int MAXS>
__global__ void __launch_bounds__(64) uv_pal_kernel(const uint16_t* __restrict__ su, const uint16_t* __restrict__ sv,
                                                    int stride, int w, int h, const uint16_t* __restrict__ pos, int n,
                                                    const mt_palette_opts opt, mt_uv_palette_cand* __restrict__ cands,
                                                    uint8_t* __restrict__ maps, int arena) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  const int wh = w * h, cx = pos[2 * b], cy = pos[2 * b + 1];
  mt_uv_palette_cand* cb = cands + (size_t)b * MT_UV_PALETTE_SLOTS;
  uint8_t* mb = maps ? maps + (size_t)b * MT_UV_PALETTE_SLOTS * wh : nullptr;
  for (int k = 0; k < MT_UV_PALETTE_SLOTS; k++) {
    cb[k].n_colors = 0;
    cb[k].exact = 0;
    cb[k].reserved[0] = cb[k].reserved[1] = 0;
    for (int i = 0; i < 8; i++) cb[k].u[i] = cb[k].v[i] = 0;
  }
  if (mb)
    for (int i = 0; i < MT_UV_PALETTE_SLOTS * wh; i++) mb[i] = 0;
  UvPalScratch<MAXS>& S = smem_arena<UvPalScratch<MAXS>>(arena);
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const size_t o = (size_t)(cy + y) * stride + cx + x;
      S.key[y * w + x] = ((uint32_t)su[o] << 16) | sv[o];
    }
  // Shell sort (gaps 701, 301, 132, 57, 23, 10, 4, 1)
  const int gaps[8] = {701, 301, 132, 57, 23, 10, 4, 1};
  for (int g = 0; g < 8; g++) {
    const int gap = gaps[g];
    for (int i = gap; i < wh; i++) {
      const uint32_t x = S.key[i];
      int j = i;
      while (j >= gap && S.key[j - gap] > x) {
        S.key[j] = S.key[j - gap];
        j -= gap;
      }
      S.key[j] = x;
    }
  }
  int hn = 0;  // uv_pair_histogram: hn <= i, so the compaction never overtakes the read
  for (int i = 0; i < wh; i++) {
    if (hn > 0 && S.key[hn - 1] == S.key[i]) {
      S.cnt[hn - 1]++;
    } else {
      S.key[hn] = S.key[i];
      S.cnt[hn] = 1;
      hn++;
    }
  }
  uint32_t centers[8];
  const int kColors[4] = {8, 4, 8, 4};
  for (int k = 0; k < MT_UV_PALETTE_SLOTS; k++) {
    int nc;
    if (hn >= 2 && hn <= 8) {  // exact_uv_palette: slot 0 only
      if (k > 0) break;
      nc = hn;
      for (int i = 0; i < nc; i++) centers[i] = S.key[i];
      cb[0].exact = 1;
    } else {
      if (!uv_lossy_centers(S.key, S.cnt, hn, kColors[k], k >= 2, centers)) continue;
      nc = kColors[k];
    }
    cb[k].n_colors = (uint8_t)nc;
    int32_t cu[8] = {}, cvv[8] = {};
    for (int i = 0; i < nc; i++) {
      cu[i] = key_u(centers[i]);
      cvv[i] = key_v(centers[i]);
      cb[k].u[i] = (int16_t)cu[i];
      cb[k].v[i] = (int16_t)cvv[i];
    }
    if (!mb) continue;
    uint8_t* map = mb + (size_t)k * wh;
    const bool exact = hn >= 2 && hn <= 8;
    if (exact) {
      for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
          const size_t o = (size_t)(cy + y) * stride + cx + x;
          const uint32_t key = ((uint32_t)su[o] << 16) | sv[o];
          int idx = 0;
          for (int i = 0; i < nc; i++)
            if (centers[i] == key) idx = i;
          map[y * w + x] = (uint8_t)idx;
        }
    } else if (opt.viterbi_lambda > 0.0f) {
      const float lam = opt.viterbi_lambda;
      const float(*costs)[8] = opt.color_costs[nc - 2];
      uint8_t back[32 * 8];
      float prev[8], cur[8];
      for (int i = 0; i < 8; i++) prev[i] = cur[i] = 0.0f;
      for (int y = 0; y < h; y++) {
        for (int x = 0; x < w; x++) {
          const size_t o = (size_t)(cy + y) * stride + cx + x;
          const int32_t u = su[o], v = sv[o];
          float dist[8];
          for (int i = 0; i < nc; i++) {
            const float eu = (float)(u - cu[i]), ev = (float)(v - cvv[i]);
            dist[i] = __fadd_rn(__fmul_rn(eu, eu), __fmul_rn(ev, ev));
          }
          if (x == 0) {
            if (y > 0) {
              const int up = map[(y - 1) * w];
              for (int i = 0; i < nc; i++) {
                int ctx, sym;
                color_ctx_nb(-1, up, 0, i, ctx, sym);
                cur[i] = __fadd_rn(dist[i], __fmul_rn(lam, costs[ctx][sym]));
              }
            } else {
              for (int i = 0; i < nc; i++) cur[i] = dist[i];
            }
          } else {
            const int up = y > 0 ? map[(y - 1) * w + x] : -1;
            const int ul = y > 0 ? map[(y - 1) * w + x - 1] : 0;
            for (int i = 0; i < nc; i++) {
              float best = __int_as_float(0x7f800000);
              int arg = 0;
              for (int j = 0; j < nc; j++) {
                int ctx, sym;
                color_ctx_nb(j, up, ul, i, ctx, sym);
                const float cc = __fadd_rn(prev[j], __fmul_rn(lam, costs[ctx][sym]));
                if (cc < best) {
                  best = cc;
                  arg = j;
                }
              }
              cur[i] = __fadd_rn(best, dist[i]);
              back[x * 8 + i] = (uint8_t)arg;
            }
          }
          for (int i = 0; i < 8; i++) prev[i] = cur[i];
        }
        int bi = 0;
        float bc = __int_as_float(0x7f800000);
        for (int i = 0; i < nc; i++)
          if (prev[i] < bc) {
            bc = prev[i];
            bi = i;
          }
        for (int x = w - 1; x >= 0; x--) {
          map[y * w + x] = (uint8_t)bi;
          if (x > 0) bi = back[x * 8 + bi];
        }
      }
    } else {
      for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
          const size_t o = (size_t)(cy + y) * stride + cx + x;
          const int32_t u = su[o], v = sv[o];
          long long bd = 0x7fffffffffffffffLL;
          int bi = 0;
          for (int i = 0; i < nc; i++) {
            const long long du = u - cu[i], dv = v - cvv[i];
            const long long d = du * du + dv * dv;
            if (d < bd) {
              bd = d;
              bi = i;
            }
          }
          map[y * w + x] = (uint8_t)bi;
        }
    }
  }
}

}  // namespace

extern "C" {

int mt_luma_palette_device(const uint16_t* d_src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd,
                           int32_t w, int32_t h, const uint16_t* d_pos, int32_t n, const mt_palette_opts* opts,
                           mt_palette_cand* d_cands, uint8_t* d_maps, void* stream) {
  const int rc = check(stride, frame_w, frame_h, bd, w, h, n, opts);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!d_src || !d_pos || !d_cands || !d_maps) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  pal_centers_kernel<<<(n + kWarps - 1) / kWarps, 32 * kWarps, 0, st>>>(d_src, stride, frame_w, frame_h, bd, w, h,
                                                                      d_pos, n, d_cands);
  const long long total = (long long)n * kSlots;
  pal_map_kernel<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(d_src, stride, w, h, d_pos, n, *opts, d_cands,
                                                                  d_maps);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_luma_palette(const uint16_t* src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd, int32_t w,
                    int32_t h, const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_palette_cand* cands,
                    uint8_t* maps) {
  int rc = check(stride, frame_w, frame_h, bd, w, h, n, opts);
  if (rc != MT_OK) return rc;
  if (n == 0) return MT_OK;
  if (!src || !pos || !cands) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)stride * frame_h * 2, ncand = (size_t)n * kSlots;
  const size_t nmap = ncand * w * h;
  const size_t o_pos = up256(plane), o_c = o_pos + up256((size_t)n * 4), o_m = o_c + up256(ncand * sizeof(mt_palette_cand));
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_m + up256(nmap)) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d, src, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_pos, pos, (size_t)n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    rc = mt_luma_palette_device(reinterpret_cast<const uint16_t*>(d), stride, frame_w, frame_h, bd, w, h,
                                reinterpret_cast<const uint16_t*>(d + o_pos), n, opts,
                                reinterpret_cast<mt_palette_cand*>(d + o_c), d + o_m, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(cands, d + o_c, ncand * sizeof(mt_palette_cand), cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && maps) e = cudaMemcpy(maps, d + o_m, nmap, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_uv_palette_device(const uint16_t* d_src_u, const uint16_t* d_src_v, int32_t stride, int32_t w, int32_t h,
                         const uint16_t* d_pos, int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* d_cands,
                         uint8_t* d_maps, void* stream) {
  if (!opts || n < 0 || w < 4 || h < 4 || w > 32 || h > 32 || stride < w) return MT_ERR_INVALID_INPUT;
  if (!(opts->viterbi_lambda >= 0.0f)) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  if (!d_src_u || !d_src_v || !d_pos || !d_cands) return MT_ERR_INVALID_INPUT;
  auto* kern = w * h <= 256 ? uv_pal_kernel<256> : uv_pal_kernel<kUvMaxSamples>;
  const int arena = w * h <= 256 ? arena_stride(sizeof(UvPalScratch<256>))
                                 : arena_stride(sizeof(UvPalScratch<kUvMaxSamples>));
  int threads = 0;
  size_t dyn = 0;
  if (!arena_launch_shape(kern, n, arena, 64, &threads, &dyn)) return MT_ERR_DEVICE;
  kern<<<(unsigned)((n + threads - 1) / threads), threads, dyn, reinterpret_cast<cudaStream_t>(stream)>>>(
      d_src_u, d_src_v, stride, w, h, d_pos, n, *opts, d_cands, d_maps, arena);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_uv_palette(const uint16_t* src_u, const uint16_t* src_v, int32_t stride, int32_t rows, int32_t w, int32_t h,
                  const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* cands,
                  uint8_t* maps) {
  if (!opts || n < 0 || rows <= 0 || stride <= 0) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  if (!src_u || !src_v || !pos || !cands) return MT_ERR_INVALID_INPUT;
  for (int32_t b = 0; b < n; b++)  // every block inside the planes
    if ((int64_t)pos[2 * b] + w > stride || (int64_t)pos[2 * b + 1] + h > rows) return MT_ERR_INVALID_INPUT;
  const size_t plane = (size_t)stride * rows * 2, pb = (size_t)n * 4, cb = (size_t)n * MT_UV_PALETTE_SLOTS *
                                                                           sizeof(mt_uv_palette_cand);
  const size_t mbytes = maps ? (size_t)n * MT_UV_PALETTE_SLOTS * w * h : 0;
  const size_t o_u = 0, o_v = up256(plane), o_p = o_v + up256(plane), o_c = o_p + up256(pb), o_m = o_c + up256(cb);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_m + up256(mbytes ? mbytes : 1)) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_u, src_u, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_v, src_v, plane, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_p, pos, pb, cudaMemcpyHostToDevice);
  int rc = MT_OK;
  if (e == cudaSuccess) {
    rc = mt_uv_palette_device(reinterpret_cast<const uint16_t*>(d + o_u), reinterpret_cast<const uint16_t*>(d + o_v),
                              stride, w, h, reinterpret_cast<const uint16_t*>(d + o_p), n, opts,
                              reinterpret_cast<mt_uv_palette_cand*>(d + o_c), maps ? d + o_m : nullptr, nullptr);
    if (rc == MT_OK) e = cudaMemcpy(cands, d + o_c, cb, cudaMemcpyDeviceToHost);
    if (rc == MT_OK && e == cudaSuccess && maps) e = cudaMemcpy(maps, d + o_m, mbytes, cudaMemcpyDeviceToHost);
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
