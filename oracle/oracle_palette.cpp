// Oracle (test infrastructure only): CPU restatement of the lossy luma
// palette candidates of src/coder/palette.rs and src/kmeans.rs, the checker
// for the device kernels in maroontree_b200/csrc/palette.cu.  Sequential and
// table-driven where the reference is (the Viterbi's transition table is
// tabulated per block here, recomputed per pixel on the device).
//
//   palette.rs:651-706    block_color_histogram (2..64 distinct values)
//   palette.rs:708-726    top_palette_centers
//   palette.rs:728-737    palette_centers' exact case
//   palette.rs:805-869    dp_palette_center_sets (the shipped palette_dp_centers)
//   palette.rs:456-537    palette_color_ctx (map form)
//   palette.rs:980-1021   palette_color_ctx_nb
//   palette.rs:1078-1172  viterbi_map_core
//   palette.rs:1173-1216  smooth_palette_map
//   palette.rs:1218-1265  lossy_luma_palette_from_centers
//   palette.rs:1911-1925  palette_index_bits
//   kmeans.rs:71-101      luma_nearest_indices_scalar
//   util.rs:63-78         dirty_log2f (f_fmlaf unfused: no FMA target feature in the default build)
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "oracle.h"

namespace {

struct Hist {
  int n = 0;
  int32_t v[64];
  uint32_t c[64];
};

// Distinct values ascending with counts; n = 0 when flat or > 64 distinct.
bool block_hist(const uint16_t* src, int stride, int px, int py, int w, int h, Hist& out) {
  std::vector<uint32_t> cnt(4096, 0);
  int distinct = 0;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int v = src[(size_t)(py + y) * stride + px + x];
      if (v >= 4096) return false;
      if (cnt[v]++ == 0 && ++distinct > 64) return false;
    }
  if (distinct < 2) return false;
  out.n = 0;
  for (int v = 0; v < 4096; v++)
    if (cnt[v]) {
      out.v[out.n] = v;
      out.c[out.n++] = cnt[v];
    }
  return true;
}

// Optimal centre sets for sizes 2..kmax; sets[k-2] empty (len 0) when k > n.
void dp_sets(const Hist& hs, int kmax, int32_t sets[7][8], int lens[7]) {
  const int h = hs.n;
  int64_t pw[65] = {0}, p1[65] = {0}, p2[65] = {0};
  for (int i = 0; i < h; i++) {
    const int64_t v = hs.v[i], c = hs.c[i];
    pw[i + 1] = pw[i] + c;
    p1[i + 1] = p1[i] + c * v;
    p2[i + 1] = p2[i] + c * v * v;
  }
  auto center = [&](int i, int j) {
    const int64_t w = pw[j] - pw[i];
    return (p1[j] - p1[i] + w / 2) / w;
  };
  std::vector<int64_t> cost(65 * 65, 0);
  for (int i = 0; i < h; i++)
    for (int j = i + 1; j <= h; j++) {
      const int64_t w = pw[j] - pw[i], s1 = p1[j] - p1[i], s2 = p2[j] - p2[i], c = center(i, j);
      cost[i * 65 + j] = s2 - 2 * c * s1 + c * c * w;
    }
  int64_t f[8][65];
  uint8_t arg[8][65];
  for (int k = 0; k < 8; k++)
    for (int j = 0; j < 65; j++) {
      f[k][j] = INT64_MAX;
      arg[k][j] = 0;
    }
  for (int j = 1; j <= h; j++) f[0][j] = cost[j];
  for (int k = 1; k < std::min(kmax, h); k++)
    for (int j = k + 1; j <= h; j++) {
      int64_t best = INT64_MAX;
      int bi = k;
      for (int i = k; i < j; i++) {
        const int64_t c = f[k - 1][i] + cost[i * 65 + j];
        if (c < best) {
          best = c;
          bi = i;
        }
      }
      f[k][j] = best;
      arg[k][j] = (uint8_t)bi;
    }
  for (int k = 0; k < 7; k++) lens[k] = 0;
  for (int nn = 2; nn <= std::min(kmax, h); nn++) {
    int bounds[9];
    bounds[nn] = h;
    for (int k = nn - 1; k >= 1; k--) bounds[k] = arg[k][bounds[k + 1]];
    bounds[0] = 0;
    for (int k = 0; k < nn; k++) sets[nn - 2][k] = (int32_t)center(bounds[k], bounds[k + 1]);
    lens[nn - 2] = nn;
  }
}

void ctx_nb(int l, int u, int ul, int cur, int& ctx, int& sym) {
  int n, r0, r1 = 0, r2 = 0;
  if (l >= 0 && u >= 0) {
    if (l == u) {
      if (l == ul) n = 1, ctx = 4, r0 = l;
      else n = 2, ctx = 3, r0 = l, r1 = ul;
    } else if (l == ul) {
      n = 2, ctx = 2, r0 = l, r1 = u;
    } else if (u == ul) {
      n = 2, ctx = 2, r0 = u, r1 = l;
    } else {
      n = 3, ctx = 1, r0 = std::min(l, u), r1 = std::max(l, u), r2 = ul;
    }
  } else if (l >= 0 || u >= 0) {
    n = 1, ctx = 0, r0 = l >= 0 ? l : u;
  } else {
    ctx = 0, sym = cur;
    return;
  }
  if (cur == r0) sym = 0;
  else if (n >= 2 && cur == r1) sym = 1;
  else if (n >= 3 && cur == r2) sym = 2;
  else sym = n + cur - ((r0 < cur) + (n >= 2 && r1 < cur) + (n >= 3 && r2 < cur));
}

// viterbi_map_core over n palette entries; dist(x, y, d) fills the squared
// error of every entry at map position (x, y).
template <typename D>
void viterbi_core(uint8_t* map, int w, int h, int n, const float costs[5][8], float lam, D dist_at) {
  std::vector<float> trans(8 * 8 * 8 * 8, 0.0f);
  float top[8][8] = {}, col[8][8] = {};
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      int ctx, sym;
      ctx_nb(j, -1, 0, i, ctx, sym);
      top[j][i] = lam * costs[ctx][sym];
      ctx_nb(-1, j, 0, i, ctx, sym);
      col[j][i] = lam * costs[ctx][sym];
      for (int u = 0; u < n; u++)
        for (int ul = 0; ul < n; ul++) {
          ctx_nb(j, u, ul, i, ctx, sym);
          trans[((u * 8 + ul) * 8 + j) * 8 + i] = lam * costs[ctx][sym];
        }
    }
  float prev[8] = {}, cur[8] = {}, dist[8];
  std::vector<uint8_t> back((size_t)w * 8, 0);
  for (int y = 0; y < h; y++) {
    for (int x = 0; x < w; x++) {
      dist_at(x, y, dist);
      if (x == 0) {
        if (y > 0) {
          const int u = map[(y - 1) * w];
          for (int i = 0; i < n; i++) cur[i] = dist[i] + col[u][i];
        } else {
          for (int i = 0; i < n; i++) cur[i] = dist[i];
        }
      } else {
        const float* t = y > 0 ? &trans[(size_t)(map[(y - 1) * w + x] * 8 + map[(y - 1) * w + x - 1]) * 64]
                               : &top[0][0];
        for (int i = 0; i < n; i++) {
          float best = INFINITY;
          uint8_t a = 0;
          for (int j = 0; j < n; j++) {
            const float cc = prev[j] + t[j * 8 + i];
            if (cc < best) {
              best = cc;
              a = (uint8_t)j;
            }
          }
          cur[i] = best + dist[i];
          back[(size_t)x * 8 + i] = a;
        }
      }
      memcpy(prev, cur, sizeof(prev));
    }
    int bi = 0;
    float bc = INFINITY;
    for (int i = 0; i < n; i++)
      if (prev[i] < bc) {
        bc = prev[i];
        bi = i;
      }
    for (int x = w - 1; x >= 0; x--) {
      map[y * w + x] = (uint8_t)bi;
      if (x > 0) bi = back[(size_t)x * 8 + bi];
    }
  }
}

// viterbi_palette_map (palette.rs:1028-1052): the luma distance.
void viterbi(uint8_t* map, const uint16_t* src, int stride, int px, int py, int w, int h, const int32_t* c, int n,
             const float costs[5][8], float lam) {
  viterbi_core(map, w, h, n, costs, lam, [&](int x, int y, float* d) {
    const int v = src[(size_t)(py + y) * stride + px + x];
    for (int i = 0; i < n; i++) {
      const float e = (float)(v - c[i]);
      d[i] = e * e;
    }
  });
}

void smooth(uint8_t* map, const uint16_t* src, int stride, int px, int py, int w, int h, const int32_t* c, int t,
            bool guard) {
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int v = src[(size_t)(py + y) * stride + px + x];
      const int i0 = map[y * w + x];
      const int d0 = std::abs(v - c[i0]);
      if (guard && d0 == 0) continue;
      int best = i0, best_d = d0 + t;
      if (x > 0) {
        const int l = map[y * w + x - 1], d = std::abs(v - c[l]);
        if (l != i0 && d <= best_d) best = l, best_d = d;
      }
      if (y > 0) {
        const int u = map[(y - 1) * w + x], d = std::abs(v - c[u]);
        if (u != i0 && u != best && d < best_d) best = u;
      }
      map[y * w + x] = (uint8_t)best;
    }
}

}  // namespace

extern "C" {

float or_dirty_log2f(float d) {
  uint32_t ix;
  memcpy(&ix, &d, 4);
  ix += 0x3f800000u - 0x3f3504f3u;
  const int e = (int)(ix >> 23) - 0x7f;
  ix = (ix & 0x007fffffu) + 0x3f3504f3u;
  float a;
  memcpy(&a, &ix, 4);
  const float x = (a - 1.0f) / (a + 1.0f);
  const float x2 = x * x;
  float u = 0.4121985850084821691e+0f;
  u = u * x2 + 0.5770780163490337802e+0f;
  u = u * x2 + 0.9617966939259845749e+0f;
  return (x2 * x) * u + (x * 0.2885390081777926802e+1f + (float)e);
}

void or_palette_color_ctx_nb(int32_t l, int32_t u, int32_t ul, int32_t cur, int32_t* ctx, int32_t* sym) {
  int c, s;
  ctx_nb(l, u, ul, cur, c, s);
  *ctx = c;
  *sym = s;
}

// palette_color_ctx over a map (the reference's specialised form; (0, 0) is
// never asked).
void or_palette_color_ctx(const uint8_t* map, int32_t stride, int32_t y, int32_t x, int32_t* ctx, int32_t* sym) {
  const int l = x > 0 ? map[y * stride + x - 1] : -1;
  const int u = y > 0 ? map[(y - 1) * stride + x] : -1;
  const int ul = (x > 0 && y > 0) ? map[(y - 1) * stride + x - 1] : 0;
  or_palette_color_ctx_nb(l, u, ul, map[y * stride + x], ctx, sym);
}

// luma_nearest_indices_scalar: first minimal squared distance (duplicates allowed).
void or_luma_nearest_indices(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                             const int32_t* centers, int32_t n, uint8_t* out) {
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int64_t s = src[(size_t)(py + y) * stride + px + x];
      int64_t bd = INT64_MAX;
      int bi = 0;
      for (int i = 0; i < n; i++) {
        const int64_t d = (s - centers[i]) * (s - centers[i]);
        if (d < bd) bd = d, bi = i;
      }
      out[y * w + x] = (uint8_t)bi;
    }
}

// Histogram (n_out = 0 when the gate rejects the block).
void or_block_color_histogram(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                              int32_t* vals, uint32_t* counts, int32_t* n_out) {
  Hist hs;
  if (!block_hist(src, stride, px, py, w, h, hs)) {
    *n_out = 0;
    return;
  }
  *n_out = hs.n;
  for (int i = 0; i < hs.n; i++) vals[i] = hs.v[i], counts[i] = hs.c[i];
}

// dp_palette_center_sets over a histogram: sets 7 x 8 (size k at row k-2), lens 7.
void or_dp_palette_center_sets(const int32_t* vals, const uint32_t* counts, int32_t n, int32_t kmax, int32_t* sets,
                               int32_t* lens) {
  Hist hs;
  hs.n = n;
  for (int i = 0; i < n; i++) hs.v[i] = vals[i], hs.c[i] = counts[i];
  int32_t s[7][8] = {};
  int l[7];
  dp_sets(hs, kmax, s, l);
  memcpy(sets, s, sizeof(s));
  for (int k = 0; k < 7; k++) lens[k] = l[k];
}

int or_luma_palette(const uint16_t* src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd, int32_t w,
                    int32_t h, const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_palette_cand* cands,
                    uint8_t* maps) {
  const int maxv = (1 << bd) - 1;
  for (int b = 0; b < n; b++) {
    const int px = pos[2 * b], py = pos[2 * b + 1];
    mt_palette_cand* cb = cands + (size_t)b * MT_PALETTE_SLOTS;
    uint8_t* mb = maps + (size_t)b * MT_PALETTE_SLOTS * w * h;
    memset(cb, 0, sizeof(mt_palette_cand) * MT_PALETTE_SLOTS);
    memset(mb, 0, (size_t)MT_PALETTE_SLOTS * w * h);
    bool ok = px + w <= frame_w && py + h <= frame_h;
    for (int y = 0; ok && y < h; y++)
      for (int x = 0; x < w; x++)
        if (src[(size_t)(py + y) * stride + px + x] > maxv) ok = false;
    Hist hs;
    if (!ok || !block_hist(src, stride, px, py, w, h, hs)) continue;
    int32_t sets[7][8] = {};
    int lens[7];
    dp_sets(hs, 8, sets, lens);
    // top_palette_centers: order by (count desc, value asc), keep the first nc, ascending
    int order[64];
    for (int i = 0; i < hs.n; i++) order[i] = i;
    std::sort(order, order + hs.n, [&](int a, int b2) {
      return hs.c[a] != hs.c[b2] ? hs.c[a] > hs.c[b2] : hs.v[a] < hs.v[b2];
    });
    for (int s = 0; s < MT_PALETTE_SLOTS; s++) {
      mt_palette_cand& cd = cb[s];
      cd.hist_len = (uint8_t)hs.n;
      int32_t c[8] = {};
      int nc = 0;
      if (s < 7) {
        cd.sel = (uint8_t)(s + 2);
        if (s + 2 <= hs.n) {
          nc = s + 2;
          if (nc == hs.n) for (int k = 0; k < nc; k++) c[k] = hs.v[k];
          else for (int k = 0; k < nc; k++) c[k] = sets[nc - 2][k];
        }
      } else {
        cd.sel = (uint8_t)(s + 3);
        if (s - 5 < hs.n) {
          nc = s - 5;
          for (int k = 0; k < nc; k++) c[k] = hs.v[order[k]];
          std::sort(c, c + nc);
        }
      }
      if (nc == 0) continue;
      cd.n_colors = (uint8_t)nc;
      for (int k = 0; k < 8; k++) cd.colors[k] = (int16_t)c[k];
      uint8_t* map = mb + (size_t)s * w * h;
      const float(*costs)[8] = opts->color_costs[nc - 2];
      if (opts->viterbi_lambda > 0.0f) {
        viterbi(map, src, stride, px, py, w, h, c, nc, costs, opts->viterbi_lambda);
      } else {
        or_luma_nearest_indices(src, stride, px, py, w, h, c, nc, map);
        if (opts->smooth_t > 0) smooth(map, src, stride, px, py, w, h, c, opts->smooth_t, opts->smooth_guard != 0);
      }
      float bits = or_dirty_log2f((float)nc);
      for (int dg = 1; dg < w + h - 1; dg++) {
        const int first_x = std::min(dg, w - 1), last_x = std::max(dg - (h - 1), 0);
        for (int x = first_x; x >= last_x; x--) {
          int ctx, sym;
          or_palette_color_ctx(map, w, dg - x, x, &ctx, &sym);
          bits += costs[ctx][sym];
        }
      }
      cd.index_bits = bits;
    }
  }
  return MT_OK;
}

}  // extern "C"

// ---- UV palette candidates ----

namespace {

using Pair = std::pair<int32_t, int32_t>;

// exact_uv_palette (palette.rs:199-262).
bool exact_uv(const uint16_t* su, const uint16_t* sv, int stride, int cx, int cy, int w, int h, std::vector<Pair>& pairs,
              uint8_t* map) {
  pairs.clear();
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const Pair p((int32_t)su[(size_t)(cy + y) * stride + cx + x], (int32_t)sv[(size_t)(cy + y) * stride + cx + x]);
      if (std::find(pairs.begin(), pairs.end(), p) == pairs.end()) {
        if (pairs.size() == 8) return false;
        pairs.push_back(p);
      }
    }
  if (pairs.size() < 2) return false;
  std::sort(pairs.begin(), pairs.end());
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const Pair p((int32_t)su[(size_t)(cy + y) * stride + cx + x], (int32_t)sv[(size_t)(cy + y) * stride + cx + x]);
      map[y * w + x] = (uint8_t)(std::find(pairs.begin(), pairs.end(), p) - pairs.begin());
    }
  return true;
}

// lossy_uv_palette_from_hist's centres (palette.rs:315-410); false: None.
bool lossy_uv_centers(const std::vector<std::pair<Pair, uint32_t>>& hist, int colors, bool top,
                      std::vector<Pair>& out) {
  if (hist.size() < 2 || (size_t)colors > hist.size()) return false;
  out.clear();
  if ((size_t)colors == hist.size()) {
    for (auto& e : hist) out.push_back(e.first);
  } else if (top) {
    std::vector<size_t> idx(hist.size());
    for (size_t i = 0; i < idx.size(); i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
      if (hist[a].second != hist[b].second) return hist[a].second > hist[b].second;
      return hist[a].first < hist[b].first;
    });
    for (int i = 0; i < colors; i++) out.push_back(hist[idx[(size_t)i]].first);
  } else {
    uint64_t total = 0;
    for (auto& e : hist) total += e.second;
    std::vector<Pair> init;
    for (int i = 0; i < colors; i++) {
      const uint32_t target = (uint32_t)((uint64_t)(2 * i + 1) * total / (uint64_t)(2 * colors));
      uint32_t acc = 0;
      Pair pick = hist.back().first;
      for (auto& e : hist) {
        acc += e.second;
        if (acc > target) {
          pick = e.first;
          break;
        }
      }
      init.push_back(pick);
    }
    init.erase(std::unique(init.begin(), init.end()), init.end());
    if ((int)init.size() != colors) return false;
    for (int it = 0; it < 8; it++) {
      int64_t su[8] = {}, sv[8] = {}, cnt[8] = {};
      for (auto& e : hist) {
        const int32_t u = e.first.first, v = e.first.second;
        int best = 0;
        int64_t bd = INT64_MAX;
        for (int i = 0; i < (int)init.size(); i++) {
          const int64_t du = u - init[(size_t)i].first, dv = v - init[(size_t)i].second;
          const int64_t d = du * du + dv * dv;
          if (d < bd) {
            bd = d;
            best = i;
          }
        }
        su[best] += (int64_t)u * e.second;
        sv[best] += (int64_t)v * e.second;
        cnt[best] += e.second;
      }
      for (int i = 0; i < (int)init.size(); i++)
        if (cnt[i] != 0)
          init[(size_t)i] = Pair((int32_t)((su[i] + cnt[i] / 2) / cnt[i]), (int32_t)((sv[i] + cnt[i] / 2) / cnt[i]));
      std::sort(init.begin(), init.end());
      init.erase(std::unique(init.begin(), init.end()), init.end());
      if ((int)init.size() != colors) return false;
    }
    out = init;
  }
  std::sort(out.begin(), out.end());
  return true;
}

}  // namespace

extern "C" int or_uv_palette(const uint16_t* su, const uint16_t* sv, int32_t stride, int32_t w, int32_t h,
                             const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* cands,
                             uint8_t* maps) {
  const size_t wh = (size_t)w * h;
  static const int kList[4][2] = {{8, 0}, {4, 0}, {8, 1}, {4, 1}};
  std::vector<Pair> pairs, centers;
  for (int b = 0; b < n; b++) {
    const int cx = pos[2 * b], cy = pos[2 * b + 1];
    mt_uv_palette_cand* cb = cands + (size_t)b * 4;
    uint8_t* mb = maps ? maps + (size_t)b * 4 * wh : nullptr;
    memset(cb, 0, 4 * sizeof(mt_uv_palette_cand));
    if (mb) memset(mb, 0, 4 * wh);
    std::vector<uint8_t> scratch(wh);
    if (exact_uv(su, sv, stride, cx, cy, w, h, pairs, mb ? mb : scratch.data())) {
      cb[0].n_colors = (uint8_t)pairs.size();
      cb[0].exact = 1;
      for (size_t i = 0; i < pairs.size(); i++) {
        cb[0].u[i] = (int16_t)pairs[i].first;
        cb[0].v[i] = (int16_t)pairs[i].second;
      }
      continue;
    }
    // uv_pair_histogram (palette.rs:264-309)
    std::vector<Pair> all;
    for (int y = 0; y < h; y++)
      for (int x = 0; x < w; x++)
        all.emplace_back((int32_t)su[(size_t)(cy + y) * stride + cx + x], (int32_t)sv[(size_t)(cy + y) * stride + cx + x]);
    std::sort(all.begin(), all.end());
    std::vector<std::pair<Pair, uint32_t>> hist;
    for (auto& p : all) {
      if (!hist.empty() && hist.back().first == p) hist.back().second++;
      else hist.emplace_back(p, 1u);
    }
    for (int k = 0; k < 4; k++) {
      if (!lossy_uv_centers(hist, kList[k][0], kList[k][1] != 0, centers)) continue;
      const int nc = (int)centers.size();
      cb[k].n_colors = (uint8_t)nc;
      int32_t cu[8] = {}, cv[8] = {};
      for (int i = 0; i < nc; i++) {
        cu[i] = centers[(size_t)i].first;
        cv[i] = centers[(size_t)i].second;
        cb[k].u[i] = (int16_t)cu[i];
        cb[k].v[i] = (int16_t)cv[i];
      }
      uint8_t* map = mb ? mb + (size_t)k * wh : scratch.data();
      if (opts->viterbi_lambda > 0.0f) {
        viterbi_core(map, w, h, nc, opts->color_costs[nc - 2], opts->viterbi_lambda, [&](int x, int y, float* d) {
          const size_t o = (size_t)(cy + y) * stride + cx + x;
          const int32_t u = su[o], v = sv[o];
          for (int i = 0; i < nc; i++) {
            const float eu = (float)(u - cu[i]), ev = (float)(v - cv[i]);
            d[i] = eu * eu + ev * ev;
          }
        });
      } else {
        for (int y = 0; y < h; y++)  // uv_nearest_indices (kmeans.rs:37-68)
          for (int x = 0; x < w; x++) {
            const size_t o = (size_t)(cy + y) * stride + cx + x;
            const int32_t u = su[o], v = sv[o];
            int64_t bd = INT64_MAX;
            int bi = 0;
            for (int i = 0; i < nc; i++) {
              const int64_t du = u - cu[i], dv = v - cv[i];
              const int64_t d = du * du + dv * dv;
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
  return MT_OK;
}
