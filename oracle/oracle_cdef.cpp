// Oracle (test infrastructure only): the reference's frame CDEF, restated
// serially in the reference's order with the plain per-candidate filter.
//   constants / constrain     src/cdef.rs:31-87
//   direction                 src/cdef.rs:89-178 (cdef_direction_partials / _cost)
//   adjust_pri                src/cdef.rs:181-189
//   filter                    src/cdef.rs:386-620 (cdef_filter_block, its generic
//                             body and sample(): taps outside the plane excluded)
//   weighted SSE              src/avx/rd.rs:767-848 (AVX2 lane order with FMA),
//                             weights / basis src/rd_sse.rs:1400-1430, rounding
//                             src/rd_sse.rs:277-287 (wsse_err, scale 1)
//   unit tables               src/coder/frame_cdef.rs:600-820: each of the 12
//                             strength pairs filtered on its own (the reference's
//                             fused candidate routine, src/cdef.rs:651-800, is
//                             asserted equal to this per candidate)
//   strength search / apply   src/coder/frame_cdef.rs:49-520, :960-1125
//   frame lambda_d            src/coder.rs:259-271, src/cost.rs:110-160, :270-292
//   tuning (SHIPPED)          src/tuning.rs:772-776, :913-915, :761-763, :964-968
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <vector>

#include "oracle.h"

namespace {

constexpr int kVeryLarge = 0x4000;
const int kDirs[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}},
};
const int kPriTaps[2][2] = {{4, 2}, {3, 3}};
const int kSecTaps[2] = {2, 1};
const int kCandPri[4] = {0, 1, 2, 4};
const int kCandSec[3] = {0, 1, 2};

int log2_floor(int v) { return v <= 0 ? 0 : 31 - __builtin_clz((unsigned)v); }

int constrain(int diff, int strength, int damping) {
  if (strength == 0) return 0;
  int shift = damping - log2_floor(strength);
  if (shift < 0) shift = 0;
  const int a = abs(diff);
  int r = strength - (a >> shift);
  r = r < 0 ? 0 : (r > a ? a : r);
  return diff < 0 ? -r : r;
}

void direction(const uint16_t* plane, int stride, int rows, int x, int y, int bd, int* dir, int* var) {
  const int cs = bd - 8;
  int64_t partial[8][15] = {};
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const int yy = std::min(y + i, rows - 1), xx = std::min(x + j, stride - 1);
      const int p = (plane[yy * stride + xx] >> cs) - 128;
      partial[0][i + j] += p;
      partial[1][i + j / 2] += p;
      partial[2][i] += p;
      partial[3][3 + i - j / 2] += p;
      partial[4][7 + i - j] += p;
      partial[5][3 - i / 2 + j] += p;
      partial[6][j] += p;
      partial[7][i / 2 + j] += p;
    }
  int64_t cost[8] = {};
  for (int i = 0; i < 8; i++) {
    cost[2] += partial[2][i] * partial[2][i];
    cost[6] += partial[6][i] * partial[6][i];
  }
  cost[2] *= 105;
  cost[6] *= 105;
  static const int64_t kDiv[8] = {0, 840, 420, 280, 210, 168, 140, 120};
  for (int i = 0; i < 7; i++) {
    cost[0] += (partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) * kDiv[i + 1];
    cost[4] += (partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) * kDiv[i + 1];
  }
  cost[0] += partial[0][7] * partial[0][7] * 105;
  cost[4] += partial[4][7] * partial[4][7] * 105;
  for (int s = 1; s < 8; s += 2) {
    for (int i = 0; i < 5; i++) cost[s] += partial[s][3 + i] * partial[s][3 + i] * 105;
    for (int i = 0; i < 3; i++)
      cost[s] += (partial[s][i] * partial[s][i] + partial[s][10 - i] * partial[s][10 - i]) * kDiv[2 * i + 2];
  }
  int best_dir = 0;
  int64_t best = cost[0];
  for (int d = 0; d < 8; d++)
    if (cost[d] > best) {
      best = cost[d];
      best_dir = d;
    }
  *dir = best_dir;
  *var = (int)((best - cost[(best_dir + 4) & 7]) >> 10);
}

int adjust_pri(int pri, int var) {
  if (var == 0) return 0;
  const int vs = var >> 6;
  const int l = vs != 0 ? std::min(log2_floor(vs), 12) : 0;
  return (pri * (4 + l) + 8) >> 4;
}

int sample(const uint16_t* plane, int stride, int rows, int x, int y) {
  if (x < 0 || y < 0 || x >= stride || y >= rows) return kVeryLarge;
  return plane[y * stride + x];
}

// cdef_filter_block (generic body): one bw x bh block at (x, y) of src into
// out[i * bw + j].
void filter_block(const uint16_t* src, int stride, int rows, int x, int y, int bw, int bh, int pri, int sec, int dir,
                  int damping, int bd, int32_t* out) {
  const int cs = bd - 8;
  const int pri_damping = std::max(damping, 1), sec_damping = std::max(damping, 1);
  const int* pri_taps = kPriTaps[(pri >> cs) & 1];
  const bool en_p = pri != 0, en_s = sec != 0, clip = en_p && en_s;
  const int maxv = (1 << bd) - 1;
  for (int i = 0; i < bh; i++)
    for (int j = 0; j < bw; j++) {
      const int cx = x + j, cy = y + i;
      int32_t& o = out[i * bw + j];
      if (cx >= stride || cy >= rows) {
        o = -1;
        continue;
      }
      const int centre = src[cy * stride + cx];
      o = centre;
      if (centre == kVeryLarge) continue;
      int sum = 0, mn = centre, mx = centre;
      for (int k = 0; k < 2; k++) {
        if (en_p) {
          for (int sg = 1; sg >= -1; sg -= 2) {
            const int p = sample(src, stride, rows, cx + sg * kDirs[dir][k][1], cy + sg * kDirs[dir][k][0]);
            if (p != kVeryLarge) {
              sum += pri_taps[k] * constrain(p - centre, pri, pri_damping);
              if (clip) {
                mx = std::max(mx, p);
                mn = std::min(mn, p);
              }
            }
          }
        }
        if (en_s) {
          for (int doff : {2, 6}) {
            const int sd = (dir + doff) & 7;
            for (int sg = 1; sg >= -1; sg -= 2) {
              const int p = sample(src, stride, rows, cx + sg * kDirs[sd][k][1], cy + sg * kDirs[sd][k][0]);
              if (p != kVeryLarge) {
                sum += kSecTaps[k] * constrain(p - centre, sec, sec_damping);
                if (clip) {
                  mx = std::max(mx, p);
                  mn = std::min(mn, p);
                }
              }
            }
          }
        }
      }
      int v = centre + ((8 + sum - (sum < 0)) >> 4);
      if (clip) v = std::min(std::max(v, mn), mx);
      o = std::min(std::max(v, 0), maxv);
    }
}

// AVX2 weighted_sse (src/avx/rd.rs:767-848): w, h multiples of 4, w <= 8.
const float kWRawMean = 0.4625f;
float wsse_avx2(const int32_t* err, int w, int h) {
  const float A = 0.5f, B = 0.6532815f, C = 0.27059805f;
  const float D[4][4] = {{A, A, A, A}, {B, C, -C, -B}, {A, -A, -A, A}, {C, -B, B, -C}};
  const float DC = 1.8f / kWRawMean, DIAG = 0.8f / kWRawMean, AXIS = 0.4f / kWRawMean, HF = 0.2f / kWRawMean,
              AC1 = 1.0f / kWRawMean;
  const float W[4][4] = {{DC, AC1, AXIS, HF}, {AC1, DIAG, HF, HF}, {AXIS, HF, HF, HF}, {HF, HF, HF, HF}};
  float total[4][8] = {};
  const int pairs = w / 8 * 8;
  for (int r0 = 0; r0 < h; r0 += 4)
    for (int c0 = 0; c0 < pairs; c0 += 8) {
      float rows[4][8];
      for (int i = 0; i < 4; i++)
        for (int ln = 0; ln < 8; ln++) rows[i][ln] = (float)err[(r0 + i) * w + c0 + ln];
      for (int k = 0; k < 4; k++) {
        float t[8];
        for (int ln = 0; ln < 8; ln++) {
          float v = rows[0][ln] * D[k][0];
          v = fmaf(rows[1][ln], D[k][1], v);
          v = fmaf(rows[2][ln], D[k][2], v);
          v = fmaf(rows[3][ln], D[k][3], v);
          t[ln] = v;
        }
        for (int ln = 0; ln < 8; ln++) {
          const int hb = ln & 4, l = ln & 3;
          float c = D[l][0] * t[hb + 0];
          c = fmaf(D[l][1], t[hb + 1], c);
          c = fmaf(D[l][2], t[hb + 2], c);
          c = fmaf(D[l][3], t[hb + 3], c);
          total[k][ln] = fmaf(W[k][l] * c, c, total[k][ln]);
        }
      }
    }
  float sum[4];
  for (int l = 0; l < 4; l++) {
    const float a = (total[0][l] + total[0][4 + l]) + (total[1][l] + total[1][4 + l]);
    sum[l] = a + ((total[2][l] + total[2][4 + l]) + (total[3][l] + total[3][4 + l]));
  }
  if (pairs < w) {
    const int c0 = pairs;
    for (int r0 = 0; r0 < h; r0 += 4) {
      float rows[4][4];
      for (int i = 0; i < 4; i++)
        for (int ln = 0; ln < 4; ln++) rows[i][ln] = (float)err[(r0 + i) * w + c0 + ln];
      for (int k = 0; k < 4; k++) {
        float t[4];
        for (int ln = 0; ln < 4; ln++) {
          float v = rows[0][ln] * D[k][0];
          v = fmaf(rows[1][ln], D[k][1], v);
          v = fmaf(rows[2][ln], D[k][2], v);
          v = fmaf(rows[3][ln], D[k][3], v);
          t[ln] = v;
        }
        for (int l = 0; l < 4; l++) {
          float c = D[l][0] * t[0];
          c = fmaf(D[l][1], t[1], c);
          c = fmaf(D[l][2], t[2], c);
          c = fmaf(D[l][3], t[3], c);
          sum[l] = fmaf(W[k][l] * c, c, sum[l]);
        }
      }
    }
  }
  const float p0 = sum[0] + sum[2], p1 = sum[1] + sum[3];
  return p0 + p1;
}

int64_t wsse_err(const int32_t* err, int w, int h) { return (int64_t)roundf(wsse_avx2(err, w, h) * 1.0f); }

int64_t sat_mul(int64_t a, int64_t b) {
  __int128 r = (__int128)a * b;
  if (r > INT64_MAX) return INT64_MAX;
  if (r < INT64_MIN) return INT64_MIN;
  return (int64_t)r;
}

int cand_index(int pri, int sec) {
  int pi = 0, si = 0;
  for (int i = 0; i < 4; i++)
    if (kCandPri[i] == pri) pi = i;
  for (int i = 0; i < 3; i++)
    if (kCandSec[i] == sec) si = i;
  return si * 4 + pi;
}

float mode_lambda_weight(int q, int sub) {
  const float scale = sub == 2 ? 0.8f : (sub == 1 ? 0.65f : 0.6f);
  int wi = ((255 - q) * 3) / 4;
  wi = std::min(std::max(wi, 0), 72) + 128;
  const float w = (float)wi * (1.0f / 128.0f);
  const float lo_floor = 0.0f, lo_full = 72.0f, lo_w = 3.0f;
  if (sub == 1 || lo_full <= lo_floor) return w * scale;
  float r = ((float)q - lo_floor) / (lo_full - lo_floor);
  r = std::min(std::max(r, 0.0f), 1.0f);
  return (lo_w + (w - lo_w) * r) * scale;
}

float frame_lambda_d(int qidx, int bd, int sub_x, int sub_y) {
  const int sub = (sub_x == 1 && sub_y == 1) ? 2 : (sub_x == 1 ? 1 : 0);
  mt_quant q;
  or_quant_init((uint8_t)qidx, (uint8_t)bd, 15, &q);
  const float dc = (float)q.dc_q;
  const float dc8 = dc / (float)(1u << (std::max(bd, 8) - 8));
  const float kf = 3.3f + 0.0015f * dc8;
  const float mlq = 0.009005174719460433f * 1.0f * dc * dc * kf;
  return mlq * mode_lambda_weight(qidx, sub) / 2.775f;
}

using Table = std::vector<std::array<int64_t, 12>>;

}  // namespace

extern "C" int or_cdef_frame(uint16_t* py, uint16_t* pu, uint16_t* pv, const uint16_t* sy, const uint16_t* su,
                             const uint16_t* sv, const uint8_t* skip8, const mt_cdef_params* prm,
                             mt_cdef_decision* out, uint8_t* grid_out, int64_t* luma_tab_out, int64_t* u_tab_out,
                             int64_t* v_tab_out, uint8_t* dirs_out, int32_t* vars_out) {
  const int w8 = prm->w8, h8 = prm->h8, disp_w = prm->disp_w, disp_h = prm->disp_h;
  const int sub_x = prm->sub_x, sub_y = prm->sub_y, bd = prm->bd;
  const bool mono = prm->mono != 0;
  const int cw8 = w8 >> sub_x, ch8 = h8 >> sub_y;
  const int signaled_damping = 3 + std::min(prm->base_q_idx / 64, 3);
  const int damping = signaled_damping + (bd - 8);
  const int cw_vis = (disp_w + (1 << sub_x) - 1) >> sub_x, ch_vis = (disp_h + (1 << sub_y) - 1) >> sub_y;
  const int cs = bd - 8;
  const int64_t margin = 40;
  const int64_t gate_thresh = 15000;

  const int nbx = (w8 + 7) / 8, nby = (h8 + 7) / 8;
  std::vector<int> ldirs(nbx * nby, 0), lvars(nbx * nby, 0);
  for (int by = 0; by < nby; by++)
    for (int bx = 0; bx < nbx; bx++)
      if (bx * 8 < w8 && by * 8 < h8) direction(py, w8, h8, bx * 8, by * 8, bd, &ldirs[by * nbx + bx], &lvars[by * nbx + bx]);
  if (dirs_out)
    for (int i = 0; i < nbx * nby; i++) dirs_out[i] = (uint8_t)ldirs[i];
  if (vars_out)
    for (int i = 0; i < nbx * nby; i++) vars_out[i] = lvars[i];
  std::vector<char> lskip(nbx * nby);
  for (int i = 0; i < nbx * nby; i++) lskip[i] = skip8[i] != 0;

  const int uc = (w8 + 63) / 64, ur = (h8 + 63) / 64, n_units = uc * ur;
  out->bits = -1;
  out->damping = signaled_damping;
  out->n_strengths = 0;
  out->unit_cols = uc;
  out->unit_rows = ur;
  memset(out->strengths, 0, sizeof(out->strengths));
  if (grid_out) memset(grid_out, 0, n_units);

  // Unit tables (all 12 candidates, needed for the comparison even when unused).
  Table luma_all(n_units), u_all(n_units), v_all(n_units);
  for (auto& t : luma_all) t.fill(0);
  for (auto& t : u_all) t.fill(0);
  for (auto& t : v_all) t.fill(0);
  {
    int32_t cand[64], err[64];
    for (int y = 0; y < h8; y += 8) {
      if (y >= disp_h) break;
      for (int x = 0; x < w8; x += 8) {
        const int bi = (y / 8) * nbx + x / 8;
        if (lskip[bi] || x >= disp_w) continue;
        const bool whole = x + 8 <= disp_w && y + 8 <= disp_h;
        const int vw = std::min(disp_w - x, 8), vh = std::min(disp_h - y, 8);
        auto& acc = luma_all[(y / 64) * uc + x / 64];
        for (int si = 0; si < 3; si++)
          for (int pi = 0; pi < 4; pi++) {
            const int pri = kCandPri[pi], sec = kCandSec[si];
            const int apri = adjust_pri(pri << cs, lvars[bi]);
            filter_block(py, w8, h8, x, y, 8, 8, apri, sec << cs, pri == 0 ? 0 : ldirs[bi], damping, bd, cand);
            int64_t d = 0;
            if (whole) {
              for (int i = 0; i < 8; i++)
                for (int j = 0; j < 8; j++) err[i * 8 + j] = cand[i * 8 + j] - sy[(y + i) * w8 + x + j];
              d = wsse_err(err, 8, 8);
            } else {
              for (int i = 0; i < vh; i++)
                for (int j = 0; j < vw; j++) {
                  const int64_t e = cand[i * 8 + j] - (int64_t)sy[(y + i) * w8 + x + j];
                  d += e * e;
                }
            }
            acc[si * 4 + pi] += d;
          }
      }
    }
  }
  const int uv_dir_422[8] = {7, 0, 2, 4, 5, 6, 6, 6};
  auto uv_dir = [&](int d) { return (sub_x == 1 && sub_y == 0) ? uv_dir_422[d] : d; };
  const int chroma_damping = damping - 1;
  const int cbw = 8 >> sub_x, cbh = 8 >> sub_y;
  if (!mono) {
    for (int pl = 0; pl < 2; pl++) {
      const uint16_t* rec = pl == 0 ? pu : pv;
      const uint16_t* src = pl == 0 ? su : sv;
      Table& tab = pl == 0 ? u_all : v_all;
      int32_t cand[64], err[64];
      for (int lby = 0; lby < nby; lby++) {
        const int cy = (lby * 8) >> sub_y;
        if (cy >= ch_vis) break;
        for (int lbx = 0; lbx < nbx; lbx++) {
          const int bi = lby * nbx + lbx;
          const int cx = (lbx * 8) >> sub_x;
          if (lskip[bi] || cx >= cw_vis) continue;
          const int vw = std::min(cw_vis - cx, cbw), vh = std::min(ch_vis - cy, cbh);
          auto& acc = tab[(lby / 8) * uc + lbx / 8];
          for (int si = 0; si < 3; si++)
            for (int pi = 0; pi < 4; pi++) {
              const int pri = kCandPri[pi], sec = kCandSec[si];
              filter_block(rec, cw8, ch8, cx, cy, cbw, cbh, pri << cs, sec << cs, pri == 0 ? 0 : uv_dir(ldirs[bi]),
                           chroma_damping, bd, cand);
              int64_t d = 0;
              if (vw == cbw && vh == cbh) {
                for (int i = 0; i < cbh; i++)
                  for (int j = 0; j < cbw; j++) err[i * cbw + j] = cand[i * cbw + j] - src[(cy + i) * cw8 + cx + j];
                d = wsse_err(err, cbw, cbh);
              } else {
                for (int i = 0; i < vh; i++)
                  for (int j = 0; j < vw; j++) {
                    const int64_t e = cand[i * cbw + j] - (int64_t)src[(cy + i) * cw8 + cx + j];
                    d += e * e;
                  }
              }
              acc[si * 4 + pi] += d;
            }
        }
      }
    }
  }
  if (luma_tab_out)
    for (int u = 0; u < n_units; u++)
      for (int c = 0; c < 12; c++) luma_tab_out[u * 12 + c] = luma_all[u][c];
  if (u_tab_out && !mono)
    for (int u = 0; u < n_units; u++)
      for (int c = 0; c < 12; c++) u_tab_out[u * 12 + c] = u_all[u][c];
  if (v_tab_out && !mono)
    for (int u = 0; u < n_units; u++)
      for (int c = 0; c < 12; c++) v_tab_out[u * 12 + c] = v_all[u][c];

  // ---- the decision (src/coder/frame_cdef.rs:116-520) ----
  std::vector<char> signaled(n_units, 0);
  for (int by = 0; by < nby; by++)
    for (int bx = 0; bx < nbx; bx++)
      if (!lskip[by * nbx + bx]) signaled[(by / 8) * uc + bx / 8] = 1;
  int n_sig = 0;
  for (char s : signaled) n_sig += s;
  if (n_sig == 0) return MT_OK;
  std::vector<int64_t> dv_sum(n_units, 0), dv_cnt(n_units, 0);
  for (int by = 0; by < nby; by++)
    for (int bx = 0; bx < nbx; bx++)
      if (!lskip[by * nbx + bx]) {
        const int u = (by / 8) * uc + bx / 8;
        dv_sum[u] += lvars[by * nbx + bx];
        dv_cnt[u] += 1;
      }
  int n_trusted = 0;
  for (int u = 0; u < n_units; u++)
    if (gate_thresh == 0 || dv_sum[u] / std::max<int64_t>(dv_cnt[u], 1) >= gate_thresh) n_trusted++;

  auto luma_tab = [&](int pri, int sec) {
    std::vector<int64_t> t(n_units);
    const int c = cand_index(pri, sec);
    for (int u = 0; u < n_units; u++) t[u] = luma_all[u][c];
    return t;
  };
  auto clears = [&](int64_t off, int64_t on) -> int64_t {
    const int64_t thr = off - sat_mul(off, margin) / 1000;
    return on < thr ? off - on : 0;
  };
  std::vector<std::pair<int, int>> cands = {{0, 0}};
  std::vector<std::vector<int64_t>> ly = {luma_tab(0, 0)};
  const std::vector<int64_t> luma_off = ly[0];
  if (prm->slow) {
    const int pri_list[3] = {1, 2, 4};
    std::vector<std::pair<int64_t, int>> ranked;
    std::vector<std::vector<int64_t>> tabs;
    for (int i = 0; i < 3; i++) tabs.push_back(luma_tab(pri_list[i], 0));
    for (int i = 0; i < 3; i++) {
      int64_t g = 0;
      for (int u = 0; u < n_units; u++) g += clears(luma_off[u], tabs[i][u]);
      ranked.push_back({g, i});
    }
    for (int i = 0; i < 3; i++) {
      cands.push_back({pri_list[i], 0});
      ly.push_back(tabs[i]);
    }
    std::stable_sort(ranked.begin(), ranked.end(), [](const std::pair<int64_t, int>& a, const std::pair<int64_t, int>& b) {
      if (a.first != b.first) return a.first > b.first;
      return a.second < b.second;
    });
    std::vector<std::pair<int, int>> stage_b;
    for (int sec : {1, 2}) {
      stage_b.push_back({0, sec});
      for (size_t r = 0; r < ranked.size() && r < 4; r++)
        if (ranked[r].first > 0) stage_b.push_back({pri_list[ranked[r].second], sec});
    }
    for (auto& ps : stage_b) {
      cands.push_back(ps);
      ly.push_back(luma_tab(ps.first, ps.second));
    }
  } else {
    for (int pri : {0, 1, 2, 4})
      for (int sec : {0, 1, 2}) {
        if (pri == 0 && sec == 0) continue;
        cands.push_back({pri, sec});
        ly.push_back(luma_tab(pri, sec));
      }
  }
  std::vector<std::pair<int, int>> c_cands;
  std::vector<std::vector<int64_t>> lc;
  if (mono) {
    c_cands = {{0, 0}};
    lc = {std::vector<int64_t>(n_units, 0)};
  } else {
    for (auto& ps : cands) {
      const int c = cand_index(ps.first, ps.second);
      std::vector<int64_t> t(n_units);
      for (int u = 0; u < n_units; u++) t[u] = u_all[u][c] + v_all[u][c];
      lc.push_back(t);
    }
    c_cands = cands;
  }
  std::vector<int64_t> d_off(n_units), thr(n_units);
  for (int u = 0; u < n_units; u++) {
    d_off[u] = luma_off[u] + lc[0][u];
    thr[u] = d_off[u] - sat_mul(d_off[u], margin) / 1000;
  }
  const size_t nc = c_cands.size(), n_pairs = cands.size() * nc;
  auto d_pair = [&](size_t p, int u) { return ly[p / nc][u] + lc[p % nc][u]; };
  size_t global_entry = 0;
  int64_t prefix_tot[4] = {INT64_MAX, INT64_MAX, INT64_MAX, INT64_MAX};
  for (size_t p = 0; p < n_pairs; p++) {
    int64_t t = 0;
    for (int u = 0; u < n_units; u++) t += signaled[u] ? d_pair(p, u) : d_off[u];
    if (t < prefix_tot[0]) {
      prefix_tot[0] = t;
      global_entry = p;
    }
  }
  std::vector<int64_t> cur_min = d_off;
  std::vector<size_t> entries = {0};
  while (entries.size() < 8) {
    size_t best_p = 0;
    int64_t best_tot = INT64_MAX;
    for (size_t p = 0; p < n_pairs; p++) {
      int64_t tot = 0;
      for (int u = 0; u < n_units; u++) {
        if (!signaled[u]) {
          tot += d_off[u];
          continue;
        }
        const int64_t b = std::min(cur_min[u], d_pair(p, u));
        tot += b >= thr[u] ? d_off[u] : b;
      }
      if (tot < best_tot) {
        best_tot = tot;
        best_p = p;
      }
    }
    entries.push_back(best_p);
    for (int u = 0; u < n_units; u++) cur_min[u] = std::min(cur_min[u], d_pair(best_p, u));
    const size_t n = entries.size();
    if ((n & (n - 1)) == 0 && n <= 8) prefix_tot[__builtin_ctzll(n)] = best_tot;
  }
  auto strength_mag = [&](size_t p) {
    return cands[p / nc].first + cands[p / nc].second + c_cands[p % nc].first + c_cands[p % nc].second;
  };
  auto assign = [&](const size_t* set, size_t nset, std::vector<uint8_t>* grid) -> int64_t {
    int z_in_set = -1;
    for (size_t e = 0; e < nset; e++)
      if (set[e] == 0) {
        z_in_set = (int)e;
        break;
      }
    int64_t total = 0;
    grid->assign(n_units, 0);
    for (int u = 0; u < n_units; u++) {
      if (!signaled[u]) {
        total += d_off[u];
        continue;
      }
      bool have = false;
      int pm = 0;
      int64_t pd = 0;
      size_t pe = 0;
      int64_t rb_d = INT64_MAX;
      size_t rb_e = 0;
      for (size_t e = 0; e < nset; e++) {
        const int64_t d = d_pair(set[e], u);
        if (d < rb_d) {
          rb_d = d;
          rb_e = e;
        }
        if (d < thr[u]) {
          const int mag = strength_mag(set[e]);
          if (!have || mag < pm || (mag == pm && d < pd)) {
            have = true;
            pm = mag;
            pd = d;
            pe = e;
          }
        }
      }
      if (have) {
        total += pd;
        (*grid)[u] = (uint8_t)pe;
      } else if (z_in_set >= 0) {
        total += d_off[u];
        (*grid)[u] = (uint8_t)z_in_set;
      } else {
        total += rb_d;
        (*grid)[u] = (uint8_t)rb_e;
      }
    }
    return total;
  };
  const float lambda = frame_lambda_d(prm->base_q_idx, bd, sub_x, sub_y);
  int64_t total_off = 0;
  for (int u = 0; u < n_units; u++) total_off += d_off[u];
  const float cost_off = (float)total_off;
  const float per_entry_bits = mono ? 6.0f : 12.0f;
  int best_bits = -1;
  float best_cost = cost_off;
  std::vector<uint8_t> g;
  for (int b = 0; b <= 3; b++) {
    const int nb = 1 << b;
    const int64_t total = b == 0 ? prefix_tot[0] : assign(entries.data(), nb, &g);
    if (total == INT64_MAX) continue;
    if (b == 0 && (global_entry == 0 || n_trusted * 4 < n_sig * 3 || total >= total_off - sat_mul(total_off, margin) / 1000))
      continue;
    const float bits_f = per_entry_bits * (float)(nb - 1) + (float)b * (float)n_sig;
    const float cost = (float)total + lambda * bits_f;
    if (cost < best_cost) {
      best_cost = cost;
      best_bits = b;
    }
  }
  if (best_bits < 0) return MT_OK;
  const int nb = 1 << best_bits;
  std::vector<size_t> set;
  if (best_bits == 0)
    set = {global_entry};
  else
    set.assign(entries.begin(), entries.begin() + nb);
  std::vector<uint8_t> grid(n_units, 0);
  if (best_bits > 0) assign(set.data(), set.size(), &grid);
  out->bits = best_bits;
  out->n_strengths = (int)set.size();
  for (size_t e = 0; e < set.size(); e++) {
    out->strengths[e][0] = (uint8_t)cands[set[e] / nc].first;
    out->strengths[e][1] = (uint8_t)cands[set[e] / nc].second;
    out->strengths[e][2] = (uint8_t)c_cands[set[e] % nc].first;
    out->strengths[e][3] = (uint8_t)c_cands[set[e] % nc].second;
  }
  if (grid_out && best_bits > 0) memcpy(grid_out, grid.data(), n_units);

  // ---- apply (src/coder/frame_cdef.rs:960-1125) from the pre-CDEF snapshots ----
  std::vector<int> uy_p(n_units), uy_s(n_units), uuv_p(n_units), uuv_s(n_units);
  bool any_y = false, any_uv = false;
  for (int u = 0; u < n_units; u++) {
    const uint8_t* st = out->strengths[grid[u]];
    uy_p[u] = st[0];
    uy_s[u] = st[1];
    uuv_p[u] = st[2];
    uuv_s[u] = st[3];
    any_y |= (st[0] | st[1]) != 0;
    any_uv |= (st[2] | st[3]) != 0;
  }
  int32_t blk[64];
  if (any_y) {
    std::vector<uint16_t> snap(py, py + (size_t)w8 * h8);
    for (int y = 0; y < h8; y += 8)
      for (int x = 0; x < w8; x += 8) {
        const int bi = (y / 8) * nbx + x / 8;
        if (lskip[bi]) continue;
        const int u = (y / 64) * uc + x / 64;
        const int pri = uy_p[u], sec = uy_s[u];
        if (pri == 0 && sec == 0) continue;
        const int dir = pri == 0 ? 0 : ldirs[bi];
        filter_block(snap.data(), w8, h8, x, y, 8, 8, adjust_pri(pri << cs, lvars[bi]), sec << cs, dir, damping, bd,
                     blk);
        for (int i = 0; i < 8 && y + i < h8; i++)
          for (int j = 0; j < 8 && x + j < w8; j++) py[(y + i) * w8 + x + j] = (uint16_t)blk[i * 8 + j];
      }
  }
  if (!mono && any_uv) {
    for (int pl = 0; pl < 2; pl++) {
      uint16_t* rec = pl == 0 ? pu : pv;
      std::vector<uint16_t> snap(rec, rec + (size_t)cw8 * ch8);
      const int nbands = (ch8 + cbh - 1) / cbh;
      for (int lby = 0; lby < nbands && lby < nby; lby++) {
        const int cy = (lby * 8) >> sub_y;
        for (int lbx = 0; lbx < nbx; lbx++) {
          const int bi = lby * nbx + lbx;
          if (lskip[bi]) continue;
          const int u = (lby / 8) * uc + lbx / 8;
          const int pri = uuv_p[u], sec = uuv_s[u];
          if (pri == 0 && sec == 0) continue;
          const int cx = (lbx * 8) >> sub_x;
          if (cx >= cw8 || cy >= ch8) continue;
          const int dir = pri == 0 ? 0 : uv_dir(ldirs[bi]);
          filter_block(snap.data(), cw8, ch8, cx, cy, cbw, cbh, pri << cs, sec << cs, dir, chroma_damping, bd, blk);
          for (int i = 0; i < cbh && cy + i < ch8; i++)
            for (int j = 0; j < cbw && cx + j < cw8; j++) rec[(cy + i) * cw8 + cx + j] = (uint16_t)blk[i * cbw + j];
        }
      }
    }
  }
  return MT_OK;
}

extern "C" float or_weighted_sse(const int32_t* err, int32_t w, int32_t h) { return wsse_avx2(err, w, h); }

// rd_sse.rs:449-475 sse_recon with the SrcBlock visibility (rd_sse.rs:61-167)
// and weighted_dist (rd_sse.rs:244-271): plain SSE, or round(wsse * scale)
// over the displayed part padded to whole 4x4 tiles.
extern "C" int or_sse_recon(const uint16_t* src, int32_t stride, int32_t vis_w, int32_t vis_h, int32_t bd,
                            const uint16_t* pos, const int32_t* pred, const int32_t* resid, int32_t n, int32_t w,
                            int32_t h, float scale, int64_t* out) {
  const int32_t maxv = (1 << bd) - 1;
  for (int b = 0; b < n; b++) {
    const int px = pos[2 * b], py = pos[2 * b + 1];
    const int vw = std::min(std::max(vis_w - px, 0), w), vh = std::min(std::max(vis_h - py, 0), h);
    const int32_t* pr = pred + (size_t)b * w * h;
    const int32_t* rs = resid ? resid + (size_t)b * w * h : nullptr;
    auto err = [&](int x, int y) {
      const int i = y * w + x;
      return (int32_t)src[(size_t)(py + y) * stride + px + x] -
             std::min(std::max(pr[i] + (rs ? rs[i] : 0), 0), maxv);
    };
    if (vw == 0 || vh == 0) {
      out[b] = 0;
      continue;
    }
    if (scale > 0.0f) {
      const int pw = (vw + 3) & ~3, ph = (vh + 3) & ~3;
      std::vector<int32_t> buf((size_t)pw * ph, 0);
      for (int y = 0; y < vh; y++)
        for (int x = 0; x < vw; x++) buf[(size_t)y * pw + x] = err(x, y);
      const float d = wsse_avx2(buf.data(), pw, ph);
      out[b] = (int64_t)roundf(d * scale);
    } else {
      int64_t s = 0;
      for (int y = 0; y < vh; y++)
        for (int x = 0; x < vw; x++) {
          const int64_t v = err(x, y);
          s += v * v;
        }
      out[b] = s;
    }
  }
  return MT_OK;
}
extern "C" float or_cdef_frame_lambda(int32_t qidx, int32_t bd, int32_t sub_x, int32_t sub_y) {
  return frame_lambda_d(qidx, bd, sub_x, sub_y);
}
