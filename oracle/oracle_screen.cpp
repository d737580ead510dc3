// Oracle (test infrastructure, the CPU checker of the CUDA path): the
// screen-content frame gate, restated from the reference in its serial order.
//
//   src/coder/screen_gate.rs:64-273  screen_frame_gate (stage 1 pre-screen, stage 2 copy gains)
//   src/coder/palette.rs:651-690     block_color_histogram (None when flat or > 64 values)
//   src/coder/block64.rs:123-131     ibc_mix; :177-188 hash8; :190-266 LossyIbcIndex::build
//                                    (direct window hashes: the reference's rolling form equals them,
//                                    rolling_hash_matches_direct); :271-329 anchor / candidates
//   src/obu.rs:306-330               loop_filter_levels (luma level)
//   src/tuning.rs:932-939            ibc_gate_beta 32, ibc_gate_dv 1, ibc_gate_prescreen 0.02,
//                                    screen_few_share 0.10
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../maroontree_b200/csrc/av1_tables.h"
#include "oracle.h"

namespace {

constexpr uint32_t kHp = 0x9E3779B1u, kHq = 0x85EBCA77u;

uint32_t ibc_mix(uint32_t h) {
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  return h ^ (h >> 16);
}

uint32_t hash8(const uint16_t* luma, int w, int x, int y) {
  uint32_t c = 0;
  for (int j = 0; j < 8; j++) {
    uint32_t r = 0;
    for (int i = 0; i < 8; i++) r = r * kHp + ((uint32_t)luma[(size_t)(y + j) * w + x + i] + 1);
    c = c * kHq + r;
  }
  return ibc_mix(c);
}

// block_color_histogram: false for a flat block or one of more than 64 values;
// else the distinct count and the value span.
bool color_hist(const uint16_t* src, int stride, int px, int py, int w, int h, int* distinct, int* span) {
  std::vector<uint8_t> seen(4096, 0);
  int n = 0, lo = 1 << 30, hi = -1;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int v = src[(size_t)(py + y) * stride + px + x] & 4095;
      if (!seen[v]) {
        seen[v] = 1;
        if (++n > 64) return false;
      }
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
  if (n < 2) return false;
  *distinct = n;
  *span = hi - lo;
  return true;
}

struct IbcIndex {
  std::vector<std::pair<uint32_t, uint32_t>> entries;  // (hash, y << 16 | x), bucketed by hash >> 16
  std::vector<uint32_t> offsets;
};

// LossyIbcIndex::build: every window origin on the chroma-parity grid, bucketed
// by the top 16 hash bits in raster order (a stable counting sort).
IbcIndex build_index(const uint16_t* luma, int w, int h, int sub_x, int sub_y) {
  IbcIndex ix;
  ix.offsets.assign((1 << 16) + 1, 0);
  if (w < 16 || h < 16) return ix;
  const int nx = w - 7, ny = h - 7;
  std::vector<std::pair<uint32_t, uint32_t>> hashes;
  for (int y = 0; y < ny; y += 1 << sub_y)
    for (int x = 0; x < nx; x += 1 << sub_x) {
      const uint32_t hh = hash8(luma, w, x, y);
      hashes.emplace_back(hh, ((uint32_t)y << 16) | (uint32_t)x);
      ix.offsets[(hh >> 16) + 1]++;
    }
  for (size_t i = 1; i < ix.offsets.size(); i++) ix.offsets[i] += ix.offsets[i - 1];
  std::vector<uint32_t> cursor(ix.offsets.begin(), ix.offsets.end() - 1);
  ix.entries.resize(hashes.size());
  for (const auto& e : hashes) ix.entries[cursor[e.first >> 16]++] = e;
  return ix;
}

uint64_t sad8(const uint16_t* luma, int w8, int x, int y) {
  uint64_t e = 0;
  for (int j = 0; j < 8; j++) {
    const uint16_t* row = luma + (size_t)(y + j) * w8 + x;
    for (int i = 0; i + 1 < 8; i++) {
      const uint64_t d = (uint64_t)std::abs((int)row[i] - (int)row[i + 1]);
      e += d * d;
    }
    if (j > 0) {
      const uint16_t* up = row - w8;
      for (int i = 0; i < 8; i++) {
        const uint64_t d = (uint64_t)std::abs((int)row[i] - (int)up[i]);
        e += d * d;
      }
    }
  }
  return e;
}

uint16_t ac_q(int q, int bd) {
  const uint16_t* t = bd == 10 ? MT_AC_QLOOKUP_10 : (bd == 12 ? MT_AC_QLOOKUP_12 : MT_AC_QLOOKUP_8);
  return t[q];
}

// loop_filter_levels(q, sub).0 with lf_level_scale 1 (src/obu.rs:314, src/tuning.rs:765).
int lf_level_y(int q) {
  const float v = (float)(q / 8) * 1.0f;
  return std::min(std::max((int)roundf(v), 0), 40);
}

}  // namespace

extern "C" {

int or_screen_gate(const uint16_t* luma, const mt_screen_gate_params* p, mt_screen_gate_result* out) {
  memset(out, 0, sizeof(*out));
  const int w8 = p->w8, h8 = p->h8, bd = p->bd;
  const int n8x = w8 / 8, n8y = h8 / 8;
  if (n8x < 2 || n8y < 2) return MT_OK;
  const int n16x = w8 / 16, n16y = h8 / 16;
  const int span_min = 64 << (bd - 8);
  std::vector<uint8_t> few((size_t)n16x * n16y, 0);
  uint32_t lenient = 0, few16 = 0, nonflat = 0, dup = 0;
  std::unordered_set<uint32_t> seen;
  for (int row = 0; row < n16y; row++)
    for (int col = 0; col < n16x; col++) {
      int nd, span;
      bool is_few = false;
      if (color_hist(luma, w8, col * 16, row * 16, 16, 16, &nd, &span) && span >= span_min) {
        lenient += nd <= 16;
        is_few = nd <= 8;
      }
      few[(size_t)row * n16x + col] = is_few;
      few16 += is_few;
      static const int subs[4][2] = {{0, 0}, {8, 0}, {0, 8}, {8, 8}};
      for (const auto& s : subs) {
        const int x = col * 16 + s[0], y = row * 16 + s[1];
        const uint16_t first = luma[(size_t)y * w8 + x];
        bool flat = true;
        for (int j = 0; j < 8 && flat; j++)
          for (int i = 0; i < 8; i++)
            if (luma[(size_t)(y + j) * w8 + x + i] != first) {
              flat = false;
              break;
            }
        if (!flat) {
          nonflat++;
          if (!seen.insert(hash8(luma, w8, x, y)).second) dup++;
        }
      }
    }
  const uint32_t t16 = (uint32_t)std::max(n16x * n16y, 1);
  const float total16 = (float)t16;
  const float few_share = (float)few16 / total16;
  out->few_colour = few_share >= 0.10f;
  out->blocks16 = (uint32_t)(n16x * n16y);
  out->few16 = few16;
  out->lenient16 = lenient;
  out->nonflat8 = nonflat;
  out->dup8 = dup;
  const float dup8 = (float)dup / (4.0f * total16);
  const float lenient_share = (float)lenient / total16;
  if (lenient_share < 0.02f && dup8 < 0.02f) return MT_OK;
  out->copy_stage = 1;
  const IbcIndex index = build_index(luma, w8, h8, p->sub_x, p->sub_y);
  const float acq = (float)ac_q(p->base_q_idx, bd);
  const float dvf = 1.0f * (acq * acq);
  const uint64_t dv_cost = dvf >= 18446744073709551616.0f ? UINT64_MAX : (uint64_t)dvf;
  uint64_t gain = 0, photo = 0;
  uint32_t copied = 0;
  static const int subs[4][2] = {{0, 0}, {8, 0}, {0, 8}, {8, 8}};
  for (int row = 0; row < n16y; row++) {
    const int py = row * 16;
    for (int col = 0; col < n16x; col++) {
      const int px = col * 16;
      uint64_t mass = 0;
      for (const auto& s : subs) mass += sad8(luma, w8, px + s[0], py + s[1]);
      if (mass == 0) continue;
      uint64_t best = UINT64_MAX;
      for (const auto& s : subs) {
        const int sx = px + s[0], sy = py + s[1];
        // candidates(luma, w8, sx, sy, 8, sy): the anchor of an 8x8 is itself.
        const uint32_t want = hash8(luma, w8, sx, sy);
        const uint32_t b = want >> 16;
        const uint32_t s0 = index.offsets[b], e0 = index.offsets[b + 1];
        // partition_point over the bucket, which is in raster order of origins
        const auto* first = index.entries.data() + s0;
        const uint32_t end = s0 + (uint32_t)(std::partition_point(first, index.entries.data() + e0,
                                                                  [&](const std::pair<uint32_t, uint32_t>& e) {
                                                                    return (int)(e.second >> 16) <= sy;
                                                                  }) - first);
        int taken = 0;
        for (uint32_t k = s0; k < end && taken < 3; k++) {
          if (index.entries[k].first != want) continue;
          const int ax = (int)(index.entries[k].second & 0xffff), ay = (int)(index.entries[k].second >> 16);
          const bool earlier = ay + 8 <= sy || (ay <= sy && ax + 8 <= sx);
          if (!earlier) continue;
          bool exact = true;
          for (int j = 0; j < 8 && exact; j++)
            exact = memcmp(luma + (size_t)(ay + j) * w8 + ax, luma + (size_t)(sy + j) * w8 + sx, 16) == 0;
          if (!exact) continue;
          taken++;
          // DV of the whole 16x16 along this anchor's offset.
          if (px + ax < sx || py + ay < sy) continue;
          const int rx = px + ax - sx, ry = py + ay - sy;
          if (rx + 16 > w8 || ry + 16 > h8 || (ry + 16 > py && rx + 16 > px && ry < py + 16 && rx < px + 16))
            continue;
          uint64_t res = 0;
          for (int j = 0; j < 16; j++)
            for (int i = 0; i < 16; i++) {
              const uint64_t d = (uint64_t)std::abs((int)luma[(size_t)(py + j) * w8 + px + i] -
                                                    (int)luma[(size_t)(ry + j) * w8 + rx + i]);
              res += d * d;
            }
          best = std::min(best, res);
          if (best == 0) break;
        }
        if (best == 0) break;
      }
      uint64_t g = 0;
      if (best != UINT64_MAX) {
        g = mass > best ? mass - best : 0;
        g = g > dv_cost ? g - dv_cost : 0;
      }
      if (g > 0) {
        gain += g;
        copied++;
      } else if (!few[(size_t)row * n16x + col]) {
        for (const auto& s : subs) {
          int nd, span;
          const bool text = color_hist(luma, w8, px + s[0], py + s[1], 8, 8, &nd, &span) && nd <= 12 &&
                            span >= span_min;
          if (!text && sad8(luma, w8, px + s[0], py + s[1]) > 0) photo++;
        }
      }
    }
  }
  out->gain = gain;
  out->photo = photo;
  out->copied = copied;
  const double acd = (double)ac_q(p->base_q_idx, bd);
  const int lvl_y = lf_level_y(p->base_q_idx);
  const double loss = lvl_y > 0 ? (double)32.0f * (double)photo * acd : 0.0;
  out->ibc_pays = copied >= 4 && (double)gain > loss;
  return MT_OK;
}

uint32_t or_hash8(const uint16_t* luma, int32_t w, int32_t x, int32_t y) { return hash8(luma, w, x, y); }

}  // extern "C"
