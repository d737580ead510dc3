// Oracle (test-only checker of the CUDA path): recursive filter-intra
// prediction (filter_intra_predict_impl, src/intrapred.rs:473-530, with the
// 4x2-cell pass scalar_filter_intra_cells, :538-565) and the Slow search's
// filter-intra shortlist ranking (rank_filter_intra_modes,
// src/coder/superblock.rs:356-400): all five modes predicted and scored by
// satd_sad_proxy (src/rd_sse.rs:559-589, :1143-1176), sorted by
// (score, mode order).
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "oracle.h"
#include "../maroontree_b200/csrc/av1_tables.h"

extern "C" {

void or_filter_intra_predict(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t w, int32_t h,
                             int32_t mode, int32_t bd, int32_t* out) {
  int32_t buf[33][33];
  const int32_t base = 1 << (bd - 1);
  const bool top = oy > 0, left = ox > 0;
  auto R = [&](int y, int x) -> int32_t { return recon[(size_t)y * stride + x]; };
  buf[0][0] = top ? (left ? R(oy - 1, ox - 1) : R(oy - 1, ox)) : (left ? R(oy, ox - 1) : base);
  for (int x = 0; x < w; x++) buf[0][x + 1] = top ? R(oy - 1, ox + x) : (left ? R(oy, ox - 1) : base - 1);
  for (int y = 0; y < h; y++) buf[y + 1][0] = left ? R(oy + y, ox - 1) : (top ? R(oy - 1, ox) : base + 1);
  const int8_t* taps = MT_INTRA_FILTER_TAPS + mode * 56;
  const int32_t mx = (1 << bd) - 1;
  for (int r = 1; r <= h; r += 2)
    for (int c = 1; c <= w; c += 4) {
      const int32_t p[7] = {buf[r - 1][c - 1], buf[r - 1][c],     buf[r - 1][c + 1], buf[r - 1][c + 2],
                            buf[r - 1][c + 3], buf[r][c - 1], buf[r + 1][c - 1]};
      for (int k = 0; k < 8; k++) {
        int32_t sum = 0;
        for (int i = 0; i < 7; i++) sum += taps[k * 7 + i] * p[i];
        int32_t v = (sum + 8) >> 4;
        buf[r + (k >> 2)][c + (k & 3)] = v < 0 ? 0 : (v > mx ? mx : v);
      }
    }
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) out[y * w + x] = buf[y + 1][x + 1];
}

int or_filter_intra_beam(const uint16_t* src, const uint16_t* recon, int32_t stride, int32_t frame_w, int32_t frame_h,
                         int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h, const uint16_t* pos,
                         int32_t n, uint64_t* scores, uint8_t* modes, int16_t* preds) {
  std::vector<int32_t> pred((size_t)w * h);
  for (int b = 0; b < n; b++) {
    const int px = pos[2 * b], py = pos[2 * b + 1];
    if (px + w > frame_w || py + h > frame_h) {
      for (int k = 0; k < 5; k++) {
        scores[(size_t)b * 5 + k] = UINT64_MAX;
        modes[(size_t)b * 5 + k] = 255;
      }
      continue;
    }
    const int vw = (vis_w > 0 ? vis_w : frame_w) - px, vh = (vis_h > 0 ? vis_h : frame_h) - py;
    std::vector<std::pair<uint64_t, int>> ranked;
    for (int m = 0; m < 5; m++) {
      or_filter_intra_predict(recon, stride, px, py, w, h, m, bd, pred.data());
      if (preds)
        for (int i = 0; i < w * h; i++) preds[((size_t)b * 5 + m) * w * h + i] = (int16_t)pred[i];
      uint64_t sad = 0, satd = 0;
      for (int ty = 0; ty < h; ty += 4)
        for (int tx = 0; tx < w; tx += 4) {
          int32_t rows[4][4];
          for (int r = 0; r < 4; r++) {
            int32_t d[4];
            for (int x = 0; x < 4; x++) {
              const bool vis = tx + x < vw && ty + r < vh;
              d[x] = vis ? (int32_t)src[(size_t)(py + ty + r) * stride + px + tx + x] - pred[(ty + r) * w + tx + x] : 0;
              sad += (uint64_t)(d[x] < 0 ? -d[x] : d[x]);
            }
            const int32_t e = d[0] + d[2], f = d[0] - d[2], g = d[1] + d[3], hh = d[1] - d[3];
            rows[r][0] = e + g;
            rows[r][1] = f + hh;
            rows[r][2] = f - hh;
            rows[r][3] = e - g;
          }
          for (int x = 0; x < 4; x++) {
            const int32_t a = rows[0][x], bb = rows[1][x], c = rows[2][x], dd = rows[3][x];
            const int32_t e = a + c, f = a - c, g = bb + dd, hh = bb - dd;
            auto ab = [](int32_t v) -> uint64_t { return (uint64_t)(v < 0 ? -v : v); };
            satd += ab(e + g) + ab(f + hh) + ab(f - hh) + ab(e - g);
          }
        }
      ranked.emplace_back(sad + (satd >> 2), m);
    }
    std::sort(ranked.begin(), ranked.end());
    for (int k = 0; k < 5; k++) {
      scores[(size_t)b * 5 + k] = ranked[k].first;
      modes[(size_t)b * 5 + k] = (uint8_t)ranked[k].second;
    }
  }
  return MT_OK;
}

}  // extern "C"
