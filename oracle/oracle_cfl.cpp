// Oracle (test-only checker of the CUDA path): chroma-from-luma alpha search
// of a batch of chroma blocks -- cfl_ac_sub / cfl_ac_444
// (src/intrapred.rs:1112-1172), cfl_pred_pixel (:1194-1199) and
// cfl_best_alpha_strided (:1211-1258) over the displayed part of each block.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "oracle.h"

namespace {

inline int32_t cfl_pred_pixel(int32_t dc, int32_t ac, int32_t alpha, int bd) {
  const int32_t diff = alpha * ac;
  const int32_t mag = ((diff < 0 ? -diff : diff) + 32) >> 6;
  const int32_t v = dc + (diff < 0 ? -mag : mag);
  const int32_t mx = (1 << bd) - 1;
  return v < 0 ? 0 : (v > mx ? mx : v);
}

inline int ilog2(int v) { return __builtin_ctz((unsigned)v); }

}  // namespace

extern "C" {

int or_cfl_alpha(const uint16_t* luma, int32_t luma_stride, const uint16_t* src_u, const uint16_t* src_v,
                 int32_t chroma_stride, int32_t sub_x, int32_t sub_y, int32_t cw, int32_t ch, int32_t vis_cw,
                 int32_t vis_ch, int32_t bd, const mt_cfl_block* blocks, int32_t n, int8_t* alpha, int32_t* ac_out) {
  std::vector<int32_t> ac((size_t)cw * ch);
  const int shift = 1 + (sub_y ? 0 : 1) + (sub_x ? 0 : 1);
  const int log2sz = ilog2(cw) + ilog2(ch);
  for (int b = 0; b < n; b++) {
    const int cx = blocks[b].cx, cy = blocks[b].cy;
    const uint16_t* l = luma + (size_t)(cy << sub_y) * luma_stride + (cx << sub_x);
    for (int y = 0; y < ch; y++)
      for (int x = 0; x < cw; x++) {
        const int ly = y << sub_y, lx = x << sub_x;
        int32_t s = l[(size_t)ly * luma_stride + lx];
        if (sub_x) s += l[(size_t)ly * luma_stride + lx + 1];
        if (sub_y) {
          s += l[(size_t)(ly + 1) * luma_stride + lx];
          if (sub_x) s += l[(size_t)(ly + 1) * luma_stride + lx + 1];
        }
        ac[y * cw + x] = s << shift;
      }
    int64_t sum = ((int64_t)1 << log2sz) >> 1;
    for (int32_t v : ac) sum += v;
    const int32_t mean = (int32_t)(sum >> log2sz);
    for (int32_t& v : ac) v -= mean;
    if (ac_out) memcpy(ac_out + (size_t)b * cw * ch, ac.data(), ac.size() * sizeof(int32_t));
    // vis 0: the whole block is displayed
    int vw = vis_cw > 0 ? vis_cw - cx : cw, vh = vis_ch > 0 ? vis_ch - cy : ch;
    vw = vw < 0 ? 0 : (vw > cw ? cw : vw);
    vh = vh < 0 ? 0 : (vh > ch ? ch : vh);
    for (int pl = 0; pl < 2; pl++) {
      const uint16_t* s = (pl ? src_v : src_u) + (size_t)cy * chroma_stride + cx;
      const int32_t dc = blocks[b].dc[pl];
      int64_t num = 0, den = 0;
      for (int y = 0; y < vh; y++)
        for (int x = 0; x < vw; x++) {
          const int64_t a = ac[y * cw + x];
          num += (int64_t)((int32_t)s[(size_t)y * chroma_stride + x] - dc) * a;
          den += a * a;
        }
      int best_a = 0;
      if (den != 0) {
        const int64_t sg = num > 0 ? 1 : (num < 0 ? -1 : 0);
        int64_t a0 = (64 * num + (den >> 1) * sg) / den;
        a0 = a0 < -16 ? -16 : (a0 > 16 ? 16 : a0);
        int64_t best_e = INT64_MAX;
        for (int cand = (int)a0 - 3; cand <= (int)a0 + 3; cand++) {
          if (cand < -16 || cand > 16) continue;
          int64_t e = 0;
          for (int y = 0; y < vh; y++)
            for (int x = 0; x < vw; x++) {
              const int64_t d =
                  (int32_t)s[(size_t)y * chroma_stride + x] - cfl_pred_pixel(dc, ac[y * cw + x], cand, bd);
              e += d * d;
            }
          if (e < best_e) {
            best_e = e;
            best_a = cand;
          }
        }
      }
      alpha[2 * b + pl] = (int8_t)best_a;
    }
  }
  return MT_OK;
}

}  // extern "C"
