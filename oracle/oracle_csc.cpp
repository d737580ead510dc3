// Oracle (test infrastructure only): the reference's RGB -> Y/Cb/Cr conversion
// and edge padding, restated as plain loops.
//   from_interleaved_rgb   src/encoder.rs:171-205 (plane0=G, plane1=B, plane2=R)
//   4:4:4 CSC              src/encoder.rs:370-410 (Q13, + half, >> 13, clamp)
//   4:2:0 CSC              src/encoder.rs:532-604 (unrounded Q13 chroma, 2x2 sum, + 2^14, >> 15)
//   pad_to_mult8_u16       src/dispatch.rs:113-131, dims :180-215
#include <stdint.h>
#include <string.h>

#include <vector>

#include "oracle.h"

namespace {
const int Q = 13, HALF = 1 << (Q - 1);
const int Y_R = 2449, Y_G = 4809, Y_B = 934;
const int CB_R = -1382, CB_G = -2714, CB_B = 4096;
const int CR_R = 4096, CR_G = -3430, CR_B = -666;
int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

// dispatch.rs:113-131: copy rows extending with the last sample, then repeat
// the last padded row.
void pad(const std::vector<uint16_t>& src, int w, int h, int pw, int ph, uint16_t* out) {
  std::vector<uint16_t> o;
  o.reserve((size_t)pw * ph);
  for (int y = 0; y < h; y++) {
    for (int x = 0; x < w; x++) o.push_back(src[(size_t)y * w + x]);
    uint16_t edge = o.back();
    for (int x = w; x < pw; x++) o.push_back(edge);
  }
  for (int y = h; y < ph; y++)
    for (int x = 0; x < pw; x++) o.push_back(o[(size_t)(h - 1) * pw + x]);
  memcpy(out, o.data(), o.size() * sizeof(uint16_t));
}
}  // namespace

extern "C" int or_csc_rgb8(const uint8_t* rgb, int32_t w, int32_t h, int32_t sub, uint16_t* yo, uint16_t* cbo,
                           uint16_t* cro) {
  if (w <= 0 || h <= 0 || (sub != 0 && sub != 2)) return MT_ERR_INVALID_INPUT;
  const size_t n = (size_t)w * h;
  std::vector<int32_t> R(n), G(n), B(n);
  for (size_t i = 0; i < n; i++) {  // from_interleaved_rgb: r,g,b per pixel
    R[i] = rgb[3 * i];
    G[i] = rgb[3 * i + 1];
    B[i] = rgb[3 * i + 2];
  }
  const int mx = 255, off_q = 128 << Q;
  std::vector<uint16_t> y(n);
  const int pw = (w + 7) & ~7, ph = (h + 7) & ~7;
  if (sub == 0) {
    std::vector<uint16_t> cb(n), cr(n);
    for (size_t i = 0; i < n; i++) {
      int r = R[i], g = G[i], b = B[i];
      y[i] = (uint16_t)clampi((Y_R * r + Y_G * g + Y_B * b + HALF) >> Q, 0, mx);
      cb[i] = (uint16_t)clampi((CB_R * r + CB_G * g + CB_B * b + off_q + HALF) >> Q, 0, mx);
      cr[i] = (uint16_t)clampi((CR_R * r + CR_G * g + CR_B * b + off_q + HALF) >> Q, 0, mx);
    }
    pad(y, w, h, pw, ph, yo);
    pad(cb, w, h, pw, ph, cbo);
    pad(cr, w, h, pw, ph, cro);
    return MT_OK;
  }
  std::vector<int32_t> fcb(n), fcr(n);
  for (size_t i = 0; i < n; i++) {
    int r = R[i], g = G[i], b = B[i];
    y[i] = (uint16_t)clampi((Y_R * r + Y_G * g + Y_B * b + HALF) >> Q, 0, mx);
    fcb[i] = CB_R * r + CB_G * g + CB_B * b + off_q;
    fcr[i] = CR_R * r + CR_G * g + CR_B * b + off_q;
  }
  const int cw = (w + 1) / 2, ch = (h + 1) / 2;
  const int half_avg = 1 << (Q + 1);
  std::vector<uint16_t> cb((size_t)cw * ch), cr((size_t)cw * ch);
  for (int row = 0; row < ch; row++)
    for (int c = 0; c < cw; c++) {
      int x0 = 2 * c, x1 = 2 * c + 1 < w - 1 ? 2 * c + 1 : w - 1;
      int y0 = 2 * row, y1 = 2 * row + 1 < h - 1 ? 2 * row + 1 : h - 1;
      auto avg = [&](const std::vector<int32_t>& f) {
        return f[(size_t)y0 * w + x0] + f[(size_t)y0 * w + x1] + f[(size_t)y1 * w + x0] + f[(size_t)y1 * w + x1];
      };
      cb[(size_t)row * cw + c] = (uint16_t)clampi((avg(fcb) + half_avg) >> (Q + 2), 0, mx);
      cr[(size_t)row * cw + c] = (uint16_t)clampi((avg(fcr) + half_avg) >> (Q + 2), 0, mx);
    }
  pad(y, w, h, pw, ph, yo);
  pad(cb, cw, ch, pw >> 1, ph >> 1, cbo);
  pad(cr, cw, ch, pw >> 1, ph >> 1, cro);
  return MT_OK;
}
