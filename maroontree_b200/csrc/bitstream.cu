// Headers and container of the still-image AV1 stream (host code): the
// bit writer and leb128 (src/bitwriter.rs:31-100), OBU framing, the reduced
// still-picture sequence header and the lossy frame header (src/obu.rs:46-771),
// the frame OBU assembly with its tile group (src/coder/frame_encode.rs:436-525),
// the spec-minimum tiling's increment bits (src/coder/tiling.rs:63-136) and
// the AVIF container (src/isobmff.rs:68-494 wrap_av1_image, src/avif.rs:676-740
// make_av1c / finalize_color).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/maroontree_b200.h"

namespace {

using Bytes = std::vector<uint8_t>;

struct BitWriter {
  Bytes bytes;
  uint8_t cur = 0;
  uint8_t nbits = 0;
  void f(uint32_t value, int n) {  // AV1 f(n), most significant bit first
    for (int i = n - 1; i >= 0; --i) {
      cur = (uint8_t)((cur << 1) | ((value >> i) & 1));
      if (++nbits == 8) {
        bytes.push_back(cur);
        cur = 0;
        nbits = 0;
      }
    }
  }
  void flag(bool b) { f(b ? 1 : 0, 1); }
  void byte_align() {
    if (nbits) {
      bytes.push_back((uint8_t)(cur << (8 - nbits)));
      cur = 0;
      nbits = 0;
    }
  }
  void trailing_bits() {
    f(1, 1);
    byte_align();
  }
  Bytes take() {
    byte_align();
    return std::move(bytes);
  }
};

void leb128(Bytes& out, uint64_t v) {
  do {
    uint8_t b = v & 0x7f;
    v >>= 7;
    if (v) b |= 0x80;
    out.push_back(b);
  } while (v);
}

enum ObuType { kSeqHeader = 1, kTemporalDelimiter = 2, kFrameHeader = 3, kTileGroup = 4, kFrame = 6 };

void wrap_obu(Bytes& out, int type, const uint8_t* payload, size_t n) {
  out.push_back((uint8_t)((type & 0xf) << 3 | 0x02));  // forbidden 0, type, extension 0, has_size 1, reserved 0
  leb128(out, n);
  out.insert(out.end(), payload, payload + n);
}

uint32_t bits_for(uint32_t v) {  // src/obu.rs:64-70
  uint32_t b = 1;
  while ((1u << b) <= (v > 0 ? v - 1 : 0)) ++b;
  return b;
}

Bytes sequence_header(const mt_sequence_header_params& p) {
  BitWriter w;
  w.f(p.profile, 3);  // seq_profile
  w.flag(true);       // still_picture
  w.flag(true);       // reduced_still_picture_header
  w.f(0, 5);          // seq_level_idx[0]
  const uint32_t wb = bits_for(p.width), hb = bits_for(p.height);
  w.f(wb - 1, 4);
  w.f(hb - 1, 4);
  w.f(p.width - 1, (int)wb);
  w.f(p.height - 1, (int)hb);
  w.flag(false);  // use_128x128_superblock
  w.flag(p.enable_filter_intra != 0);
  w.flag(p.enable_intra_edge_filter != 0);
  w.flag(false);  // enable_superres
  w.flag(true);   // enable_cdef
  w.flag(true);   // enable_restoration
  const bool high = p.bit_depth > 8;
  w.flag(high);
  if (p.profile == 2 && high) w.flag(p.bit_depth == 12);
  if (p.monochrome) {
    w.flag(true);   // mono_chrome
    w.flag(false);  // color_description_present_flag
    w.flag(p.full_range != 0);
  } else {
    if (p.profile != 1) w.flag(false);  // mono_chrome
    const bool identity = p.color_present && p.matrix == 0;
    if (p.color_present) {
      w.flag(true);
      w.f(p.primaries, 8);
      w.f(p.transfer, 8);
      w.f(p.matrix, 8);
    } else {
      w.flag(false);
    }
    if (!identity) {
      w.flag(p.color_present && p.full_range);
      if (p.profile == 2 && p.bit_depth == 12) {
        w.flag(p.ss_x == 1);
        if (p.ss_x == 1) w.flag(p.ss_y == 1);
      }
      if (p.ss_x == 1 && p.ss_y == 1) w.f(p.color_present ? p.chroma_sample_position : 0, 2);
    }
    w.flag(false);  // separate_uv_delta_q
  }
  w.flag(false);  // film_grain_params_present
  w.trailing_bits();
  Bytes payload = w.take(), out;
  wrap_obu(out, kSeqHeader, payload.data(), payload.size());
  return out;
}

uint32_t tile_log2(uint32_t blk, uint32_t target) {  // src/coder/tiling.rs:55-61
  uint32_t k = 0;
  while ((blk << k) < target) ++k;
  return k;
}

void increment_bits(uint32_t mn, uint32_t mx, uint32_t target, std::vector<bool>& v) {
  uint32_t cur = mn;
  while (cur < mx) {
    if (cur < target) {
      v.push_back(true);
      ++cur;
    } else {
      v.push_back(false);
      break;
    }
  }
}

Bytes frame_header(const mt_frame_header_params& p, bool trailing) {
  BitWriter w;
  w.flag(p.updating_cdf == 0);  // disable_cdf_update
  w.flag(true);                 // allow_screen_content_tools
  w.flag(true);                 // force_integer_mv
  w.flag(false);                // render_and_frame_size_different
  w.flag(p.allow_intrabc != 0);
  w.flag(true);  // uniform_tile_spacing_flag
  // increment_tile_{cols,rows}_log2 from the spec minimum to the plan
  const uint32_t sb_cols = (p.w8 + 63) / 64, sb_rows = (p.h8 + 63) / 64;
  const uint32_t min_c = tile_log2(64, sb_cols), max_c = tile_log2(1, sb_cols < 64 ? sb_cols : 64);
  const uint32_t max_r = tile_log2(1, sb_rows < 64 ? sb_rows : 64);
  const uint32_t min_t = min_c > tile_log2(2304, sb_rows * sb_cols) ? min_c : tile_log2(2304, sb_rows * sb_cols);
  std::vector<bool> ci, ri;
  increment_bits(min_c, max_c, p.tile_cols_log2, ci);
  increment_bits(min_t > p.tile_cols_log2 ? min_t - p.tile_cols_log2 : 0, max_r, p.tile_rows_log2, ri);
  for (bool b : ci) w.flag(b);
  for (bool b : ri) w.flag(b);
  if (p.tile_cols_log2 + p.tile_rows_log2 > 0) {
    w.f(0, (int)(p.tile_rows_log2 + p.tile_cols_log2));  // context_update_tile_id
    w.f(3, 2);                                           // tile_size_bytes_minus_1
  }
  w.f(p.base_q_idx, 8);
  w.flag(true);          // DeltaQYDc coded: luma_dc_delta -8 (src/quant.rs:350-352)
  w.f((uint32_t)(-8 & 0x7f), 7);
  if (!p.monochrome) {
    if (p.udc_delta != 0) {
      w.flag(true);
      w.f((uint32_t)(p.udc_delta & 0x7f), 7);
    } else {
      w.flag(false);
    }
    if (p.uac_delta != 0) {
      w.flag(true);
      w.f((uint32_t)(p.uac_delta & 0x7f), 7);
    } else {
      w.flag(false);
    }
  }
  const bool qm = p.qm_y < 15 || p.qm_u < 15 || p.qm_v < 15;
  w.flag(qm);
  if (qm) {
    w.f(p.qm_y, 4);
    w.f(p.qm_u, 4);
  }
  w.flag(false);  // segmentation_enabled
  if (p.aq) {
    w.flag(true);                  // delta_q_present
    w.f(p.delta_q_res_log2, 2);    // delta_q_res
    if (!p.allow_intrabc) w.flag(false);  // delta_lf_present
  } else {
    w.flag(false);
  }
  if (!p.allow_intrabc) {
    w.f((uint32_t)p.lf_y, 6);
    w.f((uint32_t)p.lf_y, 6);
    if (p.lf_y != 0 && !p.monochrome) {
      w.f((uint32_t)p.lf_u, 6);
      w.f((uint32_t)p.lf_v, 6);
    }
    w.f((uint32_t)p.lf_sharpness, 3);
    w.flag(false);  // loop_filter_delta_enabled
    // cdef_params (src/obu.rs:343-365): a no-op set when CDEF is off
    const int bits = p.cdef_bits < 0 ? 0 : p.cdef_bits;
    w.f(p.cdef_bits < 0 ? 0 : (uint32_t)(p.cdef_damping - 3), 2);
    w.f((uint32_t)bits, 2);
    auto sec = [](uint8_t s) { return s == 4 ? 3u : (uint32_t)s; };
    for (int i = 0; i < (1 << bits); ++i) {
      const uint8_t* st = p.cdef_bits < 0 ? nullptr : p.cdef_strengths[i];
      w.f(st ? st[0] : 0, 4);
      w.f(st ? sec(st[1]) : 0, 2);
      if (!p.monochrome) {
        w.f(st ? st[2] : 0, 4);
        w.f(st ? sec(st[3]) : 0, 2);
      }
    }
    // lr_params (src/obu.rs:373-394)
    w.f(p.lr_luma_wiener ? 2 : 0, 2);
    for (int k = 1; k < (p.monochrome ? 1 : 3); ++k) w.f(0, 2);
    if (p.lr_luma_wiener) w.f(0, 1);  // lr_unit_shift
  }
  w.flag(true);   // tx_mode_select
  w.flag(false);  // reduced_tx_set
  if (trailing) w.trailing_bits();
  return w.take();
}

int give(const Bytes& v, uint8_t** out, size_t* out_len) {
  uint8_t* p = (uint8_t*)malloc(v.size() ? v.size() : 1);
  if (!p) return MT_ERR_ALLOC;
  if (!v.empty()) memcpy(p, v.data(), v.size());
  *out = p;
  *out_len = v.size();
  return MT_OK;
}

// ---- ISOBMFF ------------------------------------------------------------

void w32(Bytes& b, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
}
void w16(Bytes& b, uint16_t v) {
  b.push_back((uint8_t)(v >> 8));
  b.push_back((uint8_t)v);
}
void cc(Bytes& b, const char* s) { b.insert(b.end(), s, s + 4); }
size_t box(Bytes& b, const char* c) {
  const size_t s = b.size();
  w32(b, 0);
  cc(b, c);
  return s;
}
size_t fullbox(Bytes& b, const char* c, uint8_t ver, uint32_t flags) {
  const size_t s = box(b, c);
  b.push_back(ver);
  b.push_back((uint8_t)(flags >> 16));
  b.push_back((uint8_t)(flags >> 8));
  b.push_back((uint8_t)flags);
  return s;
}
void patch(Bytes& b, size_t s) {
  const uint32_t n = (uint32_t)(b.size() - s);
  b[s] = (uint8_t)(n >> 24);
  b[s + 1] = (uint8_t)(n >> 16);
  b[s + 2] = (uint8_t)(n >> 8);
  b[s + 3] = (uint8_t)n;
}
void put32_at(Bytes& b, size_t at, uint32_t v) {
  for (int k = 0; k < 4; ++k) b[at + k] = (uint8_t)(v >> (24 - 8 * k));
}

}  // namespace

extern "C" {

int mt_leb128(uint64_t value, uint8_t* out, size_t cap, size_t* len) {
  Bytes b;
  leb128(b, value);
  if (len) *len = b.size();
  if (!out || cap < b.size()) return out ? MT_ERR_TOO_LARGE : MT_OK;
  memcpy(out, b.data(), b.size());
  return MT_OK;
}

int mt_wrap_obu(int32_t obu_type, const uint8_t* payload, size_t n, uint8_t** out, size_t* out_len) {
  if (obu_type < 1 || obu_type > 15 || (n && !payload) || !out || !out_len) return MT_ERR_INVALID_INPUT;
  Bytes b;
  wrap_obu(b, obu_type, payload, n);
  return give(b, out, out_len);
}

int mt_tiling_increments(int32_t w8, int32_t h8, int32_t tile_cols_log2, int32_t tile_rows_log2, uint8_t* cols_incr,
                         int32_t* ncols, uint8_t* rows_incr, int32_t* nrows) {
  if (w8 <= 0 || h8 <= 0 || tile_cols_log2 < 0 || tile_rows_log2 < 0) return MT_ERR_INVALID_INPUT;
  const uint32_t sb_cols = (uint32_t)(w8 + 63) / 64, sb_rows = (uint32_t)(h8 + 63) / 64;
  const uint32_t min_c = tile_log2(64, sb_cols), max_c = tile_log2(1, sb_cols < 64 ? sb_cols : 64);
  const uint32_t max_r = tile_log2(1, sb_rows < 64 ? sb_rows : 64);
  const uint32_t area = tile_log2(2304, sb_rows * sb_cols);
  const uint32_t min_t = min_c > area ? min_c : area;
  std::vector<bool> ci, ri;
  increment_bits(min_c, max_c, (uint32_t)tile_cols_log2, ci);
  increment_bits(min_t > (uint32_t)tile_cols_log2 ? min_t - tile_cols_log2 : 0, max_r, (uint32_t)tile_rows_log2, ri);
  if (ncols) *ncols = (int32_t)ci.size();
  if (nrows) *nrows = (int32_t)ri.size();
  for (size_t k = 0; cols_incr && k < ci.size() && k < 8; ++k) cols_incr[k] = ci[k];
  for (size_t k = 0; rows_incr && k < ri.size() && k < 8; ++k) rows_incr[k] = ri[k];
  return MT_OK;
}

int mt_sequence_header(const mt_sequence_header_params* p, uint8_t** out, size_t* out_len) {
  if (!p || !out || !out_len || p->width < 1 || p->height < 1 || p->width > 65536 || p->height > 65536)
    return MT_ERR_INVALID_INPUT;
  if (p->profile > 2 || (p->bit_depth != 8 && p->bit_depth != 10 && p->bit_depth != 12)) return MT_ERR_INVALID_INPUT;
  return give(sequence_header(*p), out, out_len);
}

int mt_frame_header(const mt_frame_header_params* p, int32_t trailing, uint8_t** out, size_t* out_len) {
  if (!p || !out || !out_len || p->base_q_idx == 0 || p->w8 <= 0 || p->h8 <= 0) return MT_ERR_INVALID_INPUT;
  if (p->cdef_bits > 3 || p->qm_y > 15 || p->qm_u > 15 || p->qm_v > 15 || p->delta_q_res_log2 > 3)
    return MT_ERR_INVALID_INPUT;
  return give(frame_header(*p, trailing != 0), out, out_len);
}

int mt_assemble_frame_obus(const mt_frame_header_params* p, const uint8_t* const* tiles, const size_t* tile_lens,
                           int32_t ntiles, uint8_t** out, size_t* out_len) {
  if (!p || !out || !out_len || ntiles < 1 || !tiles || !tile_lens) return MT_ERR_INVALID_INPUT;
  if (p->base_q_idx == 0) return MT_ERR_INVALID_INPUT;
  // tile group (src/coder/frame_encode.rs:444-459)
  Bytes tg;
  if (ntiles == 1) {
    tg.assign(tiles[0], tiles[0] + tile_lens[0]);
  } else {
    tg.push_back(0);  // tile_start_and_end_present_flag 0 + byte_alignment
    for (int32_t i = 0; i < ntiles; ++i) {
      if (tile_lens[i] == 0) return MT_ERR_INVALID_INPUT;
      if (i != ntiles - 1) {
        const uint32_t m = (uint32_t)(tile_lens[i] - 1);
        for (int k = 0; k < 4; ++k) tg.push_back((uint8_t)(m >> (8 * k)));
      }
      tg.insert(tg.end(), tiles[i], tiles[i] + tile_lens[i]);
    }
  }
  Bytes o;
  if (p->tile_cols_log2 + p->tile_rows_log2 > 0) {
    Bytes fh = frame_header(*p, true);
    wrap_obu(o, kFrameHeader, fh.data(), fh.size());
    wrap_obu(o, kTileGroup, tg.data(), tg.size());
  } else {
    Bytes fh = frame_header(*p, false);
    fh.insert(fh.end(), tg.begin(), tg.end());
    wrap_obu(o, kFrame, fh.data(), fh.size());
  }
  return give(o, out, out_len);
}

int mt_av1_stream(const mt_sequence_header_params* sp, const mt_frame_header_params* fp, const uint8_t* const* tiles,
                  const size_t* tile_lens, int32_t ntiles, uint8_t** out, size_t* out_len) {
  if (!sp || !fp || !out || !out_len) return MT_ERR_INVALID_INPUT;
  uint8_t* seq = nullptr;
  size_t nseq = 0;
  uint8_t* fr = nullptr;
  size_t nfr = 0;
  int rc = mt_sequence_header(sp, &seq, &nseq);
  if (rc != MT_OK) return rc;
  rc = mt_assemble_frame_obus(fp, tiles, tile_lens, ntiles, &fr, &nfr);
  if (rc != MT_OK) {
    free(seq);
    return rc;
  }
  Bytes b;
  wrap_obu(b, kTemporalDelimiter, nullptr, 0);  // temporal_delimiter (src/obu.rs:60-62)
  b.insert(b.end(), seq, seq + nseq);
  b.insert(b.end(), fr, fr + nfr);
  free(seq);
  free(fr);
  return give(b, out, out_len);
}

uint8_t mt_av1_level_for(uint32_t width, uint32_t height) {  // src/isobmff.rs:162-176 level_for
  const uint64_t px = (uint64_t)width * height;
  if (px <= 147456) return 0;
  if (px <= 278784) return 1;
  if (px <= 737280) return 4;
  if (px <= 2228224) return 8;
  if (px <= 8912896) return 12;
  if (px <= 35651584) return 16;
  return 19;
}

int mt_wrap_av1_image(const uint8_t* obu, size_t obu_len, const mt_avif_item_params* p, uint8_t** out,
                      size_t* out_len) {
  if (!obu || !p || !out || !out_len || p->width == 0 || p->height == 0) return MT_ERR_INVALID_INPUT;
  if (p->channels != 1 && p->channels != 3) return MT_ERR_INVALID_INPUT;
  if ((p->icc_len && !p->icc) || (p->exif_len && !p->exif) || p->irot_steps > 3) return MT_ERR_INVALID_INPUT;
  if (obu_len > 0xffffffffu) return MT_ERR_TOO_LARGE;
  const bool has_exif = p->exif != nullptr;
  Bytes f;
  size_t s = box(f, "ftyp");
  cc(f, "avif");
  w32(f, 0);
  cc(f, "avif");
  cc(f, "mif1");
  cc(f, "miaf");
  patch(f, s);
  const size_t meta = fullbox(f, "meta", 0, 0);
  s = fullbox(f, "hdlr", 0, 0);
  w32(f, 0);
  cc(f, "pict");
  w32(f, 0);
  w32(f, 0);
  w32(f, 0);
  f.push_back(0);
  patch(f, s);
  s = fullbox(f, "pitm", 0, 0);
  w16(f, 1);
  patch(f, s);
  s = fullbox(f, "iloc", 0, 0);
  f.push_back(0x44);  // offset_size 4, length_size 4
  f.push_back(0x00);
  w16(f, has_exif ? 2 : 1);
  w16(f, 1);
  w16(f, 0);
  w16(f, 1);
  const size_t av1_off_at = f.size();
  w32(f, 0);
  w32(f, (uint32_t)obu_len);
  size_t exif_off_at = 0;
  if (has_exif) {
    w16(f, 2);
    w16(f, 0);
    w16(f, 1);
    exif_off_at = f.size();
    w32(f, 0);
    w32(f, (uint32_t)(p->exif_len + 4));
  }
  patch(f, s);
  s = fullbox(f, "iinf", 0, 0);
  w16(f, has_exif ? 2 : 1);
  size_t si = fullbox(f, "infe", 2, 0);
  w16(f, 1);
  w16(f, 0);
  cc(f, "av01");
  f.push_back(0);
  patch(f, si);
  if (has_exif) {
    si = fullbox(f, "infe", 2, 0);
    w16(f, 2);
    w16(f, 0);
    cc(f, "Exif");
    f.push_back(0);
    patch(f, si);
  }
  patch(f, s);
  if (has_exif) {
    s = fullbox(f, "iref", 0, 0);
    si = box(f, "cdsc");
    w16(f, 2);
    w16(f, 1);
    w16(f, 1);
    patch(f, si);
    patch(f, s);
  }
  // iprp / ipco: 1 ispe, 2 pixi, 3 av1C (essential), then colr boxes, irot, imir, clli
  s = box(f, "iprp");
  si = box(f, "ipco");
  size_t sh = fullbox(f, "ispe", 0, 0);
  w32(f, p->width);
  w32(f, p->height);
  patch(f, sh);
  sh = fullbox(f, "pixi", 0, 0);
  f.push_back(p->channels);
  for (int k = 0; k < p->channels; ++k) f.push_back(p->bit_depth);
  patch(f, sh);
  sh = box(f, "av1C");
  f.push_back(0x81);
  f.push_back((uint8_t)(((p->seq_profile & 7) << 5) | (p->seq_level_idx & 0x1f)));
  f.push_back((uint8_t)((p->bit_depth > 8 ? 0x40 : 0) | (p->bit_depth == 12 ? 0x20 : 0) |
                        (p->monochrome ? 0x10 : 0) | (p->chroma_sub_x ? 0x08 : 0) | (p->chroma_sub_y ? 0x04 : 0)));
  f.push_back(0);
  patch(f, sh);
  uint8_t next = 4;
  std::vector<uint8_t> assoc = {1, 2, 0x80 | 3};
  if (p->color_present) {
    sh = box(f, "colr");
    cc(f, "nclx");
    w16(f, p->primaries);
    w16(f, p->transfer);
    w16(f, p->matrix);
    f.push_back(p->full_range ? 0x80 : 0x00);
    patch(f, sh);
    assoc.push_back(next++);
  }
  if (p->icc) {
    sh = box(f, "colr");
    cc(f, "prof");
    f.insert(f.end(), p->icc, p->icc + p->icc_len);
    patch(f, sh);
    assoc.push_back(next++);
  }
  if (p->irot_steps) {
    sh = box(f, "irot");
    f.push_back(p->irot_steps & 3);
    patch(f, sh);
    assoc.push_back(0x80 | next++);
  }
  if (p->imir_axis >= 0) {
    sh = box(f, "imir");
    f.push_back(p->imir_axis ? 1 : 0);
    patch(f, sh);
    assoc.push_back(0x80 | next++);
  }
  if (p->clli_present) {
    sh = box(f, "clli");
    w16(f, p->max_content_light_level);
    w16(f, p->max_pic_average_light_level);
    patch(f, sh);
    assoc.push_back(next++);
  }
  patch(f, si);
  si = fullbox(f, "ipma", 0, 0);
  w32(f, 1);
  w16(f, 1);
  f.push_back((uint8_t)assoc.size());
  f.insert(f.end(), assoc.begin(), assoc.end());
  patch(f, si);
  patch(f, s);
  patch(f, meta);
  s = box(f, "mdat");
  const uint32_t av1_off = (uint32_t)f.size();
  f.insert(f.end(), obu, obu + obu_len);
  const uint32_t exif_off = (uint32_t)f.size();
  if (has_exif) {
    w32(f, 0);  // exif_tiff_header_offset
    f.insert(f.end(), p->exif, p->exif + p->exif_len);
  }
  patch(f, s);
  put32_at(f, av1_off_at, av1_off);
  if (has_exif) put32_at(f, exif_off_at, exif_off);
  return give(f, out, out_len);
}

}  // extern "C"
