// Oracle encode (test infrastructure only): the library's whole-frame encoder
// (mt_encode_rgb8's decision rule) restated on the CPU, so that its AVIF bytes
// can be checked and its speed measured without the product library.
//
//   or_encode_decide  every superblock as a full split to 8x8 blocks; each 8x8
//                     luma block takes the lowest RD cost (strict <, first in
//                     (mode, type) order) of the 13 intra modes at angle
//                     delta 0 times the seven 8x8 intra transform types, each
//                     priced by the oracle's candidate chain
//                     (partition_search.rs:467-530); chroma is UV_DC_PRED
//                     with DCT_DCT (8x8 in 4:4:4, 4x4 in 4:2:0).  Superblocks
//                     run on host threads in the reference's wavefront
//                     (src/coder/wavefront.rs:77-300: a superblock after its
//                     left, top-left, top and top-right neighbours).
//   or_encode_pack    the block syntax in coding order (partition with the
//                     gathered edge bools, skip, kf_y mode, angle delta, uv
//                     mode, palette and filter-intra flags, tx depth:
//                     src/coder/superblock.rs:711-990,
//                     src/coder/block8.rs:2620-2700,
//                     src/coder/lossy_state.rs:1408-1415, :4021-4051), the
//                     coefficient tokens of the oracle's coders with their
//                     txb_skip / dc_sign contexts (src/coeffs.rs:2917-2920),
//                     and each tile's range coding (src/odec.rs:35-615
//                     OdEcEncoder, src/coder/wavefront.rs:617-657
//                     pack_wavefront_tile) with each superblock's cdef_idx
//                     literal at its read_cdef() point
//                     (src/coder/tile_encode.rs:404-466).
// Both work in the uniform tiling the caller gives (the spec minimum,
// src/coder/frame_encode.rs:75-103): each tile is coded as a frame of its own,
// with its own contexts and range coder.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

const uint8_t kTypes[7] = {MT_TX_IDTX,      MT_TX_DCT_DCT,   MT_TX_V_DCT,   MT_TX_H_DCT,
                           MT_TX_ADST_ADST, MT_TX_ADST_DCT, MT_TX_DCT_ADST};

// Position of the k-th 8x8 block of a 64x64 superblock in z-order and its
// intra-edge availability flags down the split tree
// (src/coder/superblock.rs:958-987): the root passes (top-right 1,
// bottom-left 0); the children get TL (1, 1), TR (parent's, 0), BL (1,
// parent's), BR (0, 0).
void zorder8(int k, int* bx, int* by, bool* tr, bool* bl) {
  int x = 0, y = 0;
  bool t = true, l = false;
  for (int lvl = 2; lvl >= 0; --lvl) {
    const int q = (k >> (2 * lvl)) & 3, h = 1 << lvl;
    if (q == 0) {
      t = true;
      l = true;
    } else if (q == 1) {
      x += h;
      l = false;
    } else if (q == 2) {
      y += h;
      t = true;
    } else {
      x += h;
      y += h;
      t = false;
      l = false;
    }
  }
  *bx = x;
  *by = y;
  *tr = t;
  *bl = l;
}

bool smooth(int m) { return m == MT_SMOOTH_PRED || m == MT_SMOOTH_V_PRED || m == MT_SMOOTH_H_PRED; }

struct Frame {
  int pw, ph, pcw, pch, sub, nbx, nby;
  int tw8, th8;  // the uniform tile size in 8x8 blocks
  const mt_chain_params* py;
  const mt_chain_params* pc;
  const mt_quant* qy;
  const mt_quant* qc;
  const uint8_t* qmy;
  const uint8_t* qmc;
  const mt_coef_cdfs* cdy;
  const mt_coef_cdfs* cdc;
  const uint16_t* src[3];
  uint16_t* rec[3];
  uint8_t* mode;
  uint8_t* tx;
  int32_t* lv[3];
};

// One 8x8 block: the luma decision and the chroma blocks.  The block's tile
// is coded as a frame of its own, as the reference codes a cropped tile
// (src/coder/frame_encode.rs:82-103, src/coder/tiling.rs crop_plane): tile
// coordinates, the tile's size as the frame size, the planes from the tile's
// origin.
void code_block(const Frame& f, int x8, int y8, bool thr, bool lhb) {
  const int b = y8 * f.nbx + x8;
  const int tx0 = x8 - x8 % f.tw8, ty0 = y8 - y8 % f.th8;
  const int tw = (std::min(tx0 + f.tw8, f.nbx) - tx0) * 8, th = (std::min(ty0 + f.th8, f.nby) - ty0) * 8;
  const int px = (x8 - tx0) * 8, py = (y8 - ty0) * 8;
  mt_chain_params ply = *f.py;
  ply.frame_w = tw;
  ply.frame_h = th;
  const size_t oy = (size_t)ty0 * 8 * f.pw + (size_t)tx0 * 8;
  const bool have_tr = thr && py > 0 && px + 8 < tw;
  const bool have_bl = lhb && px > 0 && py + 8 < th;
  const bool ft = (py > 0 && smooth(f.mode[b - f.nbx])) || (px > 0 && smooth(f.mode[b - 1]));
  mt_candidate cands[91];
  memset(cands, 0, sizeof(cands));
  for (int t = 0; t < 91; ++t) {
    cands[t].px = (uint16_t)px;
    cands[t].py = (uint16_t)py;
    cands[t].mode = (uint8_t)(t / 7);
    cands[t].tx_type = kTypes[t % 7];
    cands[t].flags = (uint8_t)((have_tr ? 1 : 0) | (have_bl ? 2 : 0) | (ft ? 4 : 0));
  }
  mt_candidate_result res[91];
  std::vector<int32_t> lv(91 * 64), rc(91 * 64);
  or_candidate_chain(f.src[0] + oy, f.rec[0] + oy, &ply, f.qy, f.qmy, f.cdy, cands, 91, res, lv.data(), rc.data(), 1);
  int best = 0;
  for (int t = 1; t < 91; ++t)
    if (res[t].cost < res[best].cost) best = t;
  for (int y = 0; y < 8; ++y)
    for (int x = 0; x < 8; ++x) f.rec[0][oy + (size_t)(py + y) * f.pw + px + x] = (uint16_t)rc[best * 64 + y * 8 + x];
  memcpy(f.lv[0] + (size_t)b * 64, &lv[best * 64], 64 * sizeof(int32_t));
  f.mode[b] = (uint8_t)(best / 7);
  f.tx[b] = kTypes[best % 7];
  // chroma: UV_DC_PRED, DCT_DCT
  const int n = f.sub ? 4 : 8, sh = f.sub ? 1 : 0;
  mt_chain_params plc = *f.pc;
  plc.frame_w = tw >> sh;
  plc.frame_h = th >> sh;
  const size_t oc = (size_t)(ty0 * 8 >> sh) * f.pcw + (size_t)(tx0 * 8 >> sh);
  for (int p = 1; p < 3; ++p) {
    mt_candidate c;
    memset(&c, 0, sizeof(c));
    c.px = (uint16_t)(px >> sh);
    c.py = (uint16_t)(py >> sh);
    c.mode = MT_DC_PRED;
    c.tx_type = MT_TX_DCT_DCT;
    c.flags = (uint8_t)(f.sub ? 0 : ((have_tr ? 1 : 0) | (have_bl ? 2 : 0)));
    mt_candidate_result r;
    int32_t l[64], o[64];
    or_candidate_chain(f.src[p] + oc, f.rec[p] + oc, &plc, f.qc, f.qmc, f.cdc, &c, 1, &r, l, o, 1);
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) f.rec[p][oc + (size_t)(c.py + y) * f.pcw + c.px + x] = (uint16_t)o[y * n + x];
    memcpy(f.lv[p] + (size_t)b * n * n, l, (size_t)n * n * sizeof(int32_t));
  }
}

void code_sb(const Frame& f, int sr, int sc) {
  for (int k = 0; k < 64; ++k) {
    int bx, by;
    bool tr, bl;
    zorder8(k, &bx, &by, &tr, &bl);
    const int x8 = sc * 8 + bx, y8 = sr * 8 + by;
    if (x8 < f.nbx && y8 < f.nby) code_block(f, x8, y8, tr, bl);
  }
}

// ---- tile range coder (src/odec.rs:35-615) ---------------------------------

struct RangeCoder {
  uint32_t low = 0;
  uint32_t rng = 0x8000;
  int cnt = -9;
  std::vector<uint16_t> pre;  // bytes before carry propagation, one per output byte

  void store(uint32_t fl, uint32_t fh, uint32_t nms) {  // od_ec_encode_q15
    const uint32_t r = rng;
    uint32_t u = fl >= 32768 ? r : (((r >> 8) * (fl >> 6)) >> 1) + 4 * nms;
    const uint32_t v = (((r >> 8) * (fh >> 6)) >> 1) + 4 * (nms - 1);
    uint32_t l = low + (r - u);
    const uint32_t nr = (u - v) & 0xffff;
    int d = 0;
    while (d < 16 && !((nr << d) & 0x8000)) ++d;  // 15 - ilog(nr) + 1 renormalisation shift
    int c = cnt, s = c + d;
    if (s >= 0) {
      c += 16;
      uint32_t m = (1u << c) - 1;
      if (s >= 8) {
        pre.push_back((uint16_t)(l >> c));
        l &= m;
        c -= 8;
        m >>= 8;
      }
      pre.push_back((uint16_t)(l >> c));
      s = c + d - 24;
      l &= m;
    }
    low = l << d;
    rng = (nr << d) & 0xffff;
    cnt = s;
  }
  void boolean(bool v, uint32_t f) { v ? store(f, 0, 1) : store(32768, f, 2); }
  void literal(uint32_t v, int bits) {
    for (int i = bits - 1; i >= 0; --i) boolean(((v >> i) & 1) != 0, 16384);
  }
  static void update(uint16_t* cdf, int n, int s) {  // update_cdf (src/odec.rs:47-60)
    const uint32_t count = cdf[n - 1];
    const uint32_t rate = 3 + (uint32_t)((n >> 1) < 2 ? (n >> 1) : 2) + (count >> 4);
    cdf[n - 1] = (uint16_t)(count + 1 - (count >> 5));
    for (int i = 0; i < n - 1; ++i)
      cdf[i] = (uint16_t)(i < s ? cdf[i] + ((32768u - cdf[i]) >> rate) : cdf[i] - (cdf[i] >> rate));
  }
  void symbol(int s, uint16_t* cdf, int n, bool adapt) {
    store(s > 0 ? cdf[s - 1] : 32768u, cdf[s], (uint32_t)(n - s));
    if (adapt) update(cdf, n, s);
  }
  std::vector<uint8_t> done() {  // od_ec_enc_done
    int c = cnt, s = c + 10;
    const uint32_t m = 0x3fff;
    uint32_t e = ((low + m) & ~m) | (m + 1);
    if (s > 0) {
      uint32_t n = (1u << (c + 16)) - 1;
      do {
        pre.push_back((uint16_t)(e >> (c + 16)));
        e &= n;
        s -= 8;
        c -= 8;
        n >>= 8;
      } while (s > 0);
    }
    std::vector<uint8_t> out(pre.size());
    uint32_t carry = 0;
    for (size_t i = pre.size(); i-- > 0;) {
      carry += pre[i];
      out[i] = (uint8_t)carry;
      carry >>= 8;
    }
    return out;
  }
};

const int kModeCtx[13] = {0, 1, 2, 3, 4, 4, 4, 4, 3, 0, 1, 2, 0};  // src/intrapred.rs:1088

struct SyntaxSlots {  // first CDF slot of each symbol group (Cdfs::semantic_slots order)
  int32_t skip, part_bl8, part_split, kf_y, uv_mode, angle_delta, filter_intra, palette_y_mode, palette_uv_mode,
      txsz;
};

struct Syntax {
  const Frame& f;
  const SyntaxSlots& L;
  const or_emit_slots& E;
  std::vector<uint8_t> a_part, l_part, a_skip, l_skip, a_mode, l_mode;
  std::vector<int8_t> a_tx, l_tx;
  std::vector<uint8_t> a_coef[3], l_coef[3];
  std::vector<uint32_t>* out = nullptr;
  int cdef_point = -1;

  Syntax(const Frame& fr, const SyntaxSlots& l, const or_emit_slots& e)
      : f(fr), L(l), E(e), a_part(fr.nbx, 0), l_part(fr.nby, 0), a_skip(fr.nbx * 2, 0), l_skip(fr.nby * 2, 0),
        a_mode(fr.nbx * 2, 0), l_mode(fr.nby * 2, 0), a_tx(fr.nbx * 2, -1), l_tx(fr.nby * 2, -1) {
    for (int p = 0; p < 3; ++p) {
      a_coef[p].assign(fr.nbx * 2, 0x40);
      l_coef[p].assign(fr.nby * 2, 0x40);
    }
  }
  void sym(int32_t slot, uint32_t s) { out->push_back(((uint32_t)slot << 8) | s); }
  // clear_above_context for a tile's 8x8 columns [x0, x1) and
  // clear_left_context for a superblock row's 8x8 rows [y0, y1) (decode_tile)
  void clear_above(int x0, int x1) {
    for (int x = x0; x < x1; ++x) a_part[x] = 0;
    for (int x = 2 * x0; x < 2 * x1; ++x) {
      a_skip[x] = a_mode[x] = 0;
      a_tx[x] = -1;
    }
    for (int p = 0; p < 3; ++p)
      for (int x = (p && f.sub ? 1 : 2) * x0; x < (p && f.sub ? 1 : 2) * x1; ++x) a_coef[p][x] = 0x40;
  }
  void clear_left(int y0, int y1) {
    for (int y = y0; y < y1; ++y) l_part[y] = 0;
    for (int y = 2 * y0; y < 2 * y1; ++y) {
      l_skip[y] = l_mode[y] = 0;
      l_tx[y] = -1;
    }
    for (int p = 0; p < 3; ++p)
      for (int y = (p && f.sub ? 1 : 2) * y0; y < (p && f.sub ? 1 : 2) * y1; ++y) l_coef[p][y] = 0x40;
  }
  int part_ctx(int bl, int x8, int y8) const {
    return ((a_part[x8] >> (4 - bl)) & 1) + (((l_part[y8] >> (4 - bl)) & 1) << 1);
  }

  void leaf(int x8, int y8) {
    const int b = y8 * f.nbx + x8, bx4 = x8 * 2, by4 = y8 * 2;
    const int m = f.mode[b], t = f.tx[b];
    sym(L.skip + a_skip[bx4] + l_skip[by4], 0);  // skip = 0
    if (cdef_point < 0) cdef_point = (int)out->size();
    a_skip[bx4] = a_skip[bx4 + 1] = l_skip[by4] = l_skip[by4 + 1] = 0;
    sym(L.kf_y + kModeCtx[a_mode[bx4]] * 5 + kModeCtx[l_mode[by4]], (uint32_t)m);
    if (m >= MT_V_PRED && m <= MT_D67_PRED) sym(L.angle_delta + m - MT_V_PRED, 3);  // angle delta 0
    sym(L.uv_mode + 13 + m, MT_DC_PRED);  // the CfL-allowed row at 8x8
    if (m == MT_DC_PRED) sym(L.palette_y_mode, 0);
    sym(L.palette_uv_mode, 0);
    if (m == MT_DC_PRED) sym(L.filter_intra + 3, 0);  // BLOCK_8X8
    sym(L.txsz + (l_tx[by4] >= 1) + (a_tx[bx4] >= 1), 0);
    a_tx[bx4] = a_tx[bx4 + 1] = l_tx[by4] = l_tx[by4 + 1] = 1;
    for (int p = 0; p < 3; ++p) {
      const bool full = p == 0 || f.sub == 0;
      const int u = full ? 2 : 1, n = full ? 8 : 4;
      const int cx = full ? bx4 : bx4 / 2, cy = full ? by4 : by4 / 2;
      int s = -2 * u, anz = 0, lnz = 0;
      for (int k = 0; k < u; ++k) {
        s += (a_coef[p][cx + k] >> 6) + (l_coef[p][cy + k] >> 6);
        anz |= a_coef[p][cx + k] != 0x40;
        lnz |= l_coef[p][cy + k] != 0x40;
      }
      mt_coef_block cb;
      memset(&cb, 0, sizeof(cb));
      cb.cf_offset = 0;
      cb.log2n = (uint8_t)(full ? 3 : 2);
      cb.plane = p ? 1 : 0;
      cb.skip_ctx = (uint8_t)(p == 0 ? 0 : 7 + anz + lnz);
      cb.dcs_ctx = (uint8_t)((s != 0) + (s > 0));
      cb.y_mode = (uint8_t)m;
      cb.txtp = (uint8_t)(p == 0 ? t : MT_TX_DCT_DCT);
      cb.code_txtp = p == 0;
      cb.tx_class = (uint8_t)(p == 0 && t == MT_TX_V_DCT ? 1 : (p == 0 && t == MT_TX_H_DCT ? 2 : 0));
      uint32_t toks[1024], off[2];
      uint8_t rctx = 0;
      or_emit_coeffs(f.lv[p] + (size_t)b * n * n, &cb, 1, &E, toks, 1024, off, &rctx);
      out->insert(out->end(), toks, toks + off[1]);
      for (int k = 0; k < u; ++k) a_coef[p][cx + k] = l_coef[p][cy + k] = rctx;
    }
    a_mode[bx4] = a_mode[bx4 + 1] = l_mode[by4] = l_mode[by4 + 1] = (uint8_t)m;
  }

  // code_split always taking SPLIT down to 8x8 PARTITION_NONE leaves
  // (src/coder/superblock.rs:950-990); at the frame edge the split is a
  // gathered bool of the partition CDF (src/coeffs.rs:2917-2935), or implied.
  void node(int bl, int x8, int y8, int sz8) {
    if (sz8 == 1) {
      sym(L.part_bl8 + part_ctx(4, x8, y8), 0);
      leaf(x8, y8);
      a_part[x8] = l_part[y8] = 0x1E;
      return;
    }
    const int hh = sz8 / 2;
    const bool has_cols = (x8 + hh) * 8 < f.pw, has_rows = (y8 + hh) * 8 < f.ph;
    const int32_t slot = L.part_split + (bl - 1) * 4 + part_ctx(bl, x8, y8);
    if (has_cols && has_rows)
      sym(slot, 3);
    else if (has_cols)
      out->push_back((2u << 30) | ((uint32_t)slot << 2) | 2u | 1u);  // split_or_horz: gathered from above
    else if (has_rows)
      out->push_back((2u << 30) | ((uint32_t)slot << 2) | 2u);  // split_or_vert: gathered from the left
    const int cx[4] = {x8, x8 + hh, x8, x8 + hh}, cy[4] = {y8, y8, y8 + hh, y8 + hh};
    for (int c = 0; c < 4; ++c)
      if (cx[c] * 8 < f.pw && cy[c] * 8 < f.ph) node(bl + 1, cx[c], cy[c], hh);
  }
};

// gather_split_prob_icdf (src/coeffs.rs:2927-2935)
uint32_t gather(const uint16_t* c, bool top) {
  int32_t v = top ? ((int32_t)c[1] - c[4]) + c[5] + ((int32_t)c[8] - c[7])
                  : ((int32_t)c[0] - c[1]) + ((int32_t)c[2] - c[6]) + ((int32_t)c[7] - c[8]);
  return (uint32_t)(v < 1 ? 1 : (v > 32767 ? 32767 : v));
}

}  // namespace

extern "C" {

// The decisions, reconstruction and levels of a frame (planes padded to x8:
// luma pw x ph, chroma pcw x pch; levels: 64 per block for luma and 64 / 16
// per block for chroma) in uniform tiles of tile_sb_w x tile_sb_h
// superblocks.  threads <= 1 codes the superblocks serially.
int or_encode_decide(int32_t pw, int32_t ph, int32_t sub, int32_t tile_sb_w, int32_t tile_sb_h,
                     const mt_chain_params* py, const mt_chain_params* pc, const mt_quant* qy, const mt_quant* qc,
                     const uint8_t* qmy, const uint8_t* qmc, const mt_coef_cdfs* cdy, const mt_coef_cdfs* cdc,
                     const uint16_t* src_y, const uint16_t* src_u, const uint16_t* src_v, uint16_t* rec_y,
                     uint16_t* rec_u, uint16_t* rec_v, uint8_t* mode, uint8_t* tx, int32_t* lv_y, int32_t* lv_u,
                     int32_t* lv_v, int32_t threads) {
  if (pw <= 0 || ph <= 0 || (pw & 7) || (ph & 7) || (sub != 0 && sub != 2) || tile_sb_w <= 0 || tile_sb_h <= 0)
    return MT_ERR_INVALID_INPUT;
  Frame f;
  f.tw8 = tile_sb_w * 8;
  f.th8 = tile_sb_h * 8;
  f.pw = pw;
  f.ph = ph;
  f.pcw = sub ? pw / 2 : pw;
  f.pch = sub ? ph / 2 : ph;
  f.sub = sub;
  f.nbx = pw / 8;
  f.nby = ph / 8;
  f.py = py;
  f.pc = pc;
  f.qy = qy;
  f.qc = qc;
  f.qmy = qmy;
  f.qmc = qmc;
  f.cdy = cdy;
  f.cdc = cdc;
  f.src[0] = src_y;
  f.src[1] = src_u;
  f.src[2] = src_v;
  f.rec[0] = rec_y;
  f.rec[1] = rec_u;
  f.rec[2] = rec_v;
  f.mode = mode;
  f.tx = tx;
  f.lv[0] = lv_y;
  f.lv[1] = lv_u;
  f.lv[2] = lv_v;
  const int sbc = (pw + 63) / 64, sbr = (ph + 63) / 64;
  memset(mode, 0, (size_t)f.nbx * f.nby);
  if (threads <= 1) {
    for (int r = 0; r < sbr; ++r)
      for (int c = 0; c < sbc; ++c) code_sb(f, r, c);
    return MT_OK;
  }
  // superblocks in wavefront order (d = 2 r + c, then r); each waits for its
  // left, top-left, top and top-right neighbours
  std::vector<std::pair<int, int>> order;
  for (int d = 0; d < 2 * (sbr - 1) + sbc; ++d)
    for (int r = 0; r < sbr; ++r) {
      const int c = d - 2 * r;
      if (c >= 0 && c < sbc) order.emplace_back(r, c);
    }
  std::vector<std::atomic<int>> done((size_t)sbr * sbc);
  for (auto& x : done) x.store(0);
  std::atomic<size_t> next(0);
  auto ready = [&](int r, int c) { return r < 0 || c < 0 || c >= sbc || done[(size_t)r * sbc + c].load() != 0; };
  auto worker = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= order.size()) return;
      const int r = order[i].first, c = order[i].second;
      while (!(ready(r, c - 1) && ready(r - 1, c - 1) && ready(r - 1, c) && ready(r - 1, c + 1)))
        std::this_thread::yield();
      code_sb(f, r, c);
      done[(size_t)r * sbc + c].store(1);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
  return MT_OK;
}

// The tile payloads of a decided frame in uniform tiles of tile_sb_w x
// tile_sb_h superblocks (raster order, concatenated in out; tile_lens[t] the
// length of tile t): block syntax and coefficient tokens in coding order
// (each tile's superblocks in raster order, the above contexts cleared per
// tile and the left per superblock row), each tile range coded against the
// frame-initial CDF set (cdf_data / cdf_off / cdf_len, Cdfs::new in
// semantic-slot order, copied per tile), with superblock i's cdef_idx
// (sb_cdef_idx[i], frame raster; cdef_bits wide, 0 bits: none) at its
// read_cdef() point.  slots: skip, part_bl8, part_split, kf_y, uv_mode,
// angle_delta, filter_intra, palette_y_mode, palette_uv_mode, txsz.
int or_encode_pack(int32_t pw, int32_t ph, int32_t sub, int32_t tile_sb_w, int32_t tile_sb_h, const uint8_t* mode,
                   const uint8_t* tx, const int32_t* lv_y, const int32_t* lv_u, const int32_t* lv_v,
                   const int32_t* slots, const or_emit_slots* E, const uint16_t* cdf_data, const uint32_t* cdf_off,
                   const uint16_t* cdf_len, int32_t nslots, size_t ndata, const uint8_t* sb_cdef_idx,
                   int32_t cdef_bits, int32_t updating_cdf, uint8_t* out, size_t cap, size_t* tile_lens,
                   int32_t max_tiles, int32_t* ntiles, size_t* out_len) {
  if (pw <= 0 || ph <= 0 || (pw & 7) || (ph & 7) || !slots || !E || !out_len || !ntiles || tile_sb_w <= 0 ||
      tile_sb_h <= 0)
    return MT_ERR_INVALID_INPUT;
  Frame f;
  memset(&f, 0, sizeof(f));
  f.pw = pw;
  f.ph = ph;
  f.sub = sub;
  f.nbx = pw / 8;
  f.nby = ph / 8;
  f.mode = const_cast<uint8_t*>(mode);
  f.tx = const_cast<uint8_t*>(tx);
  f.lv[0] = const_cast<int32_t*>(lv_y);
  f.lv[1] = const_cast<int32_t*>(lv_u);
  f.lv[2] = const_cast<int32_t*>(lv_v);
  SyntaxSlots L;
  memcpy(&L, slots, sizeof(L));
  Syntax syn(f, L, *E);
  const int sbc = (pw + 63) / 64, sbr = (ph + 63) / 64;
  std::vector<uint8_t> all;
  std::vector<size_t> lens;
  std::vector<uint32_t> toks;
  for (int r0 = 0; r0 < sbr; r0 += tile_sb_h)
    for (int c0 = 0; c0 < sbc; c0 += tile_sb_w) {
      const int r1 = std::min(r0 + tile_sb_h, sbr), c1 = std::min(c0 + tile_sb_w, sbc);
      std::vector<uint16_t> cdf(cdf_data, cdf_data + ndata);
      RangeCoder rc;
      syn.clear_above(c0 * 8, std::min(c1 * 8, f.nbx));
      for (int r = r0; r < r1; ++r) {
        syn.clear_left(r * 8, std::min(r * 8 + 8, f.nby));
        for (int c = c0; c < c1; ++c) {
          toks.clear();
          syn.out = &toks;
          syn.cdef_point = -1;
          syn.node(1, c * 8, r * 8, 8);
          const int i = r * sbc + c;
          for (size_t k = 0; k <= toks.size(); ++k) {
            if (cdef_bits > 0 && (int)k == syn.cdef_point) rc.literal(sb_cdef_idx[i], cdef_bits);
            if (k == toks.size()) break;
            const uint32_t t = toks[k], tag = t >> 30;
            if (tag == 0 || tag == 3) {
              const uint32_t slot = (t >> 8) & 0xffff, s = t & 0xff;
              if ((int32_t)slot >= nslots || s >= cdf_len[slot]) return MT_ERR_INVALID_INPUT;
              rc.symbol((int)s, &cdf[cdf_off[slot]], cdf_len[slot], tag == 0 && updating_cdf);
            } else if (tag == 1) {
              rc.boolean((t & 1) != 0, (t >> 1) & 0xffff);
            } else {
              const uint32_t slot = (t >> 2) & 0xffff;
              if ((int32_t)slot >= nslots || cdf_len[slot] != 10) return MT_ERR_INVALID_INPUT;
              rc.boolean((t & 2) != 0, gather(&cdf[cdf_off[slot]], (t & 1) != 0));
            }
          }
        }
      }
      const std::vector<uint8_t> bytes = rc.done();
      lens.push_back(bytes.size());
      all.insert(all.end(), bytes.begin(), bytes.end());
    }
  *ntiles = (int32_t)lens.size();
  *out_len = all.size();
  if (!tile_lens || (int32_t)lens.size() > max_tiles) return MT_ERR_TOO_LARGE;
  for (size_t t = 0; t < lens.size(); ++t) tile_lens[t] = lens[t];
  if (!out || cap < all.size()) return out ? MT_ERR_TOO_LARGE : MT_OK;
  memcpy(out, all.data(), all.size());
  return MT_OK;
}

}  // extern "C"
