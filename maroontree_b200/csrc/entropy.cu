// Host entropy path of the encoder: the AV1 multi-symbol range coder
// (src/odec.rs:35-615 OdEcEncoder, update_cdf), the frame-initial CDF set
// Cdfs::new(qctx) in its semantic-slot order (src/coder/cdfs.rs:193-355,
// :401-629), the per-tile packer that replays superblock token streams into
// one tile payload (src/coder/wavefront.rs:617-657 pack_wavefront_tile,
// src/odec.rs:315-360 replay_semantic) and the filter-syntax replay that
// inserts each 64x64 unit's cdef_idx literal at its recorded point
// (src/coder/tile_encode.rs:404-466 replay_tile_with_filters).
//
// The packer is serial per tile and stays on the host: the superblock
// decisions that produce its tokens are the data-parallel part.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <new>
#include <thread>
#include <vector>

#include "../../include/maroontree_b200.h"
#include "av1_cdfs.h"
#include "pack.h"

#if defined(__SSE2__)
#include <emmintrin.h>
#endif

namespace {

constexpr uint32_t kProbShift = 6;  // EC_PROB_SHIFT
constexpr uint32_t kMinProb = 4;    // EC_MIN_PROB
constexpr uint32_t kTagShift = 30;
constexpr uint32_t kTagMask = 3u << kTagShift;
constexpr uint32_t kTagBool = 1u << kTagShift;
constexpr uint32_t kTagNoUpdate = 3u << kTagShift;

inline int clz16(uint32_t r) { return r ? __builtin_clz(r) - 16 : 16; }  // leading zeros of a 16-bit value

}  // namespace

// ---------------------------------------------------------------------------
// The encoder.  One (fl, fh, nms) store per coded symbol; the optional trace
// keeps every store with a mark per superblock and each superblock's
// read_cdef() point so that the filter replay can re-emit the exact bytes.

struct mt_range_encoder {
  uint32_t low = 0;
  uint16_t rng = 0x8000;
  int16_t cnt = -9;
  bool updating_cdf = true;
  std::vector<uint16_t> precarry;
  bool tracing = false;
  std::vector<uint64_t> trace_ops;    // fl << 24 | fh << 8 | nms
  std::vector<uint32_t> trace_marks;  // first op of each superblock
  std::vector<uint32_t> trace_cdef;   // op index of each superblock's read_cdef(), or UINT32_MAX

  void store(uint32_t fl, uint32_t fh, uint32_t nms) {
    if (tracing) trace_ops.push_back(((uint64_t)fl << 24) | ((uint64_t)fh << 8) | nms);
    const uint32_t r = rng;
    uint32_t u = (((r >> 8) * (fl >> kProbShift)) >> (7 - kProbShift)) + kMinProb * nms;
    if (fl >= 32768) u = r;
    const uint32_t v = (((r >> 8) * (fh >> kProbShift)) >> (7 - kProbShift)) + kMinProb * (nms - 1);
    const uint32_t l = r - u;
    const uint32_t nr = (u - v) & 0xffff;
    uint32_t lo = l + low;
    int c = cnt;
    const int d = clz16(nr);
    int s = c + d;
    if (s >= 0) {
      c += 16;
      uint32_t m = (1u << c) - 1;
      if (s >= 8) {
        precarry.push_back((uint16_t)(lo >> c));
        lo &= m;
        c -= 8;
        m >>= 8;
      }
      precarry.push_back((uint16_t)(lo >> c));
      s = c + d - 24;
      lo &= m;
    }
    low = lo << d;
    rng = (uint16_t)(nr << d);
    cnt = (int16_t)s;
  }

  void encode_bool(bool val, uint16_t f) {
    const uint32_t s = val ? 1 : 0;
    store(s ? f : 32768u, s ? 0u : f, 2 - s);
  }

  void encode_symbol_noupdate(int s, const uint16_t* cdf, int len) {
    const uint32_t nms = (uint32_t)(len - s);
    store(s > 0 ? cdf[s - 1] : 32768u, cdf[s], nms);
  }

  void encode_symbol(int s, uint16_t* cdf, int len) {
    encode_symbol_noupdate(s, cdf, len);
    if (updating_cdf) update_cdf(cdf, len, s);
  }

  static void update_cdf(uint16_t* cdf, int n, int val) {
    const uint32_t count = cdf[n - 1];
    const uint32_t rate = 3 + (uint32_t)((n >> 1) < 2 ? (n >> 1) : 2) + (count >> 4);
    cdf[n - 1] = (uint16_t)(count + 1 - (count >> 5));
    // entries below val move up towards 32768, the others down towards 0
    for (int i = 0; i < n - 1; ++i) {
      const uint32_t c = cdf[i];
      const uint32_t up = c + ((32768u - c) >> rate), dn = c - (c >> rate);
      cdf[i] = (uint16_t)(i < val ? up : dn);
    }
  }

  void encode_literal(uint32_t value, uint32_t bits) {
    for (int i = (int)bits - 1; i >= 0; --i) encode_bool(((value >> i) & 1) != 0, 16384);
  }

  void encode_ns(uint32_t v, uint32_t n) {
    if (n <= 1) return;
    uint32_t w = 0;
    while ((1u << w) < n) ++w;  // ceil(log2(n)), n >= 2
    const uint32_t m = (1u << w) - n;
    if (v < m) {
      encode_literal(v, w - 1);
    } else {
      const uint32_t coded = v + m;
      encode_literal(coded >> 1, w - 1);
      encode_bool((coded & 1) != 0, 16384);
    }
  }

  void encode_subexp(uint32_t v, uint32_t num_syms, uint32_t k) {
    uint32_t i = 0, mk = 0;
    for (;;) {
      const uint32_t b2 = i ? k + i - 1 : k;
      const uint32_t a = 1u << b2;
      if (num_syms <= mk + 3 * a) {
        encode_ns(v - mk, num_syms - mk);
        return;
      } else if (v < mk + a) {
        encode_bool(false, 16384);
        encode_literal(v - mk, b2);
        return;
      }
      encode_bool(true, 16384);
      ++i;
      mk += a;
    }
  }

  static uint32_t recenter_nonneg(uint32_t r, uint32_t v) {
    if (v > (r << 1)) return v;
    if (v >= r) return (v - r) << 1;
    return ((r - v) << 1) - 1;
  }

  void encode_unsigned_subexp_with_ref(uint32_t v, uint32_t mx, uint32_t k, uint32_t r) {
    const uint32_t rc = (r << 1) <= mx ? recenter_nonneg(r, v) : recenter_nonneg(mx - 1 - r, mx - 1 - v);
    encode_subexp(rc, mx, k);
  }

  void mark_sb() {
    if (!tracing) return;
    trace_marks.push_back((uint32_t)trace_ops.size());
    trace_cdef.push_back(UINT32_MAX);
  }

  void mark_cdef() {
    if (!tracing || trace_cdef.empty() || trace_cdef.back() != UINT32_MAX) return;
    trace_cdef.back() = (uint32_t)trace_ops.size();
  }

  // store() over n recorded stores, with the coder state in locals and the
  // output written through a raw pointer (each store emits at most two
  // entries): the same arithmetic without the member round trips.
  void replay(const uint64_t* ops, size_t n) {
    if (tracing) {
      for (size_t i = 0; i < n; ++i)
        store((uint32_t)(ops[i] >> 24), (uint32_t)((ops[i] >> 8) & 0xffff), (uint32_t)(ops[i] & 0xff));
      return;
    }
    const size_t base = precarry.size();
    precarry.resize(base + 2 * n);
    uint16_t* pc = precarry.data() + base;
    uint32_t lo_s = low, r = rng;
    int c_s = cnt;
    for (size_t i = 0; i < n; ++i) {
      const uint64_t op = ops[i];
      const uint32_t fl = (uint32_t)(op >> 24), fh = (uint32_t)((op >> 8) & 0xffff), nms = (uint32_t)(op & 0xff);
      uint32_t u = (((r >> 8) * (fl >> kProbShift)) >> (7 - kProbShift)) + kMinProb * nms;
      u = fl >= 32768 ? r : u;
      const uint32_t v = (((r >> 8) * (fh >> kProbShift)) >> (7 - kProbShift)) + kMinProb * (nms - 1);
      const uint32_t nr = (u - v) & 0xffff;
      uint32_t lo = (r - u) + lo_s;
      int c = c_s;
      const int d = clz16(nr);
      int sh = c + d;
      if (sh >= 0) {
        c += 16;
        uint32_t m = (1u << c) - 1;
        if (sh >= 8) {
          *pc++ = (uint16_t)(lo >> c);
          lo &= m;
          c -= 8;
          m >>= 8;
        }
        *pc++ = (uint16_t)(lo >> c);
        sh = c + d - 24;
        lo &= m;
      }
      lo_s = lo << d;
      r = (nr << d) & 0xffff;
      c_s = sh;
    }
    precarry.resize((size_t)(pc - precarry.data()));
    low = lo_s;
    rng = (uint16_t)r;
    cnt = (int16_t)c_s;
  }

  std::vector<uint8_t> done() {
    const uint32_t l = low;
    int c = cnt;
    int s = 10;
    const uint32_t m = 0x3FFF;
    uint32_t e = ((l + m) & ~m) | (m + 1);
    s += c;
    if (s > 0) {
      uint32_t n = (1u << (c + 16)) - 1;
      do {
        precarry.push_back((uint16_t)(e >> (c + 16)));
        e &= n;
        s -= 8;
        c -= 8;
        n >>= 8;
      } while (s > 0);
    }
    std::vector<uint8_t> out(precarry.size());
    uint32_t carry = 0;
    for (size_t o = precarry.size(); o-- > 0;) {
      carry += precarry[o];
      out[o] = (uint8_t)carry;
      carry >>= 8;
    }
    return out;
  }
};

namespace {

// ---------------------------------------------------------------------------
// Cdfs::new(qctx) as a flat list of inverse CDFs (counter word last) in the
// semantic-slot order of src/coder/cdfs.rs:193-355.  The AV1 default values
// come from av1_cdfs.h; the few the reference writes inline in Cdfs::new
// (src/coder/cdfs.rs:506-627, :71-79 TXPART_CDF) are listed here.

struct CdfSet {
  std::vector<uint16_t> data;
  std::vector<uint32_t> off;
  std::vector<uint16_t> len;

  void push(const uint16_t* vals, int nvals) {  // icdf(vals): 32768 - v, then the counter 0
    off.push_back((uint32_t)data.size());
    len.push_back((uint16_t)(nvals + 1));
    for (int k = 0; k < nvals; ++k) data.push_back((uint16_t)(32768 - vals[k]));
    data.push_back(0);
  }
  void push1(uint16_t v) { push(&v, 1); }
  void rows(const uint16_t* t, int nrows, int width) {
    for (int r = 0; r < nrows; ++r) push(t + r * width, width);
  }
  void singles(const uint16_t* t, int n) {
    for (int k = 0; k < n; ++k) push1(t[k]);
  }
};

void build_cdfs(int q, CdfSet& c, mt_cdf_slot_layout* L = nullptr) {
  mt_cdf_slot_layout dummy;
  if (!L) L = &dummy;
  auto at = [&]() { return (int32_t)c.off.size(); };
  static const uint16_t kTxpart[7][3] = {{28581, 23846, 20847}, {24315, 18196, 12133}, {18791, 10887, 11005},
                                         {27179, 20004, 11281}, {26549, 19308, 14224}, {28015, 21546, 14400},
                                         {28165, 22401, 16088}};
  static const uint16_t kTxtpInter2[11] = {770, 2421, 5225, 12907, 15819, 18927, 21561, 24089, 26595, 28526, 30529};
  static const uint16_t kTxtpInter3[4] = {16384, 4167, 1998, 748};
  static const uint16_t kMvJoint[3] = {4096, 11264, 19328};
  static const uint16_t kMvClasses[10] = {28672, 30976, 31858, 32320, 32551, 32656, 32740, 32757, 32762, 32767};
  static const uint16_t kMvClassN[10] = {17408, 17920, 18944, 20480, 22528, 24576, 28672, 29952, 29952, 30720};
  static const uint16_t kPaletteUvMode[2] = {32461, 21488};
  static const uint16_t kDeltaQ[3] = {28160, 32120, 32677};
  static const uint16_t kWienerRestore = 11570;

  L->skip = at();
  c.singles(MT_CDF_SKIP_CDF, 3);                     // skip [3 ctx]
  L->intrabc = at();
  c.push1(30531);                                    // intrabc
  c.singles(&kTxpart[0][0], 21);                     // txpart [7][3]
  c.push(kTxtpInter2, 11);                           // txtp_inter2
  c.singles(kTxtpInter3, 4);                         // txtp_inter3 [4]
  c.push(kMvJoint, 3);                               // mv_joint
  for (int k = 0; k < 2; ++k) c.push1(16384);        // mv_sign [2]
  for (int k = 0; k < 2; ++k) c.push(kMvClasses, 10);  // mv_classes [2]
  for (int k = 0; k < 2; ++k) c.push1(27648);        // mv_class0 [2]
  for (int k = 0; k < 2; ++k) c.singles(kMvClassN, 10);  // mv_class_n [2][10]
  L->part_bl8 = at();
  c.rows(MT_CDF_PART_BL8_CDF, 4, 3);                 // part_bl8 [4 ctx]
  L->part_split = at();
  c.rows(MT_CDF_PART_SPLIT_CDF, 12, 9);              // part_split [3 levels][4 ctx]
  L->kf_y = at();
  c.rows(MT_CDF_KF_Y_MODE_CDF, 25, 12);              // kf_y [above * 5 + left]
  L->uv_mode = at();
  c.rows(MT_CDF_UV_MODE_NOCFL_CDF, 13, 12);          // uv_mode, CfL not allowed [13]
  c.rows(MT_CDF_UV_MODE_CFL_CDF, 13, 13);            // uv_mode, CfL allowed [13]
  L->angle_delta = at();
  c.rows(MT_CDF_ANGLE_DELTA_CDF, 8, 6);              // angle_delta [8]
  L->filter_intra = at();
  c.singles(MT_CDF_FILTER_INTRA_CDF, 22);            // filter_intra [22 block sizes]
  L->filter_intra_mode = at();
  c.push(MT_CDF_FILTER_INTRA_MODE_CDF, 4);           // filter_intra_mode
  L->palette_y_mode = at();
  c.singles(MT_CDF_PALETTE_Y_MODE, 21);              // palette_y_mode [7][3]
  L->palette_y_size = at();
  c.rows(MT_CDF_PALETTE_Y_SIZE, 7, 6);               // palette_y_size [7]
  L->palette_uv_mode = at();
  c.singles(kPaletteUvMode, 2);                      // palette_uv_mode [2]
  {
    const uint16_t* p = MT_CDF_PALETTE_Y_COLOR;      // palette_y_color [size 2..8][5 ctx]
    for (int n = 2; n <= 8; ++n)
      for (int ctx = 0; ctx < 5; ++ctx, p += n - 1) c.push(p, n - 1);
  }
  c.rows(MT_CDF_PALETTE_UV_SIZE, 7, 6);              // palette_uv_size [7]
  {
    const uint16_t* p = MT_CDF_PALETTE_UV_COLOR;     // palette_uv_color [size 2..8][5 ctx]
    for (int n = 2; n <= 8; ++n)
      for (int ctx = 0; ctx < 5; ++ctx, p += n - 1) c.push(p, n - 1);
  }
  L->cfl_sign = at();
  c.push(MT_CDF_CFL_SIGN_CDF, 7);                    // cfl_sign
  L->cfl_alpha = at();
  c.rows(MT_CDF_CFL_ALPHA_CDF, 6, 15);               // cfl_alpha [6]
  L->txsz = at();
  c.rows(MT_CDF_TXSZ_CAT0_CDF, 3, 1);                // txsz [4 cats][3 ctx]
  c.rows(MT_CDF_TXSZ_CAT1_CDF, 3, 2);
  c.rows(MT_CDF_TXSZ_CAT2_CDF, 3, 2);
  c.rows(MT_CDF_TXSZ_CAT3_CDF, 3, 2);
  L->txtp8 = at();
  c.rows(MT_CDF_TXTP_INTRA1_TX8, 13, 6);             // txtp (TX_8X8) [13 y modes]
  L->txtp4 = at();
  c.rows(MT_CDF_TXTP_INTRA1_TX4, 13, 6);             // txtp4
  L->txtp16 = at();
  c.rows(MT_CDF_TXTP_INTRA2_TX16, 13, 4);            // txtp16
  const uint16_t* skip[5] = {MT_CDF_SKIP_TX4, MT_CDF_SKIP_TX8, MT_CDF_SKIP_TX16, MT_CDF_SKIP_TX32, MT_CDF_SKIP_TX64};
  for (int k = 0; k < 5; ++k) {
    L->txb_skip[k] = at();
    c.singles(skip[k] + q * 13, 13);  // txb_skip [5 classes][13]
  }
  struct Pl { const uint16_t* t; int rows; };
  const Pl base[5][2] = {{{MT_CDF_BASE_TOK_TX4_LUMA_Q, 41}, {MT_CDF_BASE_TOK_TX4_CHROMA_Q, 41}},
                         {{MT_CDF_BASE_TOK_TX8_LUMA_Q, 41}, {MT_CDF_BASE_TOK_TX8_CHROMA_Q, 41}},
                         {{MT_CDF_BASE_TOK_TX16_LUMA_Q, 42}, {MT_CDF_BASE_TOK_TX16_CHROMA_Q, 42}},
                         {{MT_CDF_BASE_TOK_TX32_LUMA_Q, 42}, {MT_CDF_BASE_TOK_TX32_CHROMA_Q, 42}},
                         {{MT_CDF_BASE_TOK_TX64_LUMA_Q, 42}, {nullptr, 0}}};
  for (int k = 0; k < 5; ++k)
    for (int p = 0; p < 2; ++p) {
      L->base_tok[k][p] = base[k][p].t ? at() : -1;
      if (base[k][p].t) c.rows(base[k][p].t + q * base[k][p].rows * 3, base[k][p].rows, 3);
    }
  const uint16_t* br[4][2] = {{MT_CDF_BR_TOK_TX4_LUMA_Q, MT_CDF_BR_TOK_TX4_CHROMA_Q},
                              {MT_CDF_BR_TOK_TX8_LUMA_Q, MT_CDF_BR_TOK_TX8_CHROMA_Q},
                              {MT_CDF_BR_TOK_TX16_LUMA_Q, MT_CDF_BR_TOK_TX16_CHROMA_Q},
                              {MT_CDF_BR_TOK_TX32_LUMA_Q, MT_CDF_BR_TOK_TX32_CHROMA_Q}};
  for (int k = 0; k < 4; ++k)
    for (int p = 0; p < 2; ++p) {
      L->br_tok[k][p] = at();
      c.rows(br[k][p] + q * 21 * 3, 21, 3);
    }
  const uint16_t* eb[5][2] = {{MT_CDF_EOB_BASE_TX4_LUMA_Q, MT_CDF_EOB_BASE_TX4_CHROMA_Q},
                              {MT_CDF_EOB_BASE_TX8_LUMA_Q, MT_CDF_EOB_BASE_TX8_CHROMA_Q},
                              {MT_CDF_EOB_BASE_TX16_LUMA_Q, MT_CDF_EOB_BASE_TX16_CHROMA_Q},
                              {MT_CDF_EOB_BASE_TX32_LUMA_Q, MT_CDF_EOB_BASE_TX32_CHROMA_Q},
                              {MT_CDF_EOB_BASE_TX64_LUMA_Q, nullptr}};
  for (int k = 0; k < 5; ++k)
    for (int p = 0; p < 2; ++p) {
      L->eob_base[k][p] = eb[k][p] ? at() : -1;
      if (eb[k][p]) c.rows(eb[k][p] + q * 4 * 2, 4, 2);
    }
  const uint16_t* eh[5][2] = {{MT_CDF_EOB_HI_TX4_LUMA, MT_CDF_EOB_HI_TX4_CHROMA},
                              {MT_CDF_EOB_HI_TX8_LUMA, MT_CDF_EOB_HI_TX8_CHROMA},
                              {MT_CDF_EOB_HI_TX16_LUMA, MT_CDF_EOB_HI_TX16_CHROMA},
                              {MT_CDF_EOB_HI_TX32_LUMA, MT_CDF_EOB_HI_TX32_CHROMA},
                              {MT_CDF_EOB_HI_TX64_LUMA, nullptr}};
  for (int k = 0; k < 5; ++k)
    for (int p = 0; p < 2; ++p) {
      L->eob_hi[k][p] = eh[k][p] ? at() : -1;
      if (eh[k][p]) c.singles(eh[k][p] + q * 11, 11);
    }
  L->dc_sign[0] = at();
  c.singles(MT_CDF_DC_SIGN_Q + (q * 2 + 0) * 3, 3);  // dc_sign [plane][3]
  L->dc_sign[1] = at();
  c.singles(MT_CDF_DC_SIGN_Q + (q * 2 + 1) * 3, 3);
  L->eob_bin = at();  // 16_c, 16_l, 32_c, 32_l, 64_l, 16_l1d, 64_l1d, 128_l1d, 64_c, 256_l, 256_c,
                      // 128_c, 128_l, 1024_l, 1024_c, 512_c, 512_l
  c.push(MT_CDF_EOB_BIN_16_CHROMA + q * 4, 4);
  c.push(MT_CDF_EOB_BIN_16_LUMA + q * 4, 4);
  c.push(MT_CDF_EOB_BIN_32_CHROMA + q * 5, 5);
  c.push(MT_CDF_EOB_BIN_32_LUMA + q * 5, 5);
  c.push(MT_CDF_EOB_BIN_64_LUMA + q * 6, 6);
  c.push(MT_CDF_EOB_BIN_16_LUMA_1D + q * 4, 4);
  c.push(MT_CDF_EOB_BIN_64_LUMA_1D + q * 6, 6);
  c.push(MT_CDF_EOB_BIN_128_LUMA_1D + q * 7, 7);
  c.push(MT_CDF_EOB_BIN_64_CHROMA + q * 6, 6);
  c.push(MT_CDF_EOB_BIN_256_LUMA + q * 8, 8);
  c.push(MT_CDF_EOB_BIN_256_CHROMA + q * 8, 8);
  c.push(MT_CDF_EOB_BIN_128_CHROMA + q * 7, 7);
  c.push(MT_CDF_EOB_BIN_128_LUMA + q * 7, 7);
  c.push(MT_CDF_EOB_BIN_1024_LUMA + q * 10, 10);
  c.push(MT_CDF_EOB_BIN_1024_CHROMA + q * 10, 10);
  c.push(MT_CDF_EOB_BIN_512_CHROMA + q * 9, 9);
  c.push(MT_CDF_EOB_BIN_512_LUMA + q * 9, 9);
  L->delta_q = at();
  c.push(kDeltaQ, 3);          // delta_q
  L->wiener_restore = at();
  c.push1(kWienerRestore);     // wiener_restore
  L->nslots = at();
}

// The packers' CdfSet carries this many spare entries past its last CDF, so
// that every CDF can be read and written back eight entries at a time.
constexpr size_t kCdfPad = 16;

// update_cdf on a CDF of the padded CdfSet: the same per-entry arithmetic
// (entries below val move up towards 32768 by (32768 - c) >> rate, the others
// down by c >> rate), eight 16-bit lanes at a time; lanes at or past the
// counter are written back unchanged, and the counter is updated last.
inline void update_cdf_padded(uint16_t* cdf, int n, int val) {
#if defined(__SSE2__)
  const uint32_t count = cdf[n - 1];
  const uint32_t rate = 3 + (uint32_t)((n >> 1) < 2 ? (n >> 1) : 2) + (count >> 4);
  const __m128i sh = _mm_cvtsi32_si128((int)rate);
  const __m128i top = _mm_set1_epi16((short)0x8000);
  const __m128i vv = _mm_set1_epi16((short)val), nn = _mm_set1_epi16((short)(n - 1));
  __m128i idx = _mm_setr_epi16(0, 1, 2, 3, 4, 5, 6, 7);
  for (int b = 0; b < n - 1; b += 8) {
    __m128i* p = reinterpret_cast<__m128i*>(cdf + b);
    const __m128i c = _mm_loadu_si128(p);
    const __m128i up = _mm_add_epi16(c, _mm_srl_epi16(_mm_sub_epi16(top, c), sh));
    const __m128i dn = _mm_sub_epi16(c, _mm_srl_epi16(c, sh));
    const __m128i is_up = _mm_cmplt_epi16(idx, vv);
    const __m128i live = _mm_cmplt_epi16(idx, nn);
    __m128i r = _mm_or_si128(_mm_and_si128(is_up, up), _mm_andnot_si128(is_up, dn));
    r = _mm_or_si128(_mm_and_si128(live, r), _mm_andnot_si128(live, c));
    _mm_storeu_si128(p, r);
    idx = _mm_add_epi16(idx, _mm_set1_epi16(8));
  }
  cdf[n - 1] = (uint16_t)(count + 1 - (count >> 5));
#else
  mt_range_encoder::update_cdf(cdf, n, val);
#endif
}

// gather_split_prob_icdf (src/coeffs.rs:2927-2935): the edge partition's
// split probability read from a live 10-symbol partition CDF.
uint16_t gather_split_prob(const uint16_t* cdf, bool top) {
  auto v = [&](int s) { return (int32_t)cdf[s]; };
  int32_t out = top ? (v(1) - v(4)) + v(5) + (v(8) - v(7)) : (v(0) - v(1)) + (v(2) - v(6)) + (v(7) - v(8));
  if (out < 1) out = 1;
  if (out > 32767) out = 32767;
  return (uint16_t)out;
}

// One superblock's semantic stream against the live CDF set
// (src/odec.rs:315-360).  At the read_cdef() point the trace is marked and,
// when cdef_bits > 0, the unit's cdef_idx is coded there as a raw literal.
// Returns false on a malformed token.
bool replay_tokens(mt_range_encoder& enc, CdfSet& c, const uint32_t* ops, uint32_t n, int32_t cdef_point,
                   int cdef_bits = 0, uint32_t cdef_idx = 0) {
  const size_t nslots = c.off.size();
  uint16_t* const data = c.data.data();
  const uint32_t* const off = c.off.data();
  const uint16_t* const lens = c.len.data();
  for (uint32_t i = 0; i < n; ++i) {
    if (cdef_point >= 0 && (uint32_t)cdef_point == i) {
      enc.mark_cdef();
      if (cdef_bits > 0) enc.encode_literal(cdef_idx, (uint32_t)cdef_bits);
    }
    const uint32_t t = ops[i];
    const uint32_t tag = t & kTagMask;
    if (tag == 0 || tag == kTagNoUpdate) {
      const uint32_t slot = (t >> 8) & 0xffff, s = t & 0xff;
      if (slot >= nslots || s >= lens[slot]) return false;
      uint16_t* cdf = data + off[slot];
      enc.encode_symbol_noupdate((int)s, cdf, lens[slot]);
      if (tag == 0 && enc.updating_cdf) update_cdf_padded(cdf, lens[slot], (int)s);
    } else if (tag == kTagBool) {
      enc.encode_bool((t & 1) != 0, (uint16_t)((t >> 1) & 0xffff));
    } else {  // gathered partition bool (tag 2)
      const uint32_t slot = (t >> 2) & 0xffff;
      if (slot >= nslots || lens[slot] != 10) return false;
      const uint16_t p = gather_split_prob(data + off[slot], (t & 1) != 0);
      enc.encode_bool((t & 2) != 0, p);
    }
  }
  if (cdef_point >= 0 && (uint32_t)cdef_point == n) {
    enc.mark_cdef();
    if (cdef_bits > 0) enc.encode_literal(cdef_idx, (uint32_t)cdef_bits);
  }
  return true;
}

int out_bytes(const std::vector<uint8_t>& v, uint8_t** out, size_t* out_len) {
  uint8_t* p = (uint8_t*)malloc(v.size() ? v.size() : 1);
  if (!p) return MT_ERR_ALLOC;
  if (!v.empty()) memcpy(p, v.data(), v.size());
  *out = p;
  *out_len = v.size();
  return MT_OK;
}

}  // namespace

struct mt_tile_trace {
  std::vector<uint64_t> ops;
  std::vector<uint32_t> marks;
  std::vector<uint32_t> cdef;
};

extern "C" {

mt_range_encoder* mt_range_encoder_new(int32_t updating_cdf) {
  mt_range_encoder* e = new (std::nothrow) mt_range_encoder();
  if (e) e->updating_cdf = updating_cdf != 0;
  return e;
}

void mt_range_encoder_free(mt_range_encoder* e) { delete e; }

int mt_range_encode_bool(mt_range_encoder* e, int32_t value, uint16_t f) {
  if (!e || f == 0 || f >= 32768) return MT_ERR_INVALID_INPUT;
  e->encode_bool(value != 0, f);
  return MT_OK;
}

int mt_range_encode_symbol(mt_range_encoder* e, int32_t s, uint16_t* cdf, int32_t len, int32_t adapt) {
  if (!e || !cdf || len < 2 || s < 0 || s >= len) return MT_ERR_INVALID_INPUT;
  if (adapt)
    e->encode_symbol(s, cdf, len);
  else
    e->encode_symbol_noupdate(s, cdf, len);
  return MT_OK;
}

int mt_range_encode_literal(mt_range_encoder* e, uint32_t value, uint32_t bits) {
  if (!e || bits > 32) return MT_ERR_INVALID_INPUT;
  e->encode_literal(value, bits);
  return MT_OK;
}

int mt_range_encode_signed_subexp_with_ref(mt_range_encoder* e, int32_t v, int32_t low, int32_t high, uint32_t k,
                                           int32_t r) {
  if (!e || high <= low || v < low || v >= high || r < low || r >= high) return MT_ERR_INVALID_INPUT;
  e->encode_unsigned_subexp_with_ref((uint32_t)(v - low), (uint32_t)(high - low), k, (uint32_t)(r - low));
  return MT_OK;
}

int mt_range_encoder_done(mt_range_encoder* e, uint8_t** out, size_t* out_len) {
  if (!e || !out || !out_len) return MT_ERR_INVALID_INPUT;
  int rc = out_bytes(e->done(), out, out_len);
  delete e;
  return rc;
}

int mt_cdf_layout(mt_cdf_slot_layout* out) {
  if (!out) return MT_ERR_INVALID_INPUT;
  CdfSet c;
  build_cdfs(0, c, out);
  return MT_OK;
}

int32_t mt_cdf_slot_count(void) {
  CdfSet c;
  build_cdfs(0, c);
  return (int32_t)c.off.size();
}

int mt_cdfs_default(int32_t qctx, uint16_t* data, size_t data_cap, uint32_t* offsets, uint16_t* lens,
                    int32_t slots_cap, size_t* data_len, int32_t* nslots) {
  if (qctx < 0 || qctx > 3) return MT_ERR_INVALID_INPUT;
  CdfSet c;
  build_cdfs(qctx, c);
  if (data_len) *data_len = c.data.size();
  if (nslots) *nslots = (int32_t)c.off.size();
  if (!data && !offsets && !lens) return MT_OK;
  if (data_cap < c.data.size() || slots_cap < (int32_t)c.off.size() || !data || !offsets || !lens)
    return MT_ERR_TOO_LARGE;
  memcpy(data, c.data.data(), c.data.size() * sizeof(uint16_t));
  memcpy(offsets, c.off.data(), c.off.size() * sizeof(uint32_t));
  memcpy(lens, c.len.data(), c.len.size() * sizeof(uint16_t));
  return MT_OK;
}

int mt_pack_tile(uint8_t base_q_idx, int32_t updating_cdf, const uint32_t* ops, const uint32_t* sb_start,
                 const int32_t* sb_cdef_point, int32_t nsb, uint8_t** payload, size_t* payload_len,
                 mt_tile_trace** trace) {
  if (!payload || !payload_len || nsb < 0 || (nsb > 0 && (!ops || !sb_start))) return MT_ERR_INVALID_INPUT;
  for (int32_t i = 0; i < nsb; ++i)
    if (sb_start[i + 1] < sb_start[i]) return MT_ERR_INVALID_INPUT;
  int q = base_q_idx <= 20 ? 0 : base_q_idx <= 60 ? 1 : base_q_idx <= 120 ? 2 : 3;  // qcat
  CdfSet c;
  build_cdfs(q, c);
  c.data.resize(c.data.size() + kCdfPad, 0);
  mt_range_encoder enc;
  enc.updating_cdf = updating_cdf != 0;
  enc.tracing = trace != nullptr;
  if (nsb > 0) enc.precarry.reserve(sb_start[nsb] / 2 + 64);
  for (int32_t i = 0; i < nsb; ++i) {
    enc.mark_sb();
    const int32_t cp = sb_cdef_point ? sb_cdef_point[i] : -1;
    if (!replay_tokens(enc, c, ops + sb_start[i], sb_start[i + 1] - sb_start[i], cp)) return MT_ERR_INVALID_INPUT;
  }
  if (trace) {
    mt_tile_trace* t = new (std::nothrow) mt_tile_trace();
    if (!t) return MT_ERR_ALLOC;
    t->ops.swap(enc.trace_ops);
    t->marks.swap(enc.trace_marks);
    t->cdef.swap(enc.trace_cdef);
    *trace = t;
  }
  return out_bytes(enc.done(), payload, payload_len);
}

int mt_pack_tile_filtered(uint8_t base_q_idx, int32_t updating_cdf, const uint32_t* ops, const uint32_t* sb_start,
                          const int32_t* sb_cdef_point, int32_t nsb, const uint8_t* sb_cdef_idx, int32_t cdef_bits,
                          uint8_t** payload, size_t* payload_len) {
  if (!payload || !payload_len || nsb < 0 || (nsb > 0 && (!ops || !sb_start))) return MT_ERR_INVALID_INPUT;
  if (cdef_bits < 0 || cdef_bits > 3 || (cdef_bits > 0 && (!sb_cdef_idx || !sb_cdef_point)))
    return MT_ERR_INVALID_INPUT;
  for (int32_t i = 0; i < nsb; ++i) {
    if (sb_start[i + 1] < sb_start[i]) return MT_ERR_INVALID_INPUT;
    if (cdef_bits > 0 && sb_cdef_point[i] >= 0 && sb_cdef_idx[i] >= (1u << cdef_bits)) return MT_ERR_INVALID_INPUT;
  }
  const int q = base_q_idx <= 20 ? 0 : base_q_idx <= 60 ? 1 : base_q_idx <= 120 ? 2 : 3;  // qcat
  CdfSet c;
  build_cdfs(q, c);
  c.data.resize(c.data.size() + kCdfPad, 0);
  mt_range_encoder enc;
  enc.updating_cdf = updating_cdf != 0;
  if (nsb > 0) enc.precarry.reserve(sb_start[nsb] / 2 + 64);
  for (int32_t i = 0; i < nsb; ++i) {
    const int32_t cp = sb_cdef_point ? sb_cdef_point[i] : -1;
    if (!replay_tokens(enc, c, ops + sb_start[i], sb_start[i + 1] - sb_start[i], cp, cdef_bits,
                       cdef_bits > 0 ? sb_cdef_idx[i] : 0))
      return MT_ERR_INVALID_INPUT;
  }
  return out_bytes(enc.done(), payload, payload_len);
}

void mt_tile_trace_free(mt_tile_trace* t) { delete t; }

int mt_replay_tile_with_filters(const mt_tile_trace* t, int32_t tile_x0, int32_t tile_y0, int32_t tile_w,
                                int32_t tile_h, const uint8_t* cdef_grid, int32_t unit_cols, int32_t grid_len,
                                int32_t cdef_bits, int32_t updating_cdf, uint8_t** out, size_t* out_len) {
  if (!t || !out || !out_len || tile_w <= 0 || tile_h <= 0) return MT_ERR_INVALID_INPUT;
  if (cdef_grid && (cdef_bits < 1 || cdef_bits > 3 || unit_cols <= 0)) return MT_ERR_INVALID_INPUT;
  const int sb_cols = (tile_w + 63) / 64, sb_rows = (tile_h + 63) / 64;
  if ((size_t)sb_cols * sb_rows != t->marks.size()) return MT_ERR_INVALID_INPUT;
  mt_range_encoder enc;
  enc.updating_cdf = updating_cdf != 0;
  size_t i = 0;
  for (int sy = 0; sy < tile_h; sy += 64) {
    for (int sx = 0; sx < tile_w; sx += 64, ++i) {
      const size_t a = t->marks[i];
      const size_t b = i + 1 < t->marks.size() ? t->marks[i + 1] : t->ops.size();
      const uint32_t p = t->cdef[i];
      if (!cdef_grid || p == UINT32_MAX) {
        enc.replay(&t->ops[a], b - a);
        continue;
      }
      enc.replay(&t->ops[a], p - a);
      // The SB has a non-skip block: its 64x64 unit's index as a raw literal.
      const int u = ((tile_y0 + sy) / 64) * unit_cols + (tile_x0 + sx) / 64;
      const uint32_t idx = (u >= 0 && u < grid_len) ? cdef_grid[u] : 0;
      enc.encode_literal(idx, (uint32_t)cdef_bits);
      enc.replay(&t->ops[p], b - p);
    }
  }
  return out_bytes(enc.done(), out, out_len);
}

void mt_free(void* p) { free(p); }

}  // extern "C"

// ---------------------------------------------------------------------------
// The tile packer in two phases for the encoder.  Every token is one store of
// the range coder, and which store it is depends only on the token and the
// adapted CDFs, never on the coder's state or on the cdef_idx literals (raw
// bits, no CDF).  Phase 1 turns the superblocks' tokens into their stores
// (fl, fh, nms, as the tile trace holds them) with the CDF adaptation, reading
// the syntax tokens and the coefficient blocks they point to in place; phase 2
// runs the coder over the stores with each superblock's cdef_idx inserted at
// its read_cdef() point.  Phase 1 can start as soon as the tokens exist, before
// the CDEF decision is made, and phase 2 follows it superblock by superblock
// on another thread.  The bytes are those of mt_pack_tile_filtered over the
// spliced token stream.

namespace mth {

constexpr uint32_t kCoefMarker = 0xFFFFFFFFu;

// The store of one token against the live CDFs, with the CDF update; false
// for a malformed token.
inline bool token_store(uint32_t t, uint16_t* data, const uint32_t* off, const uint16_t* lens, size_t nslots,
                        bool updating, uint64_t& st) {
  const uint32_t tag = t & kTagMask;
  if (tag == 0 || tag == kTagNoUpdate) {
    const uint32_t slot = (t >> 8) & 0xffff, s = t & 0xff;
    if (slot >= nslots || s >= lens[slot]) return false;
    uint16_t* cdf = data + off[slot];
    const uint32_t fl = s > 0 ? cdf[s - 1] : 32768u;
    st = ((uint64_t)fl << 24) | ((uint64_t)cdf[s] << 8) | (uint64_t)(lens[slot] - s);
    if (tag == 0 && updating) update_cdf_padded(cdf, lens[slot], (int)s);
  } else {
    uint32_t b, p;
    if (tag == kTagBool) {
      b = t & 1;
      p = (t >> 1) & 0xffff;
    } else {  // gathered partition bool
      const uint32_t slot = (t >> 2) & 0xffff;
      if (slot >= nslots || lens[slot] != 10) return false;
      b = (t >> 1) & 1;
      p = gather_split_prob(data + off[slot], (t & 1) != 0);
    }
    st = b ? (((uint64_t)p << 24) | 1u) : (((uint64_t)32768u << 24) | ((uint64_t)p << 8) | 2u);
  }
  return true;
}

// Which phase-1 worker codes token t: symbols and gathered bools by their
// CDF slot's parity, raw-bit bools on worker 0.
inline int token_part(uint32_t t) {
  const uint32_t tag = t & kTagMask;
  if (tag == kTagBool) return 0;
  const uint32_t slot = tag == 0 || tag == kTagNoUpdate ? (t >> 8) & 0xffff : (t >> 2) & 0xffff;
  return (int)(slot % (uint32_t)kTracers);
}

void trace_tile_stores(uint8_t base_q_idx, int32_t updating_cdf, const std::vector<uint32_t>* sbs, int nsb,
                       const int32_t* cdef_point, const uint32_t* toks, const uint32_t* offs, size_t first_coef,
                       TileStores* out, int part) {
  const int q = base_q_idx <= 20 ? 0 : base_q_idx <= 60 ? 1 : base_q_idx <= 120 ? 2 : 3;  // qcat
  CdfSet c;
  build_cdfs(q, c);
  c.data.resize(c.data.size() + kCdfPad, 0);
  uint16_t* const data = c.data.data();
  const uint32_t* const off = c.off.data();
  const uint16_t* const lens = c.len.data();
  const size_t nslots = c.off.size(), cap = out->st.size();
  const bool upd = updating_cdf != 0;
  uint64_t* const w = out->st.data();
  size_t n = 0, k = first_coef;
  for (int i = 0; i < nsb; ++i) {
    const std::vector<uint32_t>& syn = sbs[i];
    uint32_t at = UINT32_MAX;
    bool ok = true;
    for (size_t t = 0; t < syn.size() && ok; ++t) {
      if ((int32_t)t == cdef_point[i]) at = (uint32_t)n;
      const uint32_t tok = syn[t];
      if (tok == kCoefMarker) {
        const uint32_t a = offs[k], b = offs[k + 1];
        ++k;
        if (n + (b - a) > cap) ok = false;
        for (uint32_t e = a; e < b && ok; ++e, ++n)
          if (token_part(toks[e]) == part) ok = token_store(toks[e], data, off, lens, nslots, upd, w[n]);
      } else {
        ok = n < cap;
        if (ok && token_part(tok) == part) ok = token_store(tok, data, off, lens, nslots, upd, w[n]);
        ++n;
      }
    }
    if (cdef_point[i] >= 0 && (size_t)cdef_point[i] == syn.size()) at = (uint32_t)n;
    if (!ok) {
      out->failed.store(true, std::memory_order_release);
      out->done[part].store(nsb, std::memory_order_release);
      return;
    }
    if (part == 0) {
      out->sb_end[(size_t)i] = (uint32_t)n;
      out->cdef_at[(size_t)i] = at;
    }
    out->done[part].store(i + 1, std::memory_order_release);
  }
}

int code_tile_stores(TileStores* in, int nsb, int32_t updating_cdf, const uint8_t* cdef_idx, int32_t cdef_bits,
                     uint8_t** payload, size_t* payload_len) {
  mt_range_encoder enc;
  enc.updating_cdf = updating_cdf != 0;
  enc.precarry.reserve(in->st.size() / 2 + 64);
  const uint64_t* const st = in->st.data();
  size_t a = 0;
  for (int i = 0; i < nsb; ++i) {
    // every phase-1 worker always reaches nsb (failure included): the wait ends
    for (int p = 0; p < kTracers; ++p)
      while (in->done[p].load(std::memory_order_acquire) <= i) std::this_thread::yield();
    if (in->failed.load(std::memory_order_acquire)) return MT_ERR_INVALID_INPUT;
    const size_t b = in->sb_end[(size_t)i], p = in->cdef_at[(size_t)i];
    if (p == UINT32_MAX || cdef_bits <= 0) {
      enc.replay(st + a, b - a);
    } else {
      enc.replay(st + a, p - a);
      enc.encode_literal(cdef_idx[i], (uint32_t)cdef_bits);
      enc.replay(st + p, b - p);
    }
    a = b;
  }
  return out_bytes(enc.done(), payload, payload_len);
}

}  // namespace mth

