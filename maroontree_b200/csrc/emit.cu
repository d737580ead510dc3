// Coefficient token emission, batched: the square 2-D coefficient coders of
// src/coeffs.rs (encode_tx4_luma_coeffs_adapt :2414, encode_4x4_chroma_coeffs
// :2310, encode_tx8_coeffs_adapt :583, encode_tx16_coeffs_adapt :707 with
// tx16_coeffs_tail :732, encode_tx32_coeffs_adapt :848; encode_dc_tail :87,
// encode_hi_tok :71, encode_golomb :34, get_lo_ctx_2d :46) writing the semantic
// tokens the tile packer replays (src/odec.rs:96-108): one adaptive-symbol
// token per CDF symbol (slot << 8 | symbol, slots of the frame CDF set) and one
// bool token per equiprobable bit.
//
// One thread walks one transform block (the coder is a serial reverse-scan
// walk over a level map).  Blocks are independent: their contexts (txb_skip,
// dc_sign) are inputs, computed from the neighbours' final levels, so a whole
// frame's coefficients emit in one launch.  A count pass sizes every block's
// stream, an exclusive scan places them, and the write pass fills them.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"

namespace {

constexpr uint32_t kTokBool = 1u << 30;

__constant__ uint8_t eScan4[16] = {0, 4, 1, 2, 5, 8, 12, 9, 6, 3, 7, 10, 13, 14, 11, 15};
__constant__ uint8_t eScan8[64] = {0,  8,  1,  2,  9,  16, 24, 17, 10, 3,  4,  11, 18, 25, 32, 40,
                                   33, 26, 19, 12, 5,  6,  13, 20, 27, 34, 41, 48, 56, 49, 42, 35,
                                   28, 21, 14, 7,  15, 22, 29, 36, 43, 50, 57, 58, 51, 44, 37, 30,
                                   23, 31, 38, 45, 52, 59, 60, 53, 46, 39, 47, 54, 61, 62, 55, 63};
__constant__ uint16_t eScan16[256] = {MT_SCAN_16X16_LIST};
__constant__ uint8_t eLoOff[25] = {0, 1, 6, 6, 21, 1, 6, 6, 21, 21, 6, 6, 21, 21, 21,
                                   6, 21, 21, 21, 21, 21, 21, 21, 21, 21};

struct EmitArgs {
  mt_cdf_slot_layout L;
};

// Token sink: counts always, writes when out != nullptr.
struct Sink {
  uint32_t* out;
  uint32_t n;
  __device__ void sym(int32_t slot, uint32_t s) {
    if (out) out[n] = ((uint32_t)slot << 8) | s;
    ++n;
  }
  __device__ void bit(bool v) {
    if (out) out[n] = kTokBool | (16384u << 1) | (v ? 1u : 0u);
    ++n;
  }
  __device__ void golomb(uint32_t v) {  // encode_golomb: unary zeros, then x MSB-first
    const uint32_t x = v + 1;
    const int length = 32 - __clz(x);
    for (int i = 0; i < length - 1; ++i) bit(false);
    for (int i = length - 1; i >= 0; --i) bit(((x >> i) & 1) != 0);
  }
  // encode_hi_tok: the base-range ladder, 3 per symbol, 4 symbols at most.
  __device__ void hi_tok(uint32_t m, int32_t br_slot) {
    const int total = min((int)m - 3, 12);
    int coded = 0;
    for (int k = 0; k < 4; ++k) {
      const int s = min(total - coded, 3);
      sym(br_slot, (uint32_t)s);
      coded += s;
      if (s < 3) break;
    }
  }
};

__device__ __forceinline__ uint8_t level_byte(uint32_t m) {
  return m == 0 ? 0 : (m <= 2 ? (uint8_t)(m * 0x41) : (uint8_t)(min(m, 15u) + 0xC0));
}

__device__ __forceinline__ int scan_at(int lg, int i) {
  return lg == 2 ? eScan4[i] : (lg == 3 ? eScan8[i] : eScan16[i]);
}

// The 1-D classes (V_DCT vertical, H_DCT horizontal) at TX_4X4 / TX_8X8:
// encode_tx4_coeffs_1d / encode_tx8_coeffs_1d (src/coeffs.rs:264-420, :109-262).
// Class coordinates (x, y) = (i mod n, i / n); the coefficient at class index
// i is cf[(x << lg) | y] for the vertical class and cf[i] for the horizontal.
__device__ void emit_block_1d(const int32_t* __restrict__ cf, const mt_coef_block& b, const mt_cdf_slot_layout& L,
                              Sink& k, uint8_t* res_ctx) {
  const int lg = b.log2n, n = 1 << lg, area = n * n;
  const int cls = lg - 2;
  const bool vertical = b.tx_class == 1;
  auto pos_rc = [&](int i) { return vertical ? (((i & (n - 1)) << lg) | (i >> lg)) : i; };
  int eob = -1;
  for (int i = area - 1; i >= 0; --i)
    if (cf[pos_rc(i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) {
    k.sym(L.txb_skip[cls] + b.skip_ctx, 1);
    *res_ctx = 0x40;
    return;
  }
  uint32_t cul = 0;
  for (int i = 0; i <= eob; ++i) cul += (uint32_t)abs(cf[pos_rc(i)]);
  k.sym(L.txb_skip[cls] + b.skip_ctx, 0);
  k.sym((cls == 0 ? L.txtp4 : L.txtp8) + b.y_mode, vertical ? 2 : 3);
  const uint8_t dcb = cf[0] == 0 ? (1 << 6) : (cf[0] < 0 ? 0 : (2 << 6));
  *res_ctx = (uint8_t)(min(cul, 63u) | dcb);
  const int32_t eb = L.eob_bin + (cls == 0 ? 5 : 6);  // eob_bin_16_l1d / eob_bin_64_l1d
  const int32_t base = L.base_tok[cls][0], br = L.br_tok[cls][0], ebase = L.eob_base[cls][0];
  if (eob == 0) {
    k.sym(eb, 0);
    const uint32_t m = (uint32_t)abs(cf[0]);
    const uint32_t bs = min(m, 3u);
    k.sym(ebase + 0, bs - 1);
    if (bs == 3) k.hi_tok(m, br + 0);
    k.sym(L.dc_sign[0] + b.dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (m >= 15) k.golomb(m - 15);
    return;
  }
  const int eob_bin = eob < 2 ? eob : 32 - __clz((uint32_t)eob);
  k.sym(eb, (uint32_t)eob_bin);
  if (eob_bin > 1) {
    const int nbits = eob_bin - 2;
    k.sym(L.eob_hi[cls][0] + eob_bin, (uint32_t)((eob >> nbits) & 1));
    for (int bb = nbits - 1; bb >= 0; --bb) k.bit(((eob >> bb) & 1) != 0);
  }
  uint8_t levels[160];  // stride 16, zero-padded: the 1-D context reaches (x, y + 4)
  for (int i = 0; i < 160; ++i) levels[i] = 0;
  auto lo_ctx = [&](int x, int y, uint32_t* hi) {
    uint32_t mag = (uint32_t)levels[x * 16 + y + 1] + levels[(x + 1) * 16 + y] + levels[x * 16 + y + 2];
    *hi = mag;
    mag += (uint32_t)levels[x * 16 + y + 3] + levels[x * 16 + y + 4];
    return 26u + (y > 1 ? 10u : (uint32_t)y * 5u) + (mag > 512 ? 4u : (mag + 64) >> 7);
  };
  const int ctx_e = 1 + (eob > (area >> 3)) + (eob > (area >> 2));
  {
    const int x = eob & (n - 1), y = eob >> lg;
    const uint32_t m = (uint32_t)abs(cf[pos_rc(eob)]);
    const uint32_t et = min(m, 3u) - 1;
    k.sym(ebase + ctx_e, et);
    if (et == 2) k.hi_tok(m, br + (y != 0 ? 14 : 7));
    levels[x * 16 + y] = level_byte(m);
  }
  for (int i = eob - 1; i >= 1; --i) {
    const int x = i & (n - 1), y = i >> lg;
    uint32_t hi;
    const uint32_t ctx = lo_ctx(x, y, &hi);
    const uint32_t m = (uint32_t)abs(cf[pos_rc(i)]);
    const uint32_t tok = min(m, 3u);
    k.sym(base + (int32_t)ctx, tok);
    if (tok == 3) {
      const uint32_t mg = hi & 63;
      k.hi_tok(m, br + (int32_t)((y != 0 ? 14 : 7) + (mg > 12 ? 6 : (mg + 1) >> 1)));
    }
    levels[x * 16 + y] = level_byte(m);
  }
  uint32_t dhi;
  const uint32_t dctx = lo_ctx(0, 0, &dhi);
  const uint32_t dm = (uint32_t)abs(cf[0]);
  const uint32_t dt = min(dm, 3u);
  k.sym(base + (int32_t)dctx, dt);
  if (dt == 3) {
    const uint32_t mg = dhi & 63;
    k.hi_tok(dm, br + (int32_t)(mg > 12 ? 6 : (mg + 1) >> 1));
  }
  if (cf[0] != 0) {
    k.sym(L.dc_sign[0] + b.dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (dm >= 15) k.golomb(dm - 15);
  }
  for (int i = 1; i <= eob; ++i) {
    const int32_t c = cf[pos_rc(i)];
    if (c != 0) {
      k.bit(c < 0);
      if ((uint32_t)abs(c) >= 15) k.golomb((uint32_t)abs(c) - 15);
    }
  }
}

// One block's tokens (and its coefficient context byte).
__device__ void emit_block(const int32_t* __restrict__ cf, const mt_coef_block& b, const mt_cdf_slot_layout& L,
                           Sink& k, uint8_t* res_ctx) {
  const int lg = b.log2n, n = 1 << lg, area = n * n;
  const int cls = lg - 2, pl = b.plane ? 1 : 0;
  // eob and the sum of magnitudes up to it (eob_and_cul)
  int eob = -1;
  for (int i = area - 1; i >= 0; --i)
    if (cf[scan_at(lg, i)] != 0) {
      eob = i;
      break;
    }
  if (eob < 0) {
    k.sym(L.txb_skip[cls] + b.skip_ctx, 1);  // all_zero = 1
    *res_ctx = 0x40;
    return;
  }
  uint32_t cul = 0;
  for (int i = 0; i <= eob; ++i) cul += (uint32_t)abs(cf[scan_at(lg, i)]);
  k.sym(L.txb_skip[cls] + b.skip_ctx, 0);
  if (!pl && b.code_txtp) {
    const int32_t tg = cls == 0 ? L.txtp4 : (cls == 1 ? L.txtp8 : L.txtp16);
    k.sym(tg + b.y_mode, b.txtp);
  }
  const uint8_t dcb = cf[0] == 0 ? (1 << 6) : (cf[0] < 0 ? 0 : (2 << 6));
  *res_ctx = (uint8_t)(min(cul, 63u) | dcb);
  // eob_pt CDF of this size and plane (16c 16l . . 64l . . . 64c 256l 256c)
  const int eb_idx = lg == 2 ? (pl ? 0 : 1) : (lg == 3 ? (pl ? 8 : 4) : (pl ? 10 : 9));
  const int32_t eb = L.eob_bin + eb_idx;
  const int32_t base = L.base_tok[cls][pl], br = L.br_tok[cls][pl], ebase = L.eob_base[cls][pl];
  if (eob == 0) {  // encode_dc_tail
    k.sym(eb, 0);
    const uint32_t m = (uint32_t)abs(cf[0]);
    const uint32_t bs = min(m, 3u);
    k.sym(ebase + 0, bs - 1);
    if (bs == 3) k.hi_tok(m, br + 0);
    k.sym(L.dc_sign[pl] + b.dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (m >= 15) k.golomb(m - 15);
    return;
  }
  const int eob_bin = eob < 2 ? eob : 32 - __clz((uint32_t)eob);
  k.sym(eb, (uint32_t)eob_bin);
  if (eob_bin > 1) {
    const int nbits = eob_bin - 2;
    k.sym(L.eob_hi[cls][pl] + eob_bin, (uint32_t)((eob >> nbits) & 1));
    for (int bb = nbits - 1; bb >= 0; --bb) k.bit(((eob >> bb) & 1) != 0);
  }
  uint8_t levels[320];
  for (int i = 0; i < 320; ++i) levels[i] = 0;
  const int ctx_e = 1 + (eob > (area >> 3)) + (eob > (area >> 2));
  {
    const int rc = scan_at(lg, eob);
    const int ex = rc >> lg, ey = rc & (n - 1);
    const uint32_t m = (uint32_t)abs(cf[rc]);
    const uint32_t et = min(m, 3u) - 1;
    k.sym(ebase + ctx_e, et);
    if (et == 2) k.hi_tok(m, br + ((ex | ey) > 1 ? 14 : 7));
    levels[ex * n + ey] = level_byte(m);
  }
  for (int i = eob - 1; i >= 1; --i) {
    const int rc = scan_at(lg, i);
    const int x = rc >> lg, y = rc & (n - 1);
    auto g = [&](int dx, int dy) { return (uint32_t)levels[(x + dx) * n + (y + dy)]; };
    const uint32_t hi_mag = g(0, 1) + g(1, 0) + g(1, 1);
    const uint32_t mag = hi_mag + g(0, 2) + g(2, 0);
    const uint32_t ctx = eLoOff[min(y, 4) * 5 + min(x, 4)] + (mag > 512 ? 4 : (mag + 64) >> 7);
    const uint32_t m = (uint32_t)abs(cf[rc]);
    const uint32_t tok = min(m, 3u);
    k.sym(base + (int32_t)ctx, tok);
    if (tok == 3) {
      const uint32_t mg = hi_mag & 63;
      const uint32_t bc = ((y | x) > 1 ? 14 : 7) + (mg > 12 ? 6 : (mg + 1) >> 1);
      k.hi_tok(m, br + (int32_t)bc);
    }
    levels[x * n + y] = level_byte(m);
  }
  const uint32_t dm = (uint32_t)abs(cf[0]);
  const uint32_t dt = min(dm, 3u);
  k.sym(base + 0, dt);
  if (dt == 3) {
    const uint32_t mg = ((uint32_t)levels[1] + levels[n] + levels[n + 1]) & 63;
    k.hi_tok(dm, br + (int32_t)(mg > 12 ? 6 : (mg + 1) >> 1));
  }
  if (cf[0] != 0) {
    k.sym(L.dc_sign[pl] + b.dcs_ctx, cf[0] < 0 ? 1 : 0);
    if (dm >= 15) k.golomb(dm - 15);
  }
  for (int i = 1; i <= eob; ++i) {
    const int32_t c = cf[scan_at(lg, i)];
    if (c != 0) {
      k.bit(c < 0);
      if ((uint32_t)abs(c) >= 15) k.golomb((uint32_t)abs(c) - 15);
    }
  }
}

template <bool WRITE>
__global__ void __launch_bounds__(128) emit_kernel(const int32_t* __restrict__ levels,
                                                   const mt_coef_block* __restrict__ blocks, int n, EmitArgs a,
                                                   uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                                                   uint32_t* __restrict__ tokens, uint8_t* __restrict__ res_ctx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const mt_coef_block b = blocks[i];
  Sink k{WRITE ? tokens + offsets[i] : nullptr, 0};
  uint8_t rc = 0;
  if (b.tx_class)
    emit_block_1d(levels + b.cf_offset, b, a.L, k, &rc);
  else
    emit_block(levels + b.cf_offset, b, a.L, k, &rc);
  if (!WRITE) counts[i] = k.n;
  if (WRITE && res_ctx) res_ctx[i] = rc;
}

// Exclusive scan of n counts into n + 1 offsets (offsets[n] = total), one CTA.
__global__ void __launch_bounds__(1024) scan_kernel(const uint32_t* __restrict__ counts, int n,
                                                    uint32_t* __restrict__ offsets) {
  __shared__ uint32_t part[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
  uint32_t s = 0;
  for (int i = lo; i < hi; ++i) s += counts[i];
  part[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const uint32_t v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint32_t run = part[t] - s;
  for (int i = lo; i < hi; ++i) {
    offsets[i] = run;
    run += counts[i];
  }
  if (t == 1023) offsets[n] = part[1023];
}

bool check_blocks_host(const mt_coef_block* b, int32_t n) {
  for (int32_t i = 0; i < n; ++i) {
    if (b[i].log2n < 2 || b[i].log2n > 4 || b[i].plane > 1 || b[i].skip_ctx > 12 || b[i].dcs_ctx > 2 ||
        b[i].y_mode > 12)
      return false;
    const int cls = b[i].log2n - 2;
    const int ntx = cls == 2 ? 5 : 7;  // INTRA2 at TX_16X16, INTRA1 below
    if (!b[i].plane && b[i].code_txtp && b[i].txtp >= ntx) return false;
    if (b[i].tx_class > 2 || (b[i].tx_class && (b[i].plane || b[i].log2n > 3))) return false;
  }
  return true;
}

}  // namespace

extern "C" {

int mt_cdf_layout(mt_cdf_slot_layout* out);

int mt_emit_coeffs_device(const int32_t* d_levels, const mt_coef_block* d_blocks, int32_t n, uint32_t* d_counts,
                          uint32_t* d_offsets, uint32_t* d_tokens, uint8_t* d_res_ctx, void* stream) {
  if (n < 0 || (n > 0 && (!d_levels || !d_blocks || !d_counts || !d_offsets))) return MT_ERR_INVALID_INPUT;
  if (n == 0) return MT_OK;
  EmitArgs a;
  if (mt_cdf_layout(&a.L) != MT_OK) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned grid = (unsigned)((n + 127) / 128);
  if (!d_tokens) {  // count pass and placement
    emit_kernel<false><<<grid, 128, 0, st>>>(d_levels, d_blocks, n, a, d_counts, nullptr, nullptr, nullptr);
    scan_kernel<<<1, 1024, 0, st>>>(d_counts, n, d_offsets);
  } else {
    emit_kernel<true><<<grid, 128, 0, st>>>(d_levels, d_blocks, n, a, nullptr, d_offsets, d_tokens, d_res_ctx);
  }
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_emit_coeffs(const int32_t* levels, size_t nlevels, const mt_coef_block* blocks, int32_t n, uint32_t** tokens,
                   uint32_t* offsets, uint8_t* res_ctx) {
  if (n < 0 || !tokens || !offsets || (n > 0 && (!levels || !blocks))) return MT_ERR_INVALID_INPUT;
  *tokens = nullptr;
  if (!check_blocks_host(blocks, n)) return MT_ERR_INVALID_INPUT;
  for (int32_t i = 0; i < n; ++i)
    if ((size_t)blocks[i].cf_offset + ((size_t)1 << (2 * blocks[i].log2n)) > nlevels) return MT_ERR_INVALID_INPUT;
  if (n == 0) {
    offsets[0] = 0;
    return MT_OK;
  }
  int32_t* d_lv = nullptr;
  mt_coef_block* d_b = nullptr;
  uint32_t *d_cnt = nullptr, *d_off = nullptr, *d_tok = nullptr;
  uint8_t* d_rc = nullptr;
  int rc = MT_ERR_DEVICE;
  uint32_t total = 0;
  if (cudaMalloc(&d_lv, nlevels * sizeof(int32_t)) != cudaSuccess) goto done;
  if (cudaMalloc(&d_b, (size_t)n * sizeof(mt_coef_block)) != cudaSuccess) goto done;
  if (cudaMalloc(&d_cnt, (size_t)n * 4) != cudaSuccess) goto done;
  if (cudaMalloc(&d_off, ((size_t)n + 1) * 4) != cudaSuccess) goto done;
  if (cudaMalloc(&d_rc, (size_t)n) != cudaSuccess) goto done;
  if (cudaMemcpy(d_lv, levels, nlevels * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  if (cudaMemcpy(d_b, blocks, (size_t)n * sizeof(mt_coef_block), cudaMemcpyHostToDevice) != cudaSuccess) goto done;
  if ((rc = mt_emit_coeffs_device(d_lv, d_b, n, d_cnt, d_off, nullptr, nullptr, nullptr)) != MT_OK) goto done;
  rc = MT_ERR_DEVICE;
  if (cudaMemcpy(&total, d_off + n, 4, cudaMemcpyDeviceToHost) != cudaSuccess) goto done;
  if (cudaMalloc(&d_tok, (size_t)(total ? total : 1) * 4) != cudaSuccess) goto done;
  if ((rc = mt_emit_coeffs_device(d_lv, d_b, n, d_cnt, d_off, d_tok, d_rc, nullptr)) != MT_OK) goto done;
  rc = MT_ERR_DEVICE;
  *tokens = (uint32_t*)malloc((size_t)(total ? total : 1) * 4);
  if (!*tokens) {
    rc = MT_ERR_ALLOC;
    goto done;
  }
  if (cudaMemcpy(*tokens, d_tok, (size_t)total * 4, cudaMemcpyDeviceToHost) != cudaSuccess) goto done;
  if (cudaMemcpy(offsets, d_off, ((size_t)n + 1) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) goto done;
  if (res_ctx && cudaMemcpy(res_ctx, d_rc, (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) goto done;
  rc = MT_OK;
done:
  if (rc != MT_OK && *tokens) {
    free(*tokens);
    *tokens = nullptr;
  }
  cudaFree(d_lv);
  cudaFree(d_b);
  cudaFree(d_cnt);
  cudaFree(d_off);
  cudaFree(d_tok);
  cudaFree(d_rc);
  return rc;
}

}  // extern "C"
