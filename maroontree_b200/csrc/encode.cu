// mt_encode_rgb8: an end-to-end AVIF encode on the device with this library's
// kernels and the reference's bitstream, entropy coder and container.
//
// What it decides, and what it does not: the reference's superblock decision
// engine (src/coder/superblock.rs:813 decode_sb and its partition / leaf
// searches) is not restated here.  This encoder codes every 64x64 superblock
// as a full split down to 8x8 blocks; each 8x8 luma block takes the lowest RD
// cost (strict <, first in (mode, type) order) of the 13 intra modes at angle
// delta 0 times the seven 8x8 intra transform types, as priced by the batched
// candidate chain (prediction, forward transform, quantisation and QM,
// trellis, inverse, SATD bridge, coefficient rate); chroma is UV_DC_PRED with
// DCT_DCT (8x8 in 4:4:4, 4x4 in 4:2:0).  Everything after the decisions is the
// reference's: the coefficient coders and block syntax with their contexts,
// the adaptive range coder and tile packer, the shipped loop-filter levels,
// the CDEF strength search with its per-unit cdef_idx replay, the sequence and
// frame headers and the AVIF container.  The result decodes under any AV1
// decoder to the reconstruction this encoder computed.
//
// Schedule: one persistent launch of 4-CTA clusters takes the frame's 8x8
// blocks from a ticket counter in dependency-level order (a block after its
// left, top, top-left and, where its edges use them, top-right and
// bottom-left neighbours inside its tile) and waits on those neighbours'
// done counts with bounded polls.  The 91 luma candidates of a block are
// split over the cluster's CTAs, each evaluated by eight lanes; the cluster
// minimum picks the winner.  Frames code in the spec-minimum uniform tiling
// (one tile up to 64 superblocks wide and 2304 in area), tiles independent.
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/maroontree_b200.h"
#include "av1_tables.h"
#include "chain4.cuh"
#include "chain8.cuh"
#include "coop8.cuh"
#include "pack.h"

namespace mth {
float scaled_trellis_lambda_host(float dc_q, float lambda0);
}

namespace {

namespace cg = cooperative_groups;

constexpr int kCands = 13 * 7;
__constant__ uint8_t kEncTypes[7] = {MT_TX_IDTX,      MT_TX_DCT_DCT,   MT_TX_V_DCT,  MT_TX_H_DCT,
                                     MT_TX_ADST_ADST, MT_TX_ADST_DCT, MT_TX_DCT_ADST};

struct EncArgs {
  const uint16_t* src[3];
  uint16_t* rec[3];
  mt_chain_params py, pc;  // luma / chroma plane parameters
  mt_quant qy, qc;
  float tly, tlc;          // scaled trellis lambdas
  int has_qm_y, has_qm_c;  // a QM row for luma / chroma (level < 15)
  int sub;                 // 0 4:4:4, 2 4:2:0
  int sb_cols;
  int w8, h8;
  int tile_w8, tile_h8;    // the uniform tile size in 8x8 blocks (the last tile may be smaller)
  uint8_t* mode;           // per 8x8 block (frame raster of 8x8 blocks)
  uint8_t* tx;
  int32_t* lv_y;           // 64 per block
  int32_t* lv_u;           // 64 (4:4:4) or 16 (4:2:0) per block
  int32_t* lv_v;
};

// One image of a launch: its arguments, its tables and its per-block done
// counts.
struct JobDesc {
  EncArgs a;
  const mt_coef_costs* cy;
  const mt_coef_costs* cc;
  const uint8_t* qmy;
  const uint8_t* qmc;
  uint32_t* done;
};

// The z-order position of the k-th 8x8 block of a superblock and its
// intra-edge flags down the quadtree (src/coder/superblock.rs:958-987: root
// (top-right 1, bottom-left 0); children TL (1, 1), TR (parent's, 0),
// BL (1, parent's), BR (0, 0)).
__host__ __device__ inline void zorder(int k, int* bx, int* by, bool* thr, bool* lhb) {
  int x = 0, y = 0;
  bool t = true, l = false;
  for (int lvl = 2; lvl >= 0; --lvl) {
    const int c = (k >> (2 * lvl)) & 3;
    const int h = 1 << lvl;
    if (c == 0) {
      t = true;
      l = true;
    } else if (c == 1) {
      x += h;
      l = false;
    } else if (c == 2) {
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
  *thr = t;
  *lhb = l;
}

__device__ __forceinline__ bool is_smooth(int m) { return m == MT_SMOOTH_PRED || m == MT_SMOOTH_V_PRED || m == MT_SMOOTH_H_PRED; }

// The 91 candidates of a block are split over a cluster of kClusterCtas CTAs
// (on as many SMs): CTA r takes candidate indices [23r, 23r + 23) (index =
// mode * 7 + type, the order ties are broken in) and runs them type by type,
// so the four octets of a warp mostly share a transform path.
constexpr int kClusterCtas = 4;
// CTAs of the decision kernel resident per SM (its register budget follows).
#ifndef MT_ENC_CTAS_PER_SM
#define MT_ENC_CTAS_PER_SM 2
#endif
constexpr int kCandPerCta = 23;
constexpr int kLumaThreads = 192;  // 23 octets, rounded up to whole warps
constexpr int kStepThreads = kLumaThreads + 32;

struct CandOrder {
  int8_t t[kClusterCtas][kLumaThreads / 8];  // candidate index per octet, -1 none
};
constexpr CandOrder make_order() {
  CandOrder o{};
  for (int r = 0; r < kClusterCtas; ++r) {
    const int lo = r * kCandPerCta, hi = lo + kCandPerCta < kCands ? lo + kCandPerCta : kCands;
    int k = 0;
    for (int ti = 0; ti < 7; ++ti)
      for (int m = 0; m < 13; ++m)
        if (m * 7 + ti >= lo && m * 7 + ti < hi) o.t[r][k++] = (int8_t)(m * 7 + ti);
    for (; k < kLumaThreads / 8; ++k) o.t[r][k] = -1;
  }
  return o;
}
__constant__ CandOrder kOrder = make_order();

// Everything one CTA keeps in shared memory.
struct StepShared {
  mt_coef_costs cy, cc;
  float qsY[64], qsC[64], lut[64];
  uint8_t qmY[64], qmC[64];
  mtd::CoopTabs tabs;
  int16_t pred[4][64];              // the predictions of this CTA's four modes (angle delta 0)
  int16_t cpred[64];                // the chroma DC prediction (4:4:4)
  uint16_t src[64], csrc[64];       // the block's luma and chroma source samples
  int16_t above[2][17], left[2][16];  // the block's luma / chroma neighbours (mtd::EdgeRead)
  mtd::Edge8 edge[5];                 // the edges of the four luma predictions and the chroma one
  unsigned long long best;
  uint32_t ticket, abort;
  int cur;                            // the image whose tables are staged (-1: none)
  JobDesc job;                        // its descriptor
  mtd::Oct8 oct[kLumaThreads / 8 + 1];  // one per candidate octet, then the chroma plane's
};

__device__ __forceinline__ void luma_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kLumaThreads) : "memory"); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Writes of a winning 8x8 chain: levels, and prediction + inverse residual
// into the reconstruction plane (lane j: row j, and levels [8j, 8j+8)).
__device__ __forceinline__ void put8(const mtd::Oct8& o, const int16_t* pred, int32_t* lv, uint16_t* rec, int stride,
                                     int px, int py, int j) {
#pragma unroll
  for (int i = 0; i < 8; ++i) lv[j * 8 + i] = o.cf[j * 8 + i];
#pragma unroll
  for (int x = 0; x < 8; ++x)
    rec[(size_t)(py + j) * stride + px + x] = (uint16_t)min(max((int)pred[j * 8 + x] + o.rr[j * 8 + x], 0), 255);
}

// A block's neighbours (above run of 17 from (ox - 1, oy - 1), left run of 16
// from (ox - 1, oy)) into shared memory for lanes k in [0, 33), read past L1
// (they were written by other SMs); only the sides inside the block's tile are
// read, and positions outside the plane are clamped (never read by the
// predictor).
__device__ __forceinline__ void stage_edges(const uint16_t* rec, int stride, int fw, int fh, int ox, int oy, bool top,
                                            bool lft, int16_t* above, int16_t* left, int k) {
  if (k < 17) {
    if (top) above[k] = (int16_t)__ldcg(rec + (size_t)(oy - 1) * stride + min(max(ox - 1 + k, 0), fw - 1));
  } else if (k < 33) {
    if (lft) left[k - 17] = (int16_t)__ldcg(rec + (size_t)min(oy + k - 17, fh - 1) * stride + ox - 1);
  }
}

constexpr uint32_t kDonePerBlock = kClusterCtas;  // each CTA of the coding cluster publishes once
constexpr int kMaxPolls = 1 << 20;               // a dependency wait gives up after this many polls

// The 8x8 blocks of the frame in dependency order, coded by persistent
// clusters (one block per cluster at a time).  A cluster takes the next block
// from the ticket counter, waits until the block's left, top, top-left and,
// where its intra edges use them, top-right and bottom-left neighbours are
// published (done[] == kDonePerBlock), stages the neighbours and the source
// block in shared memory, and evaluates the block: in each CTA the luma warps
// run its share of the 91 candidates (the first four octets also build the
// four predictions the share needs), the last warp codes a chroma plane in
// CTAs 2 (U) and 3 (V).  The cluster's winner is the minimum of the CTAs'
// keys (cost, candidate index), read through distributed shared memory; the
// CTA holding it writes it out; then every CTA publishes.  Tickets follow the
// dependency levels, so a block waits only on blocks that running clusters
// took earlier.  A wait that runs out of polls sets *err; once *err is set
// the remaining waits stop and every cluster leaves at its next ticket.
// list[i] = block index | have-top-right (bit 30) | left-has-bottom (bit 31).
__global__ void __cluster_dims__(kClusterCtas, 1, 1) __launch_bounds__(kStepThreads, MT_ENC_CTAS_PER_SM)
    encode_blocks_kernel(const JobDesc* __restrict__ jobs, const uint2* __restrict__ list, int nlist,
                         uint32_t* ticket_ctr, uint32_t* err) {
  __shared__ StepShared S;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  const int t = threadIdx.x;
  if (t < 64) {
    S.lut[t] = mtd::kCoefRateLut[t];
    S.tabs.load(t, 64);
  } else if (t == 64) {
    S.best = ~0ull;
    S.cur = -1;
  }
  __syncthreads();
  const EncArgs& a = S.job.a;
  const int mlo = rank * kCandPerCta / 7;  // first mode of this CTA's share
  const int c = t - kLumaThreads;          // lane of the chroma warp
  const int pl = rank - 2;                 // its plane (CTAs 2 and 3)
  for (;;) {
    if (rank == 0 && t == 0) {
      S.ticket = atomicAdd(ticket_ctr, 1u);
      S.abort = *(volatile uint32_t*)err;
    }
    cluster.sync();
    const uint32_t tk = *cluster.map_shared_rank(&S.ticket, 0);
    const uint32_t ab = *cluster.map_shared_rank(&S.abort, 0);
    if (ab || tk >= (uint32_t)nlist) break;  // the same for every CTA of the cluster
    const uint2 ent = list[tk];
    const int img = (int)ent.y;
    if (img != S.cur) {  // another image: its descriptor, then its cost and QM tables
      const int* gj = reinterpret_cast<const int*>(jobs + img);
      int* sj = reinterpret_cast<int*>(&S.job);
      for (int i = t; i < (int)(sizeof(JobDesc) / 4); i += blockDim.x) sj[i] = gj[i];
      __syncthreads();
      const float* gy = reinterpret_cast<const float*>(S.job.cy);
      const float* gc = reinterpret_cast<const float*>(S.job.cc);
      float* sy = reinterpret_cast<float*>(&S.cy);
      float* sc = reinterpret_cast<float*>(&S.cc);
      for (int i = t; i < (int)(sizeof(mt_coef_costs) / 4); i += blockDim.x) {
        sy[i] = gy[i];
        sc[i] = gc[i];
      }
      if (t < 64) {
        const int w = a.has_qm_y ? S.job.qmy[t] : 32;
        S.qmY[t] = (uint8_t)w;
        S.qsY[t] = mtd::fwd_qm_scale(w);
      } else if (t < 128) {
        const int i = t - 64;
        const int w = (a.has_qm_c && i < (a.sub ? 16 : 64)) ? S.job.qmc[i] : 32;
        S.qmC[i] = (uint8_t)w;
        S.qsC[i] = mtd::fwd_qm_scale(w);
      }
      __syncthreads();
      if (t == 0) S.cur = img;
    }
    uint32_t* const done = S.job.done;
    const int nbx = a.w8 / 8;
    const uint32_t e = ent.x;
    const int b = (int)(e & 0x3fffffffu);
    const int bx = b % nbx, by = b / nbx;
    const int px = bx * 8, py = by * 8;
    const bool thr = (e >> 30) & 1, lhb = (e >> 31) & 1;
    // the block's tile: neighbours outside it are unavailable (AV1 intra edges
    // and contexts stop at tile edges); the predictor works in tile coordinates
    const int tx0 = bx - bx % a.tile_w8, ty0 = by - by % a.tile_h8;
    const int tx1 = min(tx0 + a.tile_w8, nbx), ty1 = min(ty0 + a.tile_h8, a.h8 / 8);
    const bool has_l = bx > tx0, has_t = by > ty0;
    const bool have_tr = thr && has_t && bx + 1 < tx1;
    const bool have_bl = lhb && has_l && by + 1 < ty1;
    const uint8_t flags = (have_tr ? 1 : 0) | (have_bl ? 2 : 0);
    const int rx = px - tx0 * 8, ry = py - ty0 * 8;  // tile-relative position
    if (t < 5) {  // one thread per dependency
      int dep = -1;
      if (t == 0 && has_l) dep = b - 1;
      if (t == 1 && has_t) dep = b - nbx;
      if (t == 2 && has_l && has_t) dep = b - nbx - 1;
      if (t == 3 && have_tr) dep = b - nbx + 1;
      if (t == 4 && have_bl) dep = b + nbx - 1;
      if (dep >= 0) {
        int it = 0;
        while (ld_acquire(done + dep) < kDonePerBlock) {
          if (*(volatile uint32_t*)err) break;
          if (++it > kMaxPolls) {
            atomicExch(err, 1u);
            break;
          }
          __nanosleep(64);
        }
      }
    }
    __syncthreads();
    // the block's neighbours and source samples
    if (t < 33) {
      stage_edges(a.rec[0], a.py.stride, a.w8, a.h8, px, py, has_t, has_l, S.above[0], S.left[0], t);
    } else if (t >= 64 && t < 128) {
      const int i = t - 64;
      S.src[i] = a.src[0][(size_t)(py + (i >> 3)) * a.py.stride + px + (i & 7)];
    } else if (rank >= 2 && c >= 0) {
      const int cx = a.sub ? px / 2 : px, cy = a.sub ? py / 2 : py, n = a.sub ? 4 : 8;
      stage_edges(a.rec[1 + pl], a.pc.stride, a.pc.frame_w, a.pc.frame_h, cx, cy, has_t, has_l, S.above[1],
                  S.left[1], c);
      if (c == 0)
        stage_edges(a.rec[1 + pl], a.pc.stride, a.pc.frame_w, a.pc.frame_h, cx, cy, has_t, has_l, S.above[1],
                    S.left[1], 32);
      if (n == 8)
        for (int i = c; i < 64; i += 32) S.csrc[i] = a.src[1 + pl][(size_t)(cy + i / 8) * a.pc.stride + cx + (i % 8)];
    }
    __syncthreads();
    if (t < kLumaThreads) {
      const mtd::Octet g;
      const int o = t >> 3;
      const bool ft = (has_t && is_smooth(__ldcg(a.mode + b - nbx))) || (has_l && is_smooth(__ldcg(a.mode + b - 1)));
      mt_candidate cd = {};
      cd.px = (uint16_t)rx;
      cd.py = (uint16_t)ry;
      cd.flags = flags | (ft ? 4 : 0);
      const mtd::EdgeRead rd{S.above[0], S.left[0], rx, ry};
      if (o < 4 && mlo + o < 13) {
        cd.mode = (uint8_t)(mlo + o);
        mtd::coop8_predict(rd, a.py, cd, S.pred[o], S.edge[o], g);
      }
      luma_bar();
      const int ci = kOrder.t[rank][o];
      if (ci >= 0) {
        cd.mode = (uint8_t)(ci / 7);
        cd.tx_type = kEncTypes[ci % 7];
        mt_candidate_result r;
        mtd::coop8_tx(S.src, 8, 0, 0, a.py, a.qy, a.tly, a.has_qm_y ? S.qmY : nullptr, S.qsY, S.lut, S.cy, cd,
                      S.pred[cd.mode - mlo], r, S.oct[o], S.tabs, g);
        if (g.j == 0) atomicMin(&S.best, ((unsigned long long)__float_as_uint(r.cost) << 32) | (unsigned)ci);
      }
    } else if (rank >= 2) {  // chroma: UV_DC_PRED with DCT_DCT, U in CTA 2, V in CTA 3
      int32_t* lvc = pl == 0 ? a.lv_u : a.lv_v;
      if (a.sub == 0 && c < 8) {
        const mtd::Octet g;
        mt_candidate cc = {};
        cc.px = (uint16_t)rx;
        cc.py = (uint16_t)ry;
        cc.flags = flags;
        cc.mode = MT_DC_PRED;
        cc.tx_type = MT_TX_DCT_DCT;
        mtd::coop8_predict(mtd::EdgeRead{S.above[1], S.left[1], rx, ry}, a.pc, cc, S.cpred, S.edge[4], g);
        g.sync();
        mt_candidate_result r;
        mtd::Oct8& oc = S.oct[kLumaThreads / 8];
        mtd::coop8_tx(S.csrc, 8, 0, 0, a.pc, a.qc, a.tlc, a.has_qm_c ? S.qmC : nullptr, S.qsC, S.lut, S.cc, cc,
                      S.cpred, r, oc, S.tabs, g);
        put8(oc, S.cpred, lvc + (size_t)b * 64, a.rec[1 + pl], a.pc.stride, px, py, g.j);
      } else if (a.sub != 0 && c == 0) {
        mt_candidate cc = {};
        cc.mode = MT_DC_PRED;
        cc.tx_type = MT_TX_DCT_DCT;
        cc.px = (uint16_t)(rx / 2);
        cc.py = (uint16_t)(ry / 2);
        mt_candidate_result r;
        int32_t st4[mtd::kWork4Words];
        mtd::Work4 w4{st4};
        // the source plane from the tile's origin, so that tile coordinates address it
        const uint16_t* tsrc = a.src[1 + pl] + (size_t)(ty0 * 4) * a.pc.stride + tx0 * 4;
        mtd::chain4_one_rd<false>(tsrc, mtd::EdgeRead{S.above[1], S.left[1], cc.px, cc.py}, a.pc, a.qc, a.tlc,
                                  a.has_qm_c ? S.qmC : nullptr, S.qsC, S.lut, S.cc, cc, r, w4);
        const int16_t* cf = w4.cf();
        const int16_t* pr = w4.pred();
        const int16_t* rr = w4.rr();
        int32_t* lv = lvc + (size_t)b * 16;
        for (int i = 0; i < 16; ++i) lv[i] = cf[i];
        for (int y = 0; y < 4; ++y)
          for (int x = 0; x < 4; ++x)
            a.rec[1 + pl][(size_t)(py / 2 + y) * a.pc.stride + px / 2 + x] =
                (uint16_t)min(max((int)pr[y * 4 + x] + rr[y * 4 + x], 0), 255);
      }
    }
    cluster.sync();  // every CTA's key is final
    unsigned long long w = ~0ull;
    for (int q = 0; q < kClusterCtas; ++q) {
      const unsigned long long k = *cluster.map_shared_rank(&S.best, q);
      w = k < w ? k : w;
    }
    const int wi = (int)(w & 0xffffffffu);
    if (t < kLumaThreads && rank == wi / kCandPerCta && kOrder.t[rank][t >> 3] == wi) {
      const int j = t & 7;
      put8(S.oct[t >> 3], S.pred[wi / 7 - mlo], a.lv_y + (size_t)b * 64, a.rec[0], a.py.stride, px, py, j);
      if (j == 0) {
        a.mode[b] = (uint8_t)(wi / 7);
        a.tx[b] = kEncTypes[wi % 7];
      }
    }
    __syncthreads();  // this CTA's writes of the block are issued
    if (t == 0) {
      __threadfence();
      atomicAdd(done + b, 1u);
    }
    cluster.sync();  // every CTA has read the keys
    if (t == 0) S.best = ~0ull;
  }
  // The last ticket was read from CTA 0's shared memory by the other CTAs:
  // none may leave while such a read can still be in flight.
  cluster.sync();
}

// One plane of 8-bit samples into the coder's padded u16 plane, edge samples
// replicated past the displayed size (pad_to_mult8_u16, src/dispatch.rs:113-131).
__global__ void pad_plane_kernel(const uint8_t* __restrict__ in, int w, int h, uint16_t* __restrict__ out, int pw,
                                 int ph) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= pw || y >= ph) return;
  out[(size_t)y * pw + x] = in[(size_t)min(y, h - 1) * w + min(x, w - 1)];
}

// The coefficient context byte each transform block leaves for its
// neighbours (src/coeffs.rs eob_and_cul): min(sum of |levels| up to the end
// of block, 63) | the DC sign bits, 0x40 when all levels are zero; the sum
// runs in the block's coding order (the 2-D scan, or the 1-D classes' row /
// column order).  res[3 b + p] for 8x8 block b and plane p.
__global__ void res_ctx_kernel(const int32_t* __restrict__ lv_y, const int32_t* __restrict__ lv_u,
                               const int32_t* __restrict__ lv_v, const uint8_t* __restrict__ tx, int nb, int sub,
                               uint8_t* __restrict__ res) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nb) return;
  const int b = i / 3, p = i % 3;
  const int n = (p == 0 || sub == 0) ? 8 : 4, cl = sub ? 16 : 64;
  const int32_t* cf = p == 0 ? lv_y + (size_t)b * 64 : (p == 1 ? lv_u : lv_v) + (size_t)b * cl;
  const int cls = p == 0 ? (tx[b] == MT_TX_V_DCT ? 1 : (tx[b] == MT_TX_H_DCT ? 2 : 0)) : 0;
  auto at = [&](int k) -> int {
    if (cls == 1) return ((k & (n - 1)) * n) + k / n;  // vertical class order
    if (cls == 2) return k;
    return n == 4 ? mtd::kScan4[k] : mtd::kScan8[k];
  };
  int eob = -1;
  for (int k = 0; k < n * n; ++k)
    if (cf[at(k)]) eob = k;
  if (eob < 0) {
    res[i] = 0x40;
    return;
  }
  uint32_t cul = 0;
  for (int k = 0; k <= eob; ++k) cul += (uint32_t)abs(cf[at(k)]);
  const uint8_t dcb = cf[0] == 0 ? 0x40 : (cf[0] < 0 ? 0 : 0x80);
  res[i] = (uint8_t)((cul < 63 ? cul : 63) | dcb);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side.

namespace {

const int kIntraModeCtx[13] = {0, 1, 2, 3, 4, 4, 4, 4, 3, 0, 1, 2, 0};  // src/intrapred.rs:1088

struct BlockSyntax {
  const mt_cdf_slot_layout& L;
  int w8, h8, sub, nbx;
  const uint8_t* mode;
  const uint8_t* tx;
  std::vector<uint8_t> a_part, l_part, a_skip, l_skip, a_mode, l_mode;
  std::vector<int8_t> a_tx, l_tx;
  std::vector<uint8_t> a_coef[3], l_coef[3];
  const uint8_t* res_ctx;  // per coefficient block, in coding order: (Y, U, V) per 8x8 block
  std::vector<mt_coef_block>* blocks;
  std::vector<std::vector<uint32_t>> sbs;  // tokens with coefficient placeholders
  std::vector<int32_t> cdef_points;

  static constexpr uint32_t kCoef = 0xFFFFFFFFu;  // placeholder: next coefficient block's tokens
  std::vector<uint32_t>* out;

  void tok(int32_t slot, uint32_t s) { out->push_back(((uint32_t)slot << 8) | s); }
  int part_ctx(int bl, int x8, int y8) const {
    const int sh = 4 - bl;
    return ((a_part[x8] >> sh) & 1) + (((l_part[y8] >> sh) & 1) << 1);
  }

  void block8(int x8, int y8, int* cdef_point) {
    const int px = x8 * 8, py = y8 * 8, bx4 = px / 4, by4 = py / 4;
    const int b = y8 * nbx + x8;
    const int m = mode[b], t = tx[b];
    tok(L.skip + a_skip[bx4] + l_skip[by4], 0);
    if (*cdef_point < 0) *cdef_point = (int)out->size();  // read_cdef() follows the SB's first coded skip flag
    a_skip[bx4] = a_skip[bx4 + 1] = 0;
    l_skip[by4] = l_skip[by4 + 1] = 0;
    tok(L.kf_y + kIntraModeCtx[a_mode[bx4]] * 5 + kIntraModeCtx[l_mode[by4]], (uint32_t)m);
    if (m >= MT_V_PRED && m <= MT_D67_PRED) tok(L.angle_delta + m - MT_V_PRED, 3);  // delta 0
    tok(L.uv_mode + 13 + m, MT_DC_PRED);  // CfL allowed at 8x8
    if (m == MT_DC_PRED) tok(L.palette_y_mode + 0, 0);
    tok(L.palette_uv_mode + 0, 0);
    if (m == MT_DC_PRED) tok(L.filter_intra + 3, 0);  // BLOCK_8X8
    tok(L.txsz + 0 * 3 + (l_tx[by4] >= 1) + (a_tx[bx4] >= 1), 0);
    a_tx[bx4] = a_tx[bx4 + 1] = 1;
    l_tx[by4] = l_tx[by4 + 1] = 1;
    // residual: Y (TX_8X8), then U and V (TX_8X8 in 4:4:4, TX_4X4 in 4:2:0)
    for (int p = 0; p < 3; ++p) {
      const int u = (p == 0 || sub == 0) ? 2 : 1;  // 4x4 units the transform spans
      const int cx = (p == 0 || sub == 0) ? bx4 : bx4 / 2, cy = (p == 0 || sub == 0) ? by4 : by4 / 2;
      std::vector<uint8_t>& A = a_coef[p];
      std::vector<uint8_t>& Ll = l_coef[p];
      int s = -2 * u, anz = 0, lnz = 0;
      for (int k = 0; k < u; ++k) {
        s += (A[cx + k] >> 6) + (Ll[cy + k] >> 6);
        anz |= A[cx + k] != 0x40;
        lnz |= Ll[cy + k] != 0x40;
      }
      mt_coef_block cb = {};
      cb.log2n = u == 2 ? 3 : 2;
      cb.plane = p ? 1 : 0;
      cb.skip_ctx = (uint8_t)(p == 0 ? 0 : 7 + anz + lnz);
      cb.dcs_ctx = (uint8_t)((s != 0) + (s > 0));
      cb.y_mode = (uint8_t)m;
      cb.txtp = (uint8_t)(p == 0 ? t : MT_TX_DCT_DCT);
      cb.code_txtp = p == 0;
      cb.tx_class = (uint8_t)(p == 0 && t == MT_TX_V_DCT ? 1 : (p == 0 && t == MT_TX_H_DCT ? 2 : 0));
      blocks->push_back(cb);
      out->push_back(kCoef);
    }
    a_mode[bx4] = a_mode[bx4 + 1] = (uint8_t)m;
    l_mode[by4] = l_mode[by4 + 1] = (uint8_t)m;
  }

  // clear_above_context at a tile's start for its 8x8 columns [x0, x1), and
  // clear_left_context at each superblock row of a tile for rows [y0, y1):
  // the values of an unavailable neighbour.
  void clear_above(int x0, int x1) {
    for (int x = x0; x < x1; ++x) a_part[x] = 0;
    for (int x = 2 * x0; x < 2 * x1; ++x) {
      a_skip[x] = a_mode[x] = 0;
      a_tx[x] = -1;
    }
    for (int p = 0; p < 3; ++p) {
      const int k = (p == 0 || sub == 0) ? 2 : 1;
      for (int x = k * x0; x < k * x1; ++x) a_coef[p][x] = 0x40;
    }
  }
  void clear_left(int y0, int y1) {
    for (int y = y0; y < y1; ++y) l_part[y] = 0;
    for (int y = 2 * y0; y < 2 * y1; ++y) {
      l_skip[y] = l_mode[y] = 0;
      l_tx[y] = -1;
    }
    for (int p = 0; p < 3; ++p) {
      const int k = (p == 0 || sub == 0) ? 2 : 1;
      for (int y = k * y0; y < k * y1; ++y) l_coef[p][y] = 0x40;
    }
  }

  // After a block's coefficient contexts are known: its res_ctx bytes.
  void commit_res(int x8, int y8, const uint8_t r[3]) {
    const int bx4 = x8 * 2, by4 = y8 * 2;
    for (int p = 0; p < 3; ++p) {
      const int u = (p == 0 || sub == 0) ? 2 : 1;
      const int cx = (p == 0 || sub == 0) ? bx4 : bx4 / 2, cy = (p == 0 || sub == 0) ? by4 : by4 / 2;
      for (int k = 0; k < u; ++k) {
        a_coef[p][cx + k] = r[p];
        l_coef[p][cy + k] = r[p];
      }
    }
  }

  // code_split (src/coder/superblock.rs:950-990) always taking SPLIT, down to
  // 8x8 PARTITION_NONE leaves.
  template <class F>
  void node(int bl, int x8, int y8, int sz8, int* cdef_point, F&& leaf) {
    if (sz8 == 1) {
      tok(L.part_bl8 + part_ctx(4, x8, y8), 0);
      leaf(x8, y8);
      a_part[x8] = 0x1E;
      l_part[y8] = 0x1E;
      return;
    }
    const int hh = sz8 / 2;
    const bool have_h = (x8 + hh) * 8 < w8, have_v = (y8 + hh) * 8 < h8;
    const int32_t slot = L.part_split + (bl - 1) * 4 + part_ctx(bl, x8, y8);
    if (have_h && have_v)
      tok(slot, 3);
    else if (have_h)
      out->push_back((2u << 30) | ((uint32_t)slot << 2) | (1u << 1) | 1u);  // gathered: split, top
    else if (have_v)
      out->push_back((2u << 30) | ((uint32_t)slot << 2) | (1u << 1) | 0u);  // gathered: split, left
    const int cx[4] = {x8, x8 + hh, x8, x8 + hh}, cy[4] = {y8, y8, y8 + hh, y8 + hh};
    for (int c = 0; c < 4; ++c)
      if (cx[c] * 8 < w8 && cy[c] * 8 < h8) node(bl + 1, cx[c], cy[c], hh, cdef_point, leaf);
  }
};

// The device buffers of the images of an encode call.  Each device keeps
// sets of them -- one per image of the largest batch seen, each grown to the
// largest frame it carried, each with a stream -- until
// mt_encode_release_buffers or exit.  A call uses them when no other call on
// that device holds them; otherwise it allocates its own for the call.
constexpr int kSlots = 16;
enum Slot { kRgb, kPlanes, kTables, kDecisions, kLevels, kSched, kEmit, kTokens, kMaps, kDeblock, kFiltered, kSkip8,
            kCdef, kRes, kList, kJobs };
struct BufSet {
  void* p[kSlots] = {};
  size_t cap[kSlots] = {};
  cudaStream_t st = nullptr;
};
struct Arena {
  std::mutex mu;
  std::vector<BufSet> sets;
};
Arena g_arenas[16];

class Buffers {
 public:
  explicit Buffers(int n) : own_((size_t)n) {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 16 && g_arenas[dev].mu.try_lock()) {
      ar_ = &g_arenas[dev];
      if ((int)ar_->sets.size() < n) ar_->sets.resize((size_t)n);
    }
  }
  ~Buffers() {
    if (ar_) ar_->mu.unlock();
    for (BufSet& b : own_) {
      for (void* q : b.p) cudaFree(q);
      if (b.st) cudaStreamDestroy(b.st);
    }
  }
  template <class T>
  T* get(int i, Slot s, size_t n) {
    BufSet& b = set(i);
    n = n ? n : 1;
    if (b.cap[s] < n) {
      cudaFree(b.p[s]);
      b.p[s] = nullptr;
      b.cap[s] = 0;
      if (cudaMalloc(&b.p[s], n) != cudaSuccess) return nullptr;
      b.cap[s] = n;
    }
    return reinterpret_cast<T*>(b.p[s]);
  }
  cudaStream_t stream(int i) {
    BufSet& b = set(i);
    if (!b.st && cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking) != cudaSuccess) b.st = nullptr;
    return b.st;
  }

 private:
  BufSet& set(int i) { return ar_ ? ar_->sets[(size_t)i] : own_[(size_t)i]; }
  Arena* ar_ = nullptr;
  std::vector<BufSet> own_;
};

// The stats of one call: copies, launches and CUDA-event times (the events
// exist only when the caller asked for stats).
struct CallStats {
  mt_encode_stats* s;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // call start, blocks start, blocks end, call end
  explicit CallStats(mt_encode_stats* st) : s(st) {
    if (!s) return;
    memset(s, 0, sizeof(*s));
    for (auto& e : ev) cudaEventCreate(&e);
  }
  ~CallStats() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  }
  void h2d(size_t n) {
    if (s) s->h2d_bytes += n;
  }
  void d2h(size_t n) {
    if (s) s->d2h_bytes += n;
  }
  void launches(int n) {
    if (s) s->kernel_launches += (uint32_t)n;
  }
  void mark(int k, cudaStream_t st) {
    if (s) cudaEventRecord(ev[k], st);
  }
  void finish() {
    if (!s) return;
    cudaEventSynchronize(ev[3]);
    cudaEventElapsedTime(&s->blocks_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&s->call_ms, ev[0], ev[3]);
  }
};


// One image of an encode call, through its three phases.
struct Job {
  // the call's inputs
  const uint8_t* rgb = nullptr;
  bool rgb_on_device = false;
  const uint8_t* const* yuv = nullptr;
  uint32_t width = 0, height = 0;
  const mt_encode_config* cfg = nullptr;
  uint8_t** out = nullptr;
  size_t* out_len = nullptr;
  uint16_t** recon_out = nullptr;
  mt_encode_stats* stats = nullptr;
  // the frame
  mt_encode_plan plan = {};
  int sub = 0, sx = 0, nbx = 0, nby = 0, nb = 0, sb_cols = 0, sb_rows = 0, cl = 0;
  int32_t tcl = 0, trl = 0;      // TileColsLog2, TileRowsLog2
  int tile_sb_w = 0, tile_sb_h = 0;  // the uniform tile size in superblocks
  int32_t pw = 0, ph = 0, pcw = 0, pch = 0;
  size_t ny = 0, nc = 0;
  EncArgs a = {};
  JobDesc desc = {};
  uint16_t* src[3] = {};
  uint16_t* rec[3] = {};
  uint8_t* d_res = nullptr;
  std::vector<uint32_t> sched;  // blocks in dependency-level order
  std::vector<int> lstart;      // first entry of each level
  cudaStream_t st = nullptr;
  std::unique_ptr<CallStats> cs;
  int rc = MT_OK;
};

}  // namespace

namespace mth {
void cdef_frame_transfer_bytes(const mt_cdef_params* p, size_t* d2h, size_t* h2d);
extern thread_local int cdef_last_launches;
extern thread_local int deblock_last_launches;
}  // namespace mth

extern "C" {
int mt_coef_costs_build(const mt_coef_cdfs* cdfs, mt_coef_costs* out);
const uint8_t* mt_qm_row(int32_t qm_level, int32_t chroma, int32_t w, int32_t h);
int mt_emit_coeffs_device(const int32_t* d_levels, const mt_coef_block* d_blocks, int32_t n, uint32_t* d_counts,
                          uint32_t* d_offsets, uint32_t* d_tokens, uint8_t* d_res_ctx, void* stream);
}

namespace {

// Validation, device buffers, the input on the device (colour conversion or
// padding), the frame laws' tables, the kernel arguments and the dependency
// schedule of image i.
int job_setup(Job& j, Buffers& buf, int i) {
  if (!j.out || !j.out_len) return MT_ERR_INVALID_INPUT;
  *j.out = nullptr;
  *j.out_len = 0;
  int rc = mt_encode_config_validate(j.cfg);
  if (rc != MT_OK) return rc;
  const mt_encode_config* cfg = j.cfg;
  const uint32_t width = j.width, height = j.height;
  rc = mt_validate_rgb8_input(width, height, (size_t)width * height * 3);
  if (rc != MT_OK) return rc;
  if (!j.rgb && (!j.yuv || !j.yuv[0] || !j.yuv[1] || !j.yuv[2])) return MT_ERR_INVALID_INPUT;
  if (cfg->chroma != MT_CHROMA_420 && cfg->chroma != MT_CHROMA_444) return MT_ERR_UNSUPPORTED_CHROMA_FORMAT;
  if ((rc = mt_encode_config_effective(cfg, &j.plan)) != MT_OK) return rc;
  if (j.plan.base_q_idx == 0) return MT_ERR_UNSUPPORTED;  // lossless is a separate encoder
  const int sub = j.sub = cfg->chroma == MT_CHROMA_420 ? 2 : 0;
  const int sx = j.sx = sub ? 1 : 0;
  if ((rc = mt_padded_plane_dims((int)width, (int)height, sub, &j.pw, &j.ph, &j.pcw, &j.pch)) != MT_OK) return rc;
  const int32_t pw = j.pw, ph = j.ph, pcw = j.pcw, pch = j.pch;
  const int nbx = j.nbx = pw / 8, nby = j.nby = ph / 8, nb = j.nb = nbx * nby;
  const int sb_cols = j.sb_cols = (pw + 63) / 64, sb_rows = j.sb_rows = (ph + 63) / 64;
  // the spec-minimum uniform tiling (src/coder/frame_encode.rs:75-80): one
  // tile unless the frame exceeds the AV1 maximum tile width (64 superblocks)
  // or area (2304 superblocks)
  if ((rc = mt_tiling_spec_min(pw, ph, &j.tcl, &j.trl)) != MT_OK) return rc;
  j.tile_sb_w = (sb_cols + (1 << j.tcl) - 1) >> j.tcl;
  j.tile_sb_h = (sb_rows + (1 << j.trl) - 1) >> j.trl;
  const int cl = j.cl = sub ? 16 : 64;  // chroma levels per block
  // quantisers, QM rows, default CDF slices and their bit costs, lambdas
  mt_quant qy, qc;
  if (mt_quant_init(j.plan.base_q_idx, 8, j.plan.qm_y, &qy) != MT_OK) return MT_ERR_INVALID_INPUT;
  if (mt_quant_init_chroma(j.plan.base_q_idx, 0, 0, 8, j.plan.qm_u, &qc) != MT_OK) return MT_ERR_INVALID_INPUT;
  mt_coef_cdfs cdy, cdc;
  mt_coef_costs cy, cc;
  const int qctx = mt_qcat(j.plan.base_q_idx);
  mt_coef_cdfs_default(qctx, 8, 8, 0, &cdy);
  mt_coef_cdfs_default(qctx, sub ? 4 : 8, sub ? 4 : 8, 1, &cdc);
  mt_coef_costs_build(&cdy, &cy);
  mt_coef_costs_build(&cdc, &cc);
  mt_rd_lambdas lam;
  if (mt_rd_lambdas_init(j.plan.base_q_idx, qy.dc_q, sub, 8, &lam) != MT_OK) return MT_ERR_INVALID_INPUT;
  const uint8_t* qmy = mt_qm_row(j.plan.qm_y, 0, 8, 8);
  const uint8_t* qmc = mt_qm_row(j.plan.qm_u, 1, sub ? 4 : 8, sub ? 4 : 8);
  // device buffers
  const size_t ny = j.ny = (size_t)pw * ph, nc = j.nc = (size_t)pcw * pch;
  const size_t in_bytes = j.rgb ? (size_t)width * height * 3
                                : (size_t)width * height + 2 * (size_t)((width + sx) >> sx) * ((height + sx) >> sx);
  uint8_t* d_rgbbuf = buf.get<uint8_t>(i, kRgb, j.rgb_on_device ? 1 : in_bytes);
  uint16_t* d_planes = buf.get<uint16_t>(i, kPlanes, (ny + 2 * nc) * 2 * 2);
  uint8_t* d_tabs = buf.get<uint8_t>(i, kTables, 2 * sizeof(mt_coef_costs) + 128);
  uint8_t* d_decs = buf.get<uint8_t>(i, kDecisions, (size_t)nb * 2);
  int32_t* d_levels = buf.get<int32_t>(i, kLevels, (size_t)nb * (64 + 2 * cl) * 4);
  j.d_res = buf.get<uint8_t>(i, kRes, (size_t)nb * 3);
  uint32_t* d_done = buf.get<uint32_t>(i, kSched, (size_t)nb * 4);
  const cudaStream_t st = j.st = buf.stream(i);
  if (!d_rgbbuf || !d_planes || !d_tabs || !d_decs || !d_levels || !j.d_res || !d_done || !st) return MT_ERR_DEVICE;
  uint16_t* const* src = j.src;
  for (int p = 0; p < 3; ++p) {
    j.src[p] = d_planes + (p == 0 ? 0 : ny + (size_t)(p - 1) * nc);
    j.rec[p] = d_planes + ny + 2 * nc + (p == 0 ? 0 : ny + (size_t)(p - 1) * nc);
  }
  mt_coef_costs* d_cy = reinterpret_cast<mt_coef_costs*>(d_tabs);
  mt_coef_costs* d_cc = d_cy + 1;
  uint8_t* d_qmy = reinterpret_cast<uint8_t*>(d_cc + 1);
  uint8_t* d_qmc = d_qmy + 64;
  j.cs.reset(new CallStats(j.stats));
  CallStats& cs = *j.cs;
  cs.mark(0, st);
  if (j.rgb) {
    const uint8_t* d_in = j.rgb;
    if (!j.rgb_on_device) {
      if (cudaMemcpyAsync(d_rgbbuf, j.rgb, in_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return MT_ERR_DEVICE;
      cs.h2d(in_bytes);
      d_in = d_rgbbuf;
    }
    if ((rc = mt_csc_rgb8_device(d_in, (int)width, (int)height, sub, src[0], src[1], src[2], st)) != MT_OK) return rc;
    cs.launches(2);
  } else {
    const int cw = (int)((width + sx) >> sx), ch = (int)((height + sx) >> sx);
    uint8_t* d_in = d_rgbbuf;
    const size_t n0 = (size_t)width * height, n1 = (size_t)cw * ch;
    if (cudaMemcpyAsync(d_in, j.yuv[0], n0, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_in + n0, j.yuv[1], n1, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(d_in + n0 + n1, j.yuv[2], n1, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return MT_ERR_DEVICE;
    pad_plane_kernel<<<dim3((pw + 127) / 128, ph), 128, 0, st>>>(d_in, (int)width, (int)height, src[0], pw, ph);
    pad_plane_kernel<<<dim3((pcw + 127) / 128, pch), 128, 0, st>>>(d_in + n0, cw, ch, src[1], pcw, pch);
    pad_plane_kernel<<<dim3((pcw + 127) / 128, pch), 128, 0, st>>>(d_in + n0 + n1, cw, ch, src[2], pcw, pch);
    cs.h2d(n0 + 2 * n1);
    cs.launches(3);
  }
  cudaMemsetAsync(d_tabs, 32, 2 * sizeof(mt_coef_costs) + 128, st);  // flat QM weights past a 4x4 row
  cudaMemcpyAsync(d_cy, &cy, sizeof(cy), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_cc, &cc, sizeof(cc), cudaMemcpyHostToDevice, st);
  if (qmy) cudaMemcpyAsync(d_qmy, qmy, 64, cudaMemcpyHostToDevice, st);
  if (qmc) cudaMemcpyAsync(d_qmc, qmc, sub ? 16 : 64, cudaMemcpyHostToDevice, st);
  cs.h2d(2 * sizeof(mt_coef_costs) + (qmy ? 64 : 0) + (qmc ? (sub ? 16 : 64) : 0));
  EncArgs& a = j.a;
  a = EncArgs{};
  for (int p = 0; p < 3; ++p) {
    a.src[p] = j.src[p];
    a.rec[p] = j.rec[p];
  }
  a.py = {};
  a.py.tx_size = 8;
  a.py.bd = 8;
  a.py.frame_w = pw;
  a.py.frame_h = ph;
  a.py.stride = pw;
  a.py.trellis_lambda0 = lam.trellis_lambda0;
  a.py.mode_lambda = lam.mode_lambda;
  a.py.satd_scale = lam.satd_scale;
  a.py.satd_bridge = lam.satd_bridge;
  a.pc = a.py;
  a.pc.tx_size = sub ? 4 : 8;
  a.pc.frame_w = pcw;
  a.pc.frame_h = pch;
  a.pc.stride = pcw;
  a.qy = qy;
  a.qc = qc;
  a.tly = mth::scaled_trellis_lambda_host((float)qy.dc_q, lam.trellis_lambda0);
  a.tlc = mth::scaled_trellis_lambda_host((float)qc.dc_q, lam.trellis_lambda0);
  a.has_qm_y = qmy != nullptr;
  a.has_qm_c = qmc != nullptr;
  a.sub = sub;
  a.sb_cols = sb_cols;
  a.w8 = pw;
  a.h8 = ph;
  a.tile_w8 = j.tile_sb_w * 8;
  a.tile_h8 = j.tile_sb_h * 8;
  a.mode = d_decs;
  a.tx = a.mode + nb;
  a.lv_y = d_levels;
  a.lv_u = a.lv_y + (size_t)nb * 64;
  a.lv_v = a.lv_u + (size_t)nb * cl;
  j.desc.a = a;
  j.desc.cy = d_cy;
  j.desc.cc = d_cc;
  j.desc.qmy = d_qmy;
  j.desc.qmc = d_qmc;
  j.desc.done = d_done;
  if (cudaMemsetAsync(a.mode, 0, (size_t)nb * 2, st) != cudaSuccess ||
      cudaMemsetAsync(d_done, 0, (size_t)nb * 4, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  // Dependency levels of the 8x8 blocks: a block needs its left, top,
  // top-left neighbours and, where the intra edge uses them, its top-right and
  // bottom-left ones, all inside its tile (tiles are independent).
  std::vector<int32_t> T((size_t)nb, -1);
  std::vector<uint32_t> entry((size_t)nb);
  std::vector<int> cnt;
  for (int sr = 0; sr < sb_rows; ++sr)
    for (int sc = 0; sc < sb_cols; ++sc)
      for (int k = 0; k < 64; ++k) {
        int bx, by;
        bool thr, lhb;
        zorder(k, &bx, &by, &thr, &lhb);
        const int x = sc * 8 + bx, y = sr * 8 + by;
        if (x >= nbx || y >= nby) continue;
        const int tx0 = x - x % a.tile_w8, ty0 = y - y % a.tile_h8;
        const int tx1 = std::min(tx0 + a.tile_w8, nbx), ty1 = std::min(ty0 + a.tile_h8, nby);
        const bool has_l = x > tx0, has_t = y > ty0;
        const bool tr = thr && has_t && x + 1 < tx1;
        const bool bl = lhb && has_l && y + 1 < ty1;
        int lv = 0;
        auto dep = [&](int xx, int yy) { lv = std::max(lv, T[(size_t)yy * nbx + xx] + 1); };
        if (has_l) dep(x - 1, y);
        if (has_t) dep(x, y - 1);
        if (has_l && has_t) dep(x - 1, y - 1);
        if (tr) dep(x + 1, y - 1);
        if (bl) dep(x - 1, y + 1);
        const size_t bi = (size_t)y * nbx + x;
        T[bi] = lv;
        entry[bi] = (uint32_t)bi | (thr ? 1u << 30 : 0u) | (lhb ? 1u << 31 : 0u);
        if ((int)cnt.size() <= lv) cnt.resize(lv + 1, 0);
        ++cnt[lv];
      }
  j.lstart.assign(cnt.size() + 1, 0);
  for (size_t l = 0; l < cnt.size(); ++l) j.lstart[l + 1] = j.lstart[l] + cnt[l];
  j.sched.resize((size_t)nb);
  std::vector<int> fill(j.lstart.begin(), j.lstart.end() - 1);
  for (int sr = 0; sr < sb_rows; ++sr)  // coding order inside a level
    for (int sc = 0; sc < sb_cols; ++sc)
      for (int k = 0; k < 64; ++k) {
        int bx, by;
        bool thr, lhb;
        zorder(k, &bx, &by, &thr, &lhb);
        const int x = sc * 8 + bx, y = sr * 8 + by;
        if (x >= nbx || y >= nby) continue;
        const size_t bi = (size_t)y * nbx + x;
        j.sched[fill[T[bi]]++] = entry[bi];
      }
  if (j.stats) {
    j.stats->blocks = (uint32_t)nb;
    j.stats->levels = (uint32_t)(j.lstart.size() - 1);
  }
  return MT_OK;
}

// The decisions of every image that set up, in one launch: the images'
// blocks merged level by level into one ticket list (each image's order is
// still a dependency order), the persistent clusters taking tickets across
// images.
int decide_all(std::vector<Job>& jobs, Buffers& buf) {
  std::vector<uint2> list;
  std::vector<JobDesc> descs;
  std::vector<int> slot;  // job index per descriptor
  int levels = 0;
  for (size_t i = 0; i < jobs.size(); ++i)
    if (jobs[i].rc == MT_OK) {
      slot.push_back((int)i);
      descs.push_back(jobs[i].desc);
      levels = std::max(levels, (int)jobs[i].lstart.size() - 1);
    }
  if (slot.empty()) return MT_OK;
  int width_max = 1;
  for (int l = 0; l < levels; ++l) {
    const size_t before = list.size();
    for (size_t d = 0; d < slot.size(); ++d) {
      const Job& j = jobs[(size_t)slot[d]];
      if (l + 1 >= (int)j.lstart.size()) continue;
      for (int k = j.lstart[l]; k < j.lstart[l + 1]; ++k) list.push_back(make_uint2(j.sched[(size_t)k], (unsigned)d));
    }
    width_max = std::max(width_max, (int)(list.size() - before));
  }
  const int i0 = slot[0];
  const cudaStream_t ks = jobs[(size_t)i0].st;
  uint2* d_list = buf.get<uint2>(i0, kList, list.size() * sizeof(uint2) + 16);
  JobDesc* d_jobs = buf.get<JobDesc>(i0, kJobs, descs.size() * sizeof(JobDesc));
  if (!d_list || !d_jobs) return MT_ERR_DEVICE;
  uint32_t* d_ctl = reinterpret_cast<uint32_t*>(d_list + list.size());  // [0] ticket counter, [1] timeout flag
  // the launch waits for every image's set-up on its own stream
  std::vector<cudaEvent_t> evs;
  for (size_t d = 1; d < slot.size(); ++d) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MT_ERR_DEVICE;
    evs.push_back(e);
    cudaEventRecord(e, jobs[(size_t)slot[d]].st);
    cudaStreamWaitEvent(ks, e, 0);
  }
  if (cudaMemcpyAsync(d_list, list.data(), list.size() * sizeof(uint2), cudaMemcpyHostToDevice, ks) != cudaSuccess ||
      cudaMemcpyAsync(d_jobs, descs.data(), descs.size() * sizeof(JobDesc), cudaMemcpyHostToDevice, ks) !=
          cudaSuccess ||
      cudaMemsetAsync(d_ctl, 0, 8, ks) != cudaSuccess)
    return MT_ERR_DEVICE;
  // one cluster per block that can run at once (the widest merged level), at
  // most as many as the SMs hold
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
    return MT_ERR_DEVICE;
  const int nclusters = std::max(1, std::min(width_max, sms * MT_ENC_CTAS_PER_SM / kClusterCtas));
  for (int d : slot) {
    jobs[(size_t)d].cs->h2d(jobs[(size_t)d].sched.size() * 8 + sizeof(JobDesc));
    jobs[(size_t)d].cs->mark(1, ks);
  }
  encode_blocks_kernel<<<nclusters * kClusterCtas, kStepThreads, 0, ks>>>(d_jobs, d_list, (int)list.size(), d_ctl,
                                                                          d_ctl + 1);
  for (int d : slot) {
    jobs[(size_t)d].cs->mark(2, ks);
    jobs[(size_t)d].cs->launches(1);
    jobs[(size_t)d].cs->d2h(4);
  }
  // every image's finishing work waits for the launch
  cudaEvent_t done_ev;
  if (cudaEventCreateWithFlags(&done_ev, cudaEventDisableTiming) != cudaSuccess) return MT_ERR_DEVICE;
  evs.push_back(done_ev);
  cudaEventRecord(done_ev, ks);
  for (int d : slot) cudaStreamWaitEvent(jobs[(size_t)d].st, done_ev, 0);
  uint32_t timed_out = 0;
  const bool ok = cudaMemcpyAsync(&timed_out, d_ctl + 1, 4, cudaMemcpyDeviceToHost, ks) == cudaSuccess &&
                  cudaStreamSynchronize(ks) == cudaSuccess && cudaGetLastError() == cudaSuccess;
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  if (!ok || timed_out) return MT_ERR_DEVICE;
  return MT_OK;
}

// Everything after the decisions for image i: the context bytes, the block
// syntax walk, the coefficient tokens, the filters, range coding, headers
// and container.
// A CUDA event destroyed with its scope.
struct EventGuard {
  cudaEvent_t e = nullptr;
  ~EventGuard() {
    if (e) cudaEventDestroy(e);
  }
};

// Host threads joined when their scope ends, on every return path.
struct ThreadGroup {
  std::vector<std::thread> v;
  ~ThreadGroup() { join(); }
  void join() {
    for (std::thread& w : v)
      if (w.joinable()) w.join();
    v.clear();
  }
};

int job_finish(Job& j, Buffers& buf, int i) {
  int rc = MT_OK;
  const cudaStream_t st = j.st;
  CallStats& cs = *j.cs;
  const mt_encode_config* cfg = j.cfg;
  const uint32_t width = j.width, height = j.height;
  const int sub = j.sub, sx = j.sx, nbx = j.nbx, nby = j.nby, nb = j.nb, sb_cols = j.sb_cols, sb_rows = j.sb_rows,
            cl = j.cl;
  const int32_t pw = j.pw, ph = j.ph;
  const size_t ny = j.ny, nc = j.nc;
  const EncArgs& a = j.a;
  uint16_t* const* src = j.src;
  uint16_t* const* rec = j.rec;
  std::vector<uint8_t> mode(nb), tx(nb);
  // The coefficient contexts of a block depend on its neighbours' context
  // bytes, which depend on their levels only: computed on the device for
  // every transform block, read back as three bytes per 8x8 block.
  res_ctx_kernel<<<(unsigned)((3 * (size_t)nb + 255) / 256), 256, 0, st>>>(a.lv_y, a.lv_u, a.lv_v, a.tx, nb, sub,
                                                                           j.d_res);
  cs.launches(1);
  std::vector<uint8_t> resb((size_t)nb * 3);
  if (cudaMemcpyAsync(mode.data(), a.mode, nb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(tx.data(), a.tx, nb, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(resb.data(), j.d_res, resb.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MT_ERR_DEVICE;
  cs.d2h(2 * (size_t)nb + resb.size());
  // block syntax in coding order, with the coefficient blocks it carries
  mt_cdf_slot_layout L;
  mt_cdf_layout(&L);
  std::vector<mt_coef_block> blocks;
  blocks.reserve((size_t)nb * 3);
  BlockSyntax bs{L, pw, ph, sub, nbx, mode.data(), tx.data()};
  bs.a_part.assign(nbx, 0);
  bs.l_part.assign(nby, 0);
  bs.a_skip.assign(nbx * 2, 0);
  bs.l_skip.assign(nby * 2, 0);
  bs.a_mode.assign(nbx * 2, 0);
  bs.l_mode.assign(nby * 2, 0);
  bs.a_tx.assign(nbx * 2, -1);
  bs.l_tx.assign(nby * 2, -1);
  for (int p = 0; p < 3; ++p) {
    bs.a_coef[p].assign(nbx * 2, 0x40);
    bs.l_coef[p].assign(nby * 2, 0x40);
  }
  bs.blocks = &blocks;
  // tiles in raster order, superblocks in raster order inside each tile
  // (decode_tile: the above context cleared per tile, the left per SB row)
  std::vector<int> tile_first;  // first coded superblock of each tile
  std::vector<int> sb_unit;     // frame-raster 64x64 unit of each coded superblock
  std::vector<size_t> sb_coef_first;  // first coefficient block of each coded superblock
  for (int r0 = 0; r0 < sb_rows; r0 += j.tile_sb_h)
    for (int c0 = 0; c0 < sb_cols; c0 += j.tile_sb_w) {
      const int r1 = std::min(r0 + j.tile_sb_h, sb_rows), c1 = std::min(c0 + j.tile_sb_w, sb_cols);
      tile_first.push_back((int)bs.sbs.size());
      bs.clear_above(c0 * 8, std::min(c1 * 8, nbx));
      for (int sr = r0; sr < r1; ++sr) {
        bs.clear_left(sr * 8, std::min(sr * 8 + 8, nby));
        for (int sc = c0; sc < c1; ++sc) {
          bs.sbs.emplace_back();
          bs.out = &bs.sbs.back();
          sb_coef_first.push_back(blocks.size());
          sb_unit.push_back(sr * sb_cols + sc);
          int cp = -1;
          bs.node(1, sc * 8, sr * 8, 8, &cp, [&](int x8, int y8) {
            const size_t first = blocks.size();
            bs.block8(x8, y8, &cp);
            const int b = y8 * nbx + x8;
            const uint32_t off[3] = {(uint32_t)((size_t)b * 64), (uint32_t)((size_t)nb * 64 + (size_t)b * cl),
                                     (uint32_t)((size_t)nb * (64 + cl) + (size_t)b * cl)};
            for (int p = 0; p < 3; ++p) blocks[first + p].cf_offset = off[p];
            bs.commit_res(x8, y8, &resb[(size_t)b * 3]);
          });
          bs.cdef_points.push_back(cp);
        }
      }
    }
  tile_first.push_back((int)bs.sbs.size());
  sb_coef_first.push_back(blocks.size());
  // coefficient tokens of every block in one launch
  const int ncb = (int)blocks.size();
  mt_coef_block* d_blocks = buf.get<mt_coef_block>(i, kEmit, (size_t)ncb * (sizeof(mt_coef_block) + 8) + 8);
  if (!d_blocks) return MT_ERR_DEVICE;
  uint32_t* d_cnt = reinterpret_cast<uint32_t*>(d_blocks + ncb);
  uint32_t* d_off = d_cnt + ncb;
  if (cudaMemcpyAsync(d_blocks, blocks.data(), (size_t)ncb * sizeof(mt_coef_block), cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return MT_ERR_DEVICE;
  if ((rc = mt_emit_coeffs_device(a.lv_y, d_blocks, ncb, d_cnt, d_off, nullptr, nullptr, st)) != MT_OK) return rc;
  cs.h2d((size_t)ncb * sizeof(mt_coef_block));
  cs.launches(2);
  uint32_t total = 0;
  if (cudaMemcpyAsync(&total, d_off + ncb, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MT_ERR_DEVICE;
  uint32_t* d_tok = buf.get<uint32_t>(i, kTokens, (size_t)total * 4);
  if (!d_tok) return MT_ERR_DEVICE;
  if ((rc = mt_emit_coeffs_device(a.lv_y, d_blocks, ncb, d_cnt, d_off, d_tok, nullptr, st)) != MT_OK) return rc;
  cs.launches(1);
  std::vector<uint32_t> toks(total), offs((size_t)ncb + 1);
  if (cudaMemcpyAsync(toks.data(), d_tok, (size_t)total * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(offs.data(), d_off, offs.size() * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  // the tokens are on the host once this event has passed; the filters
  // carry on behind it on the stream
  EventGuard tok_ev;
  if (cudaEventCreateWithFlags(&tok_ev.e, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(tok_ev.e, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  // deblocking (uniform 8x8 blocks and transforms) and the CDEF decision,
  // enqueued before the host splices the tokens
  int32_t ly, luv, sharp;
  mt_loop_filter_levels(j.plan.base_q_idx, sx, sx, &ly, &luv, &sharp);
  const int n4 = (pw / 4) * (ph / 4);
  std::vector<uint8_t> maps((size_t)n4 * 6);
  for (int r = 0; r < ph / 4; ++r)
    for (int c = 0; c < pw / 4; ++c) {
      const size_t k = (size_t)r * (pw / 4) + c;
      maps[k] = 2;
      maps[n4 + k] = 2;
      maps[2 * (size_t)n4 + k] = (c % 2) == 0;
      maps[3 * (size_t)n4 + k] = (r % 2) == 0;
      maps[4 * (size_t)n4 + k] = 2;
      maps[5 * (size_t)n4 + k] = 2;
    }
  mt_deblock_frame_params g = {};
  g.w8 = pw;
  g.h8 = ph;
  g.disp_w = (int)width;
  g.disp_h = (int)height;
  g.sub_x = g.sub_y = sx;
  g.bd = 8;
  const size_t dbs = mt_deblock_frame_scratch_bytes(&g);
  uint8_t* d_maps = buf.get<uint8_t>(i, kMaps, maps.size());
  void* d_db = buf.get<void>(i, kDeblock, dbs);
  if (!d_maps || !d_db) return MT_ERR_DEVICE;
  if (cudaMemcpyAsync(d_maps, maps.data(), maps.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  cs.h2d(maps.size());
  // the recon planes are kept: the filters write planes of their own
  uint16_t* d_flt = buf.get<uint16_t>(i, kFiltered, (ny + 2 * nc) * 2);
  if (!d_flt) return MT_ERR_DEVICE;
  uint16_t* flt[3] = {d_flt, d_flt + ny, d_flt + ny + nc};
  const uint8_t* m0 = d_maps;
  if ((rc = mt_deblock_frame_device_to(rec[0], rec[1], rec[2], flt[0], flt[1], flt[2], m0, m0 + n4,
                                       m0 + 2 * (size_t)n4, m0 + 3 * (size_t)n4, m0 + 4 * (size_t)n4,
                                       m0 + 5 * (size_t)n4, &g, ly, luv, luv, d_db, st)) != MT_OK)
    return rc;
  cs.launches(mth::deblock_last_launches);
  // phase 1 of the range coding (each token's store, with the CDF
  // adaptation), one host thread per tile, reading the superblocks' syntax
  // tokens and the coefficient blocks in place while the filters run
  if (cudaEventSynchronize(tok_ev.e) != cudaSuccess) return MT_ERR_DEVICE;
  cs.d2h(4 + (size_t)total * 4 + offs.size() * 4);
  const int ntiles = (int)tile_first.size() - 1;
  std::vector<std::unique_ptr<mth::TileStores>> stores((size_t)ntiles);
  size_t nstores = 0;
  for (int t = 0; t < ntiles; ++t) {
    const int f = tile_first[(size_t)t], l = tile_first[(size_t)t + 1];
    const size_t k0 = sb_coef_first[(size_t)f], k1 = sb_coef_first[(size_t)l];
    size_t n = (size_t)offs[k1] - offs[k0];
    for (int sb = f; sb < l; ++sb) n += bs.sbs[(size_t)sb].size();
    n -= k1 - k0;  // the placeholders
    auto ts = std::make_unique<mth::TileStores>();
    ts->st.resize(n);
    ts->sb_end.assign((size_t)(l - f), 0);
    ts->cdef_at.assign((size_t)(l - f), UINT32_MAX);
    stores[(size_t)t] = std::move(ts);
    nstores += n;
  }
  ThreadGroup tracers;  // joined on every return path
  for (int t = 0; t < ntiles; ++t) {
    const int f = tile_first[(size_t)t];
    for (int part = 0; part < mth::kTracers; ++part)
      tracers.v.emplace_back(mth::trace_tile_stores, j.plan.base_q_idx, cfg->updating_cdf, &bs.sbs[(size_t)f],
                             tile_first[(size_t)t + 1] - f, bs.cdef_points.data() + f, toks.data(), offs.data(),
                             sb_coef_first[(size_t)f], stores[(size_t)t].get(), part);
  }
  mt_cdef_params cp = {};
  cp.w8 = pw;
  cp.h8 = ph;
  cp.disp_w = (int)width;
  cp.disp_h = (int)height;
  cp.sub_x = cp.sub_y = sx;
  cp.base_q_idx = j.plan.base_q_idx;
  cp.bd = 8;
  cp.slow = cfg->speed <= MT_SPEED_SLOW;
  const int unit_cols = (pw + 63) / 64, unit_rows = (ph + 63) / 64;
  uint8_t* d_skip8 = buf.get<uint8_t>(i, kSkip8, (size_t)nb);
  void* d_cs = buf.get<void>(i, kCdef, mt_cdef_scratch_bytes(&cp));
  if (!d_skip8 || !d_cs) return MT_ERR_DEVICE;
  if (cudaMemsetAsync(d_skip8, 0, (size_t)nb, st) != cudaSuccess) return MT_ERR_DEVICE;
  mt_cdef_decision dec = {};
  std::vector<uint8_t> grid((size_t)unit_cols * unit_rows);
  if (j.plan.cdef) {
    if ((rc = mt_cdef_frame_device(flt[0], flt[1], flt[2], src[0], src[1], src[2], d_skip8, &cp, d_cs, &dec,
                                   grid.data(), st)) != MT_OK)
      return rc;
    size_t cd2h = 0, ch2d = 0;
    mth::cdef_frame_transfer_bytes(&cp, &cd2h, &ch2d);
    cs.launches(mth::cdef_last_launches);
    cs.d2h(cd2h);
    if (mth::cdef_last_launches == 3) cs.h2d(ch2d);
  } else {
    dec.bits = -1;
  }
  if (j.recon_out) {  // the decoder's output: deblocked and CDEF-filtered
    if (cudaMemcpyAsync(j.recon_out[0], flt[0], ny * 2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(j.recon_out[1], flt[1], nc * 2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(j.recon_out[2], flt[2], nc * 2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return MT_ERR_DEVICE;
    cs.d2h((ny + 2 * nc) * 2);
  }
  // phase 2: each tile's coder over its stores, following phase 1, with each
  // superblock's cdef_idx (its 64x64 unit's) at its read_cdef() point; tiles
  // are coded independently, on threads of their own when there are several
  std::vector<uint8_t> sb_idx(sb_unit.size());
  for (size_t k2 = 0; k2 < sb_unit.size(); ++k2) sb_idx[k2] = grid[(size_t)sb_unit[k2]];
  std::vector<uint8_t*> tiles((size_t)ntiles, nullptr);
  std::vector<size_t> tile_lens((size_t)ntiles, 0);
  std::vector<int> tile_rc((size_t)ntiles, MT_OK);
  auto code = [&](int t) {
    const int f = tile_first[(size_t)t], n = tile_first[(size_t)t + 1] - f;
    tile_rc[(size_t)t] = mth::code_tile_stores(stores[(size_t)t].get(), n, cfg->updating_cdf,
                                               dec.bits > 0 ? sb_idx.data() + f : nullptr, dec.bits > 0 ? dec.bits : 0,
                                               &tiles[(size_t)t], &tile_lens[(size_t)t]);
  };
  if (ntiles == 1) {
    code(0);
  } else {
    ThreadGroup coders;
    for (int t = 0; t < ntiles; ++t) coders.v.emplace_back(code, t);
    coders.join();
  }
  tracers.join();
  auto free_tiles = [&]() {
    for (uint8_t* t : tiles) free(t);
  };
  for (int r2 : tile_rc)
    if (r2 != MT_OK) {
      free_tiles();
      return r2;
    }
  // headers and container
  mt_sequence_header_params sp = {};
  sp.width = width;
  sp.height = height;
  sp.profile = sub ? 0 : 1;
  sp.bit_depth = 8;
  sp.color_present = cfg->color_present;
  sp.primaries = cfg->primaries;
  sp.transfer = cfg->transfer;
  sp.matrix = cfg->matrix;
  sp.full_range = cfg->full_range;
  sp.chroma_sample_position = cfg->chroma_sample_position;
  sp.ss_x = sp.ss_y = (uint32_t)sx;
  sp.enable_filter_intra = sp.enable_intra_edge_filter = 1;
  mt_frame_header_params fp = {};
  fp.w8 = pw;
  fp.h8 = ph;
  fp.base_q_idx = j.plan.base_q_idx;
  fp.qm_y = j.plan.qm_y;
  fp.qm_u = fp.qm_v = j.plan.qm_u;
  fp.updating_cdf = cfg->updating_cdf;
  fp.lf_y = ly;
  fp.lf_u = fp.lf_v = luv;
  fp.lf_sharpness = sharp;
  fp.cdef_bits = dec.bits;
  fp.cdef_damping = dec.bits >= 0 ? dec.damping : 3;
  for (int e = 0; e < dec.n_strengths && e < 8; ++e)
    for (int q = 0; q < 4; ++q) fp.cdef_strengths[e][q] = dec.strengths[e][q];
  fp.tile_cols_log2 = j.tcl;
  fp.tile_rows_log2 = j.trl;
  std::vector<const uint8_t*> ctiles(tiles.begin(), tiles.end());
  uint8_t* obu = nullptr;
  size_t obu_len = 0;
  rc = mt_av1_stream(&sp, &fp, ctiles.data(), tile_lens.data(), ntiles, &obu, &obu_len);
  free_tiles();
  if (rc != MT_OK) return rc;
  mt_avif_item_params ip = {};
  ip.width = width;
  ip.height = height;
  ip.bit_depth = 8;
  ip.channels = 3;
  ip.seq_profile = (uint8_t)sp.profile;
  ip.seq_level_idx = mt_av1_level_for(width, height);
  ip.chroma_sub_x = ip.chroma_sub_y = sx;
  ip.color_present = cfg->color_present;
  ip.primaries = (uint16_t)cfg->primaries;
  ip.transfer = (uint16_t)cfg->transfer;
  ip.matrix = (uint16_t)cfg->matrix;
  ip.full_range = cfg->full_range;
  ip.icc = cfg->icc;
  ip.icc_len = cfg->icc_len;
  ip.exif = cfg->exif;
  ip.exif_len = cfg->exif_len;
  ip.imir_axis = -1;
  ip.clli_present = cfg->clli_present;
  ip.max_content_light_level = cfg->max_content_light_level;
  ip.max_pic_average_light_level = cfg->max_pic_average_light_level;
  rc = mt_wrap_av1_image(obu, obu_len, &ip, j.out, j.out_len);
  free(obu);
  if (j.stats) j.stats->tokens = (uint32_t)nstores;
  cs.mark(3, st);
  cs.finish();
  return rc;
}

// The encode of a batch of images: set-up per image, one launch for all
// their decisions, then each image's finishing work on a host thread of its
// own (the calling thread for one image).  Every image's bytes are those of
// encoding it alone.
void encode_jobs(std::vector<Job>& jobs) {
  const int n = (int)jobs.size();
  Buffers buf(n);
  for (int i = 0; i < n; ++i) jobs[(size_t)i].rc = job_setup(jobs[(size_t)i], buf, i);
  const int rc = decide_all(jobs, buf);
  for (Job& j : jobs)
    if (j.rc == MT_OK && rc != MT_OK) j.rc = rc;
  if (n == 1) {
    if (jobs[0].rc == MT_OK) jobs[0].rc = job_finish(jobs[0], buf, 0);
    return;
  }
  std::vector<std::thread> pool;
  for (int i = 0; i < n; ++i)
    if (jobs[(size_t)i].rc == MT_OK)
      pool.emplace_back([&jobs, &buf, i]() { jobs[(size_t)i].rc = job_finish(jobs[(size_t)i], buf, i); });
  for (std::thread& t : pool) t.join();
}

int encode_one(const uint8_t* rgb, bool rgb_on_device, const uint8_t* const* yuv, uint32_t width, uint32_t height,
               const mt_encode_config* cfg, uint8_t** out, size_t* out_len, uint16_t* recon_out[3],
               mt_encode_stats* stats) {
  std::vector<Job> jobs(1);
  Job& j = jobs[0];
  j.rgb = rgb;
  j.rgb_on_device = rgb_on_device;
  j.yuv = yuv;
  j.width = width;
  j.height = height;
  j.cfg = cfg;
  j.out = out;
  j.out_len = out_len;
  j.recon_out = recon_out;
  j.stats = stats;
  encode_jobs(jobs);
  return j.rc;
}

}  // namespace

extern "C" {

int mt_encode_rgb8_ex(const uint8_t* rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg,
                      uint8_t** out, size_t* out_len, uint16_t* recon_out[3], mt_encode_stats* stats) {
  if (!rgb) return MT_ERR_INVALID_INPUT;
  return encode_one(rgb, false, nullptr, width, height, cfg, out, out_len, recon_out, stats);
}

int mt_encode_rgb8(const uint8_t* rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg, uint8_t** out,
                   size_t* out_len) {
  return mt_encode_rgb8_ex(rgb, width, height, cfg, out, out_len, nullptr, nullptr);
}

int mt_encode_rgb8_device(const uint8_t* d_rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg,
                          uint8_t** out, size_t* out_len, mt_encode_stats* stats) {
  if (!d_rgb) return MT_ERR_INVALID_INPUT;
  return encode_one(d_rgb, true, nullptr, width, height, cfg, out, out_len, nullptr, stats);
}

int mt_encode_rgb8_batch(int32_t n, const uint8_t* const* rgb, const uint32_t* widths, const uint32_t* heights,
                         const mt_encode_config* cfgs, uint8_t** outs, size_t* out_lens, int32_t* rcs,
                         mt_encode_stats* stats) {
  if (n < 1 || n > 64 || !rgb || !widths || !heights || !cfgs || !outs || !out_lens) return MT_ERR_INVALID_INPUT;
  std::vector<Job> jobs((size_t)n);
  for (int i = 0; i < n; ++i) {
    Job& j = jobs[(size_t)i];
    outs[i] = nullptr;
    out_lens[i] = 0;
    j.rgb = rgb[i];
    j.width = widths[i];
    j.height = heights[i];
    j.cfg = &cfgs[i];
    j.out = &outs[i];
    j.out_len = &out_lens[i];
    j.stats = stats ? &stats[i] : nullptr;
    if (!rgb[i]) j.rc = MT_ERR_INVALID_INPUT;
  }
  std::vector<Job> live;  // images with an input: the others keep their code
  std::vector<int> idx;
  for (int i = 0; i < n; ++i)
    if (jobs[(size_t)i].rgb) {
      idx.push_back(i);
      live.push_back(std::move(jobs[(size_t)i]));
    }
  encode_jobs(live);
  int first = MT_OK;
  for (size_t k = 0; k < live.size(); ++k) jobs[(size_t)idx[k]].rc = live[k].rc;
  for (int i = 0; i < n; ++i) {
    if (rcs) rcs[i] = jobs[(size_t)i].rc;
    if (first == MT_OK && jobs[(size_t)i].rc != MT_OK) first = jobs[(size_t)i].rc;
  }
  return first;
}

void mt_encode_release_buffers(void) {
  int cur = 0;
  cudaGetDevice(&cur);
  for (int d = 0; d < 16; ++d) {
    Arena& ar = g_arenas[d];
    std::lock_guard<std::mutex> lock(ar.mu);
    if (ar.sets.empty()) continue;
    cudaSetDevice(d);
    for (BufSet& b : ar.sets) {
      for (void*& q : b.p) {
        cudaFree(q);
        q = nullptr;
      }
      if (b.st) cudaStreamDestroy(b.st);
    }
    ar.sets.clear();
  }
  cudaSetDevice(cur);
}

int mt_encode_yuv8(const uint8_t* y, const uint8_t* u, const uint8_t* v, uint32_t width, uint32_t height,
                   const mt_encode_config* cfg, uint8_t** out, size_t* out_len, uint16_t* recon_out[3]) {
  const uint8_t* planes[3] = {y, u, v};
  if (!y || !u || !v) return MT_ERR_INVALID_INPUT;
  return encode_one(nullptr, false, planes, width, height, cfg, out, out_len, recon_out, nullptr);
}

}  // extern "C"
