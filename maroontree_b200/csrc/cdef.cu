// Frame CDEF (src/coder/frame_cdef.rs:49-520 and src/cdef.rs).
//
// Device side, per frame:
//   cdef_dir_kernel      one thread per luma 8x8: the spec direction search
//                        (src/cdef.rs:89-178), plus the per-64x64-unit
//                        directional-variance sums of the non-skip blocks that
//                        the strength search gates on.
//   cdef_tab_kernel      one 64-thread CTA per (plane, luma 8x8): all 12
//                        (pri, sec) candidates of the block at once -- every tap
//                        is read and constrained once per strength, as the
//                        reference's fused candidate routine does
//                        (src/cdef.rs:651-800) -- then the decision distortion of
//                        each: the weighted SSE in the AVX2 lane order
//                        (src/avx/rd.rs:767-848) for whole blocks, plain SSE for
//                        blocks the visible window cuts; summed per unit with
//                        64-bit integer atomics (order-free).
//   cdef_apply_kernel    one 64-thread CTA per (plane, luma 8x8): the chosen
//                        strengths filtered from a pre-CDEF snapshot into the
//                        reconstruction (src/coder/frame_cdef.rs:960-1125).
// Host side: the staged strength search over the unit tables
// (src/coder/frame_cdef.rs:116-520), a few hundred kilobytes of integers.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "../../include/maroontree_b200.h"

namespace {

constexpr int kVeryLarge = 0x4000;  // the spec's out-of-frame tap value
constexpr int kNCand = 12;

// Cdef_Directions (row, col) per direction and tap distance.
__constant__ int8_t cDirs[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}},
};
__constant__ int8_t cUvDir422[8] = {7, 0, 2, 4, 5, 6, 6, 6};

// Weighted-SSE 4x4 DCT basis and weights (src/rd_sse.rs:1400-1430).
constexpr float kRawMean = 0.4625f;
__constant__ float cD[4][4] = {{0.5f, 0.5f, 0.5f, 0.5f},
                               {0.6532815f, 0.27059805f, -0.27059805f, -0.6532815f},
                               {0.5f, -0.5f, -0.5f, 0.5f},
                               {0.27059805f, -0.6532815f, 0.6532815f, -0.27059805f}};
__constant__ float cW[4][4] = {
    {1.8f / kRawMean, 1.0f / kRawMean, 0.4f / kRawMean, 0.2f / kRawMean},
    {1.0f / kRawMean, 0.8f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
    {0.4f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
    {0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean, 0.2f / kRawMean},
};

__host__ __device__ __forceinline__ int log2_floor(int v) {
#ifdef __CUDA_ARCH__
  return v <= 0 ? 0 : 31 - __clz(v);
#else
  return v <= 0 ? 0 : 31 - __builtin_clz((unsigned)v);
#endif
}

// adjust_pri (src/cdef.rs:181-189): primary strength scaled by the block variance.
__host__ __device__ __forceinline__ int adjust_pri(int pri, int var) {
  if (var == 0) return 0;
  const int vs = var >> 6;
  const int l = vs != 0 ? min(log2_floor(vs), 12) : 0;
  return (pri * (4 + l) + 8) >> 4;
}

__device__ __forceinline__ int strength_shift(int s, int damping) {
  return s == 0 ? 0 : max(damping - log2_floor(s), 0);
}

__device__ __forceinline__ int constrain(int diff, int strength, int shift) {
  const int a = abs(diff);
  const int c = min(max(strength - (a >> shift), 0), a);
  return diff < 0 ? -c : c;
}

struct Geo {
  int w8, h8, cw8, ch8, nbx, nby, uc, ur;
  int disp_w, disp_h, cw_vis, ch_vis;
  int sub_x, sub_y, bd, damping;
};

// ---------------------------------------------------------------------------
// Direction search: one thread per luma 8x8.
__global__ void __launch_bounds__(128) cdef_dir_kernel(const uint16_t* __restrict__ py, Geo g,
                                                       const uint8_t* __restrict__ skip8, uint8_t* __restrict__ dirs,
                                                       int32_t* __restrict__ vars,
                                                       unsigned long long* __restrict__ dv_sum,
                                                       int* __restrict__ dv_cnt) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= g.nbx * g.nby) return;
  const int bx = b % g.nbx, by = b / g.nbx;
  const int x = bx * 8, y = by * 8;
  const int cs = g.bd - 8;
  int part[8][15];
#pragma unroll
  for (int d = 0; d < 8; d++)
#pragma unroll
    for (int k = 0; k < 15; k++) part[d][k] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int yy = min(y + i, g.h8 - 1);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int xx = min(x + j, g.w8 - 1);
      const int p = (py[(size_t)yy * g.w8 + xx] >> cs) - 128;
      part[0][i + j] += p;
      part[1][i + j / 2] += p;
      part[2][i] += p;
      part[3][3 + i - j / 2] += p;
      part[4][7 + i - j] += p;
      part[5][3 - i / 2 + j] += p;
      part[6][j] += p;
      part[7][i / 2 + j] += p;
    }
  }
  long long cost[8];
#pragma unroll
  for (int d = 0; d < 8; d++) cost[d] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    cost[2] += (long long)part[2][i] * part[2][i];
    cost[6] += (long long)part[6][i] * part[6][i];
  }
  cost[2] *= 105;
  cost[6] *= 105;
  const long long kDiv[8] = {0, 840, 420, 280, 210, 168, 140, 120};
#pragma unroll
  for (int i = 0; i < 7; i++) {
    cost[0] += ((long long)part[0][i] * part[0][i] + (long long)part[0][14 - i] * part[0][14 - i]) * kDiv[i + 1];
    cost[4] += ((long long)part[4][i] * part[4][i] + (long long)part[4][14 - i] * part[4][14 - i]) * kDiv[i + 1];
  }
  cost[0] += (long long)part[0][7] * part[0][7] * 105;
  cost[4] += (long long)part[4][7] * part[4][7] * 105;
#pragma unroll
  for (int s = 1; s < 8; s += 2) {
#pragma unroll
    for (int i = 0; i < 5; i++) cost[s] += (long long)part[s][3 + i] * part[s][3 + i] * 105;
#pragma unroll
    for (int i = 0; i < 3; i++)
      cost[s] += ((long long)part[s][i] * part[s][i] + (long long)part[s][10 - i] * part[s][10 - i]) * kDiv[2 * i + 2];
  }
  int best_dir = 0;
  long long best = cost[0];
#pragma unroll
  for (int d = 1; d < 8; d++)
    if (cost[d] > best) {
      best = cost[d];
      best_dir = d;
    }
  long long opp = cost[0];
#pragma unroll
  for (int d = 0; d < 8; d++)
    if (d == ((best_dir + 4) & 7)) opp = cost[d];
  const int var = (int)((best - opp) >> 10);
  dirs[b] = (uint8_t)best_dir;
  vars[b] = var;
  if (dv_sum && !skip8[b]) {
    const int u = (by >> 3) * g.uc + (bx >> 3);
    atomicAdd(&dv_sum[u], (unsigned long long)(long long)var);
    atomicAdd(&dv_cnt[u], 1);
  }
}

// ---------------------------------------------------------------------------
// The 12 candidate outputs of one sample (src/cdef.rs:651-800 semantics).
struct BlockCtx {
  const uint16_t* plane;
  int stride, rows;
  int dir, damping, bd;
  int pri_eff[3];  // effective primary strength of pri 1, 2, 4 (0 = off)
};

__device__ __forceinline__ int tap_at(const BlockCtx& b, int cx, int cy) {
  if (cx < 0 || cy < 0 || cx >= b.stride || cy >= b.rows) return kVeryLarge;
  return b.plane[(size_t)cy * b.stride + cx];
}

__device__ __forceinline__ void sample_candidates(const BlockCtx& b, int cx, int cy, int out[kNCand]) {
  const int cs = b.bd - 8;
  const int damp = max(b.damping, 1);
  const int c = b.plane[(size_t)cy * b.stride + cx];
  int pshift[3], pw0[3], pw1[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    pshift[q] = strength_shift(b.pri_eff[q], damp);
    const int odd = (b.pri_eff[q] >> cs) & 1;
    pw0[q] = odd ? 3 : 4;
    pw1[q] = odd ? 3 : 2;
  }
  const int sec_eff0 = 1 << cs, sec_eff1 = 2 << cs;
  const int sshift0 = strength_shift(sec_eff0, damp), sshift1 = strength_shift(sec_eff1, damp);
  int psum[3] = {0, 0, 0}, ssum[2] = {0, 0}, ssum0[2] = {0, 0};
  int mn = c, mx = c;
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int pdr = cDirs[b.dir][k][0], pdc = cDirs[b.dir][k][1];
#pragma unroll
    for (int sg = 1; sg >= -1; sg -= 2) {
      const int tp = tap_at(b, cx + sg * pdc, cy + sg * pdr);
      if (tp != kVeryLarge) {
        const int d = tp - c;
#pragma unroll
        for (int q = 0; q < 3; q++)
          if (b.pri_eff[q] != 0) psum[q] += (k == 0 ? pw0[q] : pw1[q]) * constrain(d, b.pri_eff[q], pshift[q]);
        mn = min(mn, tp);
        mx = max(mx, tp);
      }
    }
    const int sw = k == 0 ? 2 : 1;
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
      const int sdir = pass == 0 ? b.dir : 0;
      if (pass == 1 && b.dir == 0) break;
#pragma unroll
      for (int doff = 2; doff <= 6; doff += 4) {
        const int sd = (sdir + doff) & 7;
        const int sdr = cDirs[sd][k][0], sdc = cDirs[sd][k][1];
#pragma unroll
        for (int sg = 1; sg >= -1; sg -= 2) {
          const int tp = tap_at(b, cx + sg * sdc, cy + sg * sdr);
          if (tp != kVeryLarge) {
            const int d = tp - c;
            const int a0 = sw * constrain(d, sec_eff0, sshift0), a1 = sw * constrain(d, sec_eff1, sshift1);
            if (pass == 0) {
              ssum[0] += a0;
              ssum[1] += a1;
              mn = min(mn, tp);
              mx = max(mx, tp);
            } else {
              ssum0[0] += a0;
              ssum0[1] += a1;
            }
          }
        }
      }
    }
  }
  if (b.dir == 0) {
    ssum0[0] = ssum[0];
    ssum0[1] = ssum[1];
  }
  const int maxv = (1 << b.bd) - 1;
#pragma unroll
  for (int si = 0; si < 3; si++)
#pragma unroll
    for (int pi = 0; pi < 4; pi++) {
      const bool en_p = pi != 0 && b.pri_eff[pi - 1] != 0, en_s = si != 0;
      int sum;
      if (pi == 0)
        sum = en_s ? ssum0[si - 1] : 0;
      else
        sum = (en_p ? psum[pi - 1] : 0) + (en_s ? ssum[si - 1] : 0);
      int v = c + ((8 + sum - (sum < 0)) >> 4);
      if (en_p && en_s) v = min(max(v, mn), mx);
      out[si * 4 + pi] = min(max(v, 0), maxv);
    }
}

// Weighted SSE of a w x h error block (w, h in {4, 8}) for 12 candidates at
// once, in the AVX2 kernel's float order.  err: [12][64] (row pitch w);
// part: [12][32] scratch.  Called by all 64 threads of the CTA.
__device__ __forceinline__ void wsse12(const int* err, int w, int h, float* part, float* res) {
  const int t = threadIdx.x;
  if (t < 4 * kNCand) {
    const int cand = t >> 2;
    const int* e = err + cand * 64;
    if (w == 8) {
      // Thread (cand, k): the 8 lane accumulators of row accumulator k.
      const int k = t & 3;
      float acc[8];
#pragma unroll
      for (int ln = 0; ln < 8; ln++) acc[ln] = 0.0f;
      for (int r0 = 0; r0 < h; r0 += 4) {
        float tt[8];
#pragma unroll
        for (int ln = 0; ln < 8; ln++) {
          float v = __fmul_rn((float)e[(r0 + 0) * 8 + ln], cD[k][0]);
          v = __fmaf_rn((float)e[(r0 + 1) * 8 + ln], cD[k][1], v);
          v = __fmaf_rn((float)e[(r0 + 2) * 8 + ln], cD[k][2], v);
          v = __fmaf_rn((float)e[(r0 + 3) * 8 + ln], cD[k][3], v);
          tt[ln] = v;
        }
#pragma unroll
        for (int ln = 0; ln < 8; ln++) {
          const int hb = ln & 4, l = ln & 3;
          float cc = __fmul_rn(cD[l][0], tt[hb + 0]);
          cc = __fmaf_rn(cD[l][1], tt[hb + 1], cc);
          cc = __fmaf_rn(cD[l][2], tt[hb + 2], cc);
          cc = __fmaf_rn(cD[l][3], tt[hb + 3], cc);
          acc[ln] = __fmaf_rn(__fmul_rn(cW[k][l], cc), cc, acc[ln]);
        }
      }
#pragma unroll
      for (int ln = 0; ln < 8; ln++) part[cand * 32 + k * 8 + ln] = acc[ln];
    } else {
      // Thread (cand, l): output lane l of the 4-wide tail path.
      const int l = t & 3;
      float s = 0.0f;
      for (int r0 = 0; r0 < h; r0 += 4) {
        float tt[4][4];
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
          for (int j = 0; j < 4; j++) {
            float v = __fmul_rn((float)e[(r0 + 0) * 4 + j], cD[k][0]);
            v = __fmaf_rn((float)e[(r0 + 1) * 4 + j], cD[k][1], v);
            v = __fmaf_rn((float)e[(r0 + 2) * 4 + j], cD[k][2], v);
            v = __fmaf_rn((float)e[(r0 + 3) * 4 + j], cD[k][3], v);
            tt[k][j] = v;
          }
#pragma unroll
        for (int k = 0; k < 4; k++) {
          float cc = __fmul_rn(cD[l][0], tt[k][0]);
          cc = __fmaf_rn(cD[l][1], tt[k][1], cc);
          cc = __fmaf_rn(cD[l][2], tt[k][2], cc);
          cc = __fmaf_rn(cD[l][3], tt[k][3], cc);
          s = __fmaf_rn(__fmul_rn(cW[k][l], cc), cc, s);
        }
      }
      part[cand * 32 + l] = s;
    }
  }
  __syncthreads();
  if (t < kNCand) {
    const float* p = part + t * 32;
    float s[4];
    if (w == 8) {
#pragma unroll
      for (int l = 0; l < 4; l++) {
        const float a = __fadd_rn(__fadd_rn(p[0 * 8 + l], p[0 * 8 + 4 + l]), __fadd_rn(p[1 * 8 + l], p[1 * 8 + 4 + l]));
        const float b2 = __fadd_rn(__fadd_rn(p[2 * 8 + l], p[2 * 8 + 4 + l]), __fadd_rn(p[3 * 8 + l], p[3 * 8 + 4 + l]));
        s[l] = __fadd_rn(a, b2);
      }
    } else {
#pragma unroll
      for (int l = 0; l < 4; l++) s[l] = p[l];
    }
    res[t] = __fadd_rn(__fadd_rn(s[0], s[2]), __fadd_rn(s[1], s[3]));
  }
}

struct TabArgs {
  const uint16_t* rec[3];
  const uint16_t* src[3];
  unsigned long long* tab[3];
};

// One CTA of 64 threads per (luma 8x8 block, plane).  blockIdx.z: 0 luma,
// 1 / 2 chroma U / V.
__global__ void __launch_bounds__(64) cdef_tab_kernel(TabArgs ta, Geo g, const uint8_t* __restrict__ skip8,
                                                      const uint8_t* __restrict__ dirs,
                                                      const int32_t* __restrict__ vars) {
  __shared__ int sErr[kNCand * 64];
  __shared__ float sPart[kNCand * 32];
  __shared__ float sRes[kNCand];
  __shared__ unsigned sSse[2][kNCand];
  const int bx = blockIdx.x, by = blockIdx.y, pl = blockIdx.z;
  const int bi = by * g.nbx + bx;
  if (skip8[bi]) return;
  const bool luma = pl == 0;
  const int sx = luma ? 0 : g.sub_x, sy = luma ? 0 : g.sub_y;
  const int bw = 8 >> sx, bh = 8 >> sy;
  const int x = (bx * 8) >> sx, y = (by * 8) >> sy;
  const int vis_w = luma ? g.disp_w : g.cw_vis, vis_h = luma ? g.disp_h : g.ch_vis;
  if (x >= vis_w || y >= vis_h) return;
  const int cs = g.bd - 8;
  BlockCtx b;
  b.plane = ta.rec[pl];
  b.stride = luma ? g.w8 : g.cw8;
  b.rows = luma ? g.h8 : g.ch8;
  b.bd = g.bd;
  b.damping = luma ? g.damping : g.damping - 1;
  const int d0 = dirs[bi];
  b.dir = luma ? d0 : ((g.sub_x == 1 && g.sub_y == 0) ? (int)cUvDir422[d0] : d0);
  const int var = vars[bi];
  b.pri_eff[0] = luma ? adjust_pri(1 << cs, var) : 1 << cs;
  b.pri_eff[1] = luma ? adjust_pri(2 << cs, var) : 2 << cs;
  b.pri_eff[2] = luma ? adjust_pri(4 << cs, var) : 4 << cs;
  const int vw = min(vis_w - x, bw), vh = min(vis_h - y, bh);
  const bool whole = vw == bw && vh == bh;
  const int t = threadIdx.x;
  const int n = bw * bh;
  const int i = t / bw, j = t % bw;
  int o[kNCand];
  int s = 0;
  if (t < n) {
    sample_candidates(b, x + j, y + i, o);
    s = ta.src[pl][(size_t)(y + i) * b.stride + x + j];
  }
  const int u = (by >> 3) * g.uc + (bx >> 3);
  unsigned long long* tab = ta.tab[pl] + (size_t)u * kNCand;
  if (whole) {
    if (t < n)
#pragma unroll
      for (int c = 0; c < kNCand; c++) sErr[c * 64 + t] = o[c] - s;
    __syncthreads();
    wsse12(sErr, bw, bh, sPart, sRes);
    __syncthreads();
    if (t < kNCand) atomicAdd(&tab[t], (unsigned long long)(long long)roundf(sRes[t]));
  } else {
    const bool vis = t < n && i < vh && j < vw;
#pragma unroll
    for (int c = 0; c < kNCand; c++) {
      const int e = vis ? o[c] - s : 0;
      const unsigned r = __reduce_add_sync(0xffffffffu, (unsigned)(e * e));
      if ((t & 31) == 0) sSse[t >> 5][c] = r;
    }
    __syncthreads();
    if (t < kNCand) atomicAdd(&tab[t], (unsigned long long)sSse[0][t] + sSse[1][t]);
  }
}

// ---------------------------------------------------------------------------
// Apply: one CTA of 64 threads per (luma 8x8 block, plane).  ustr: per unit
// (luma pri, luma sec, chroma pri, chroma sec).
struct ApplyArgs {
  uint16_t* rec[3];
  const uint16_t* snap[3];
};

__global__ void __launch_bounds__(64) cdef_apply_kernel(ApplyArgs aa, Geo g, const uint8_t* __restrict__ skip8,
                                                        const uint8_t* __restrict__ dirs,
                                                        const int32_t* __restrict__ vars,
                                                        const uint8_t* __restrict__ ustr) {
  const int bx = blockIdx.x, by = blockIdx.y, pl = blockIdx.z;
  const int bi = by * g.nbx + bx;
  if (skip8[bi]) return;
  const bool luma = pl == 0;
  const int u = (by >> 3) * g.uc + (bx >> 3);
  const int pri = ustr[u * 4 + (luma ? 0 : 2)], sec = ustr[u * 4 + (luma ? 1 : 3)];
  if (pri == 0 && sec == 0) return;
  const int sx = luma ? 0 : g.sub_x, sy = luma ? 0 : g.sub_y;
  const int bw = 8 >> sx, bh = 8 >> sy;
  const int x = (bx * 8) >> sx, y = (by * 8) >> sy;
  const int stride = luma ? g.w8 : g.cw8, rows = luma ? g.h8 : g.ch8;
  if (x >= stride || y >= rows) return;
  const int t = threadIdx.x;
  if (t >= bw * bh) return;
  const int cx = x + t % bw, cy = y + t / bw;
  if (cx >= stride || cy >= rows) return;
  const int cs = g.bd - 8;
  const int d0 = dirs[bi];
  const int bdir = luma ? d0 : ((g.sub_x == 1 && g.sub_y == 0) ? (int)cUvDir422[d0] : d0);
  const int dir = pri == 0 ? 0 : bdir;
  const int p_str = luma ? adjust_pri(pri << cs, vars[bi]) : pri << cs;
  const int s_str = sec << cs;
  const int damp = max(luma ? g.damping : g.damping - 1, 1);
  const uint16_t* src = aa.snap[pl];
  const int c = src[(size_t)cy * stride + cx];
  const bool en_p = p_str != 0, en_s = s_str != 0, clip = en_p && en_s;
  const int odd = (p_str >> cs) & 1;
  const int pshift = strength_shift(p_str, damp), sshift = strength_shift(s_str, damp);
  int sum = 0, mn = c, mx = c;
  auto tap = [&](int xx, int yy) -> int {
    if (xx < 0 || yy < 0 || xx >= stride || yy >= rows) return kVeryLarge;
    return src[(size_t)yy * stride + xx];
  };
#pragma unroll
  for (int k = 0; k < 2; k++) {
    if (en_p) {
      const int w = k == 0 ? (odd ? 3 : 4) : (odd ? 3 : 2);
#pragma unroll
      for (int sg = 1; sg >= -1; sg -= 2) {
        const int p = tap(cx + sg * cDirs[dir][k][1], cy + sg * cDirs[dir][k][0]);
        if (p != kVeryLarge) {
          sum += w * constrain(p - c, p_str, pshift);
          if (clip) {
            mx = max(mx, p);
            mn = min(mn, p);
          }
        }
      }
    }
    if (en_s) {
      const int w = k == 0 ? 2 : 1;
#pragma unroll
      for (int doff = 2; doff <= 6; doff += 4) {
        const int sd = (dir + doff) & 7;
#pragma unroll
        for (int sg = 1; sg >= -1; sg -= 2) {
          const int p = tap(cx + sg * cDirs[sd][k][1], cy + sg * cDirs[sd][k][0]);
          if (p != kVeryLarge) {
            sum += w * constrain(p - c, s_str, sshift);
            if (clip) {
              mx = max(mx, p);
              mn = min(mn, p);
            }
          }
        }
      }
    }
  }
  int v = c + ((8 + sum - (sum < 0)) >> 4);
  if (clip) v = min(max(v, mn), mx);
  aa.rec[pl][(size_t)cy * stride + cx] = (uint16_t)min(max(v, 0), (1 << g.bd) - 1);
}

// ---------------------------------------------------------------------------
// Host side.

int check_params(const mt_cdef_params* p) {
  if (!p) return MT_ERR_INVALID_INPUT;
  if (p->w8 <= 0 || p->h8 <= 0 || (p->w8 & 7) || (p->h8 & 7) || p->w8 > 16384 || p->h8 > 16384)
    return MT_ERR_INVALID_INPUT;
  if (p->disp_w <= p->w8 - 8 || p->disp_w > p->w8 || p->disp_h <= p->h8 - 8 || p->disp_h > p->h8)
    return MT_ERR_INVALID_INPUT;
  if (p->sub_x < 0 || p->sub_x > 1 || p->sub_y < 0 || p->sub_y > p->sub_x) return MT_ERR_INVALID_INPUT;
  if (p->base_q_idx < 1 || p->base_q_idx > 255) return MT_ERR_INVALID_INPUT;
  if (p->bd != 8) return MT_ERR_UNSUPPORTED;
  return MT_OK;
}

Geo make_geo(const mt_cdef_params* p) {
  Geo g;
  g.w8 = p->w8;
  g.h8 = p->h8;
  g.cw8 = p->w8 >> p->sub_x;
  g.ch8 = p->h8 >> p->sub_y;
  g.nbx = p->w8 / 8;
  g.nby = p->h8 / 8;
  g.uc = (p->w8 + 63) / 64;
  g.ur = (p->h8 + 63) / 64;
  g.disp_w = p->disp_w;
  g.disp_h = p->disp_h;
  g.cw_vis = (p->disp_w + (1 << p->sub_x) - 1) >> p->sub_x;
  g.ch_vis = (p->disp_h + (1 << p->sub_y) - 1) >> p->sub_y;
  g.sub_x = p->sub_x;
  g.sub_y = p->sub_y;
  g.bd = p->bd;
  g.damping = 3 + std::min(p->base_q_idx / 64, 3) + (p->bd - 8);
  return g;
}

// Scratch layout of mt_cdef_frame_device (256-byte aligned pieces).
struct Layout {
  size_t dirs, vars, tabs, dv_sum, dv_cnt, ustr, snap_y, snap_u, snap_v, total;
  size_t tab_bytes;  // one plane's table
  size_t read_bytes; // tabs .. dv_cnt end (the block read back to the host)
};

size_t up256(size_t v) { return (v + 255) & ~(size_t)255; }

Layout make_layout(const Geo& g, bool mono) {
  Layout L;
  const size_t nb = (size_t)g.nbx * g.nby, nu = (size_t)g.uc * g.ur;
  L.tab_bytes = nu * kNCand * 8;
  size_t o = 0;
  L.dirs = o;
  o += up256(nb);
  L.vars = o;
  o += up256(nb * 4);
  L.tabs = o;
  o += 3 * L.tab_bytes;
  L.dv_sum = o;
  o += nu * 8;
  L.dv_cnt = o;
  o += nu * 4;
  L.read_bytes = o - L.tabs;
  o = up256(o);
  L.ustr = o;
  o += up256(nu * 4);
  L.snap_y = o;
  o += up256((size_t)g.w8 * g.h8 * 2);
  L.snap_u = o;
  L.snap_v = o;
  if (!mono) {
    o += up256((size_t)g.cw8 * g.ch8 * 2);
    L.snap_v = o;
    o += up256((size_t)g.cw8 * g.ch8 * 2);
  }
  L.total = o;
  return L;
}

}  // namespace

namespace mth {
// Kernels the calling thread's last mt_cdef_frame_device launched (the
// direction and table kernels, and the apply kernel when a unit filters).
thread_local int cdef_last_launches = 0;
// Bytes mt_cdef_frame_device moves between the device and the host: the
// per-unit tables read back for the strength search (d2h) and the chosen
// per-unit strengths sent back (h2d, only when the apply kernel runs).
void cdef_frame_transfer_bytes(const mt_cdef_params* p, size_t* d2h, size_t* h2d) {
  const Geo g = make_geo(p);
  const Layout L = make_layout(g, p->mono != 0);
  *d2h = L.read_bytes;
  *h2d = (size_t)g.uc * g.ur * 4;
}
}  // namespace mth

namespace {

int launch_tables(const uint16_t* y, const uint16_t* u, const uint16_t* v, const uint16_t* sy, const uint16_t* su,
                  const uint16_t* sv, const uint8_t* skip8, const Geo& g, bool mono, uint8_t* dirs, int32_t* vars,
                  int64_t* ltab, int64_t* utab, int64_t* vtab, unsigned long long* dv_sum, int* dv_cnt,
                  cudaStream_t st) {
  const size_t nu = (size_t)g.uc * g.ur;
  if (cudaMemsetAsync(ltab, 0, nu * kNCand * 8, st) != cudaSuccess) return MT_ERR_DEVICE;
  if (!mono) {
    if (cudaMemsetAsync(utab, 0, nu * kNCand * 8, st) != cudaSuccess) return MT_ERR_DEVICE;
    if (cudaMemsetAsync(vtab, 0, nu * kNCand * 8, st) != cudaSuccess) return MT_ERR_DEVICE;
  }
  if (dv_sum) {
    if (cudaMemsetAsync(dv_sum, 0, nu * 8, st) != cudaSuccess) return MT_ERR_DEVICE;
    if (cudaMemsetAsync(dv_cnt, 0, nu * 4, st) != cudaSuccess) return MT_ERR_DEVICE;
  }
  const int nb = g.nbx * g.nby;
  cdef_dir_kernel<<<(nb + 127) / 128, 128, 0, st>>>(y, g, skip8, dirs, vars, dv_sum, dv_cnt);
  TabArgs ta;
  ta.rec[0] = y;
  ta.rec[1] = u;
  ta.rec[2] = v;
  ta.src[0] = sy;
  ta.src[1] = su;
  ta.src[2] = sv;
  ta.tab[0] = reinterpret_cast<unsigned long long*>(ltab);
  ta.tab[1] = reinterpret_cast<unsigned long long*>(utab);
  ta.tab[2] = reinterpret_cast<unsigned long long*>(vtab);
  cdef_tab_kernel<<<dim3(g.nbx, g.nby, mono ? 1 : 3), 64, 0, st>>>(ta, g, skip8, dirs, vars);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

// frame lambda_d (src/coder.rs:259-271): mode_lambda_q(dc_q) *
// mode_lambda_weight(qidx, sub) / K_PART_LAMBDA with the shipped tuning.
float frame_lambda_d(int qidx, int bd, int sub_x, int sub_y, float dc_q) {
  const int sub = (sub_x == 1 && sub_y == 1) ? 2 : (sub_x == 1 ? 1 : 0);
  const float dc8 = dc_q / (float)(1u << (std::max(bd, 8) - 8));
  volatile float kf = 0.0015f * dc8;
  kf = 3.3f + kf;
  volatile float mlq = 0.009005174719460433f * 1.0f;
  mlq = mlq * dc_q;
  mlq = mlq * dc_q;
  mlq = mlq * kf;
  const float scale = sub == 2 ? 0.8f : (sub == 1 ? 0.65f : 0.6f);
  int wi = ((255 - qidx) * 3) / 4;
  wi = std::min(std::max(wi, 0), 72) + 128;
  const float w = (float)wi * (1.0f / 128.0f);
  float weight;
  if (sub == 1) {
    weight = w * scale;
  } else {
    volatile float r = ((float)qidx - 0.0f) / (72.0f - 0.0f);
    float rr = std::min(std::max((float)r, 0.0f), 1.0f);
    volatile float m = (w - 3.0f) * rr;
    weight = (3.0f + m) * scale;
  }
  volatile float num = mlq * weight;
  return num / 2.775f;
}

int64_t sat_mul(int64_t a, int64_t b) {
  __int128 r = (__int128)a * b;
  if (r > INT64_MAX) return INT64_MAX;
  if (r < INT64_MIN) return INT64_MIN;
  return (int64_t)r;
}

// The staged strength search (src/coder/frame_cdef.rs:116-520) over the unit
// tables.  Returns the decision; ustr receives per-unit strengths.
void decide(const mt_cdef_params* p, const Geo& g, const int64_t* ltab, const int64_t* utab, const int64_t* vtab,
            const int64_t* dv_sum, const int32_t* dv_cnt, float dc_q, mt_cdef_decision* out, uint8_t* grid_out,
            std::vector<uint8_t>& ustr) {
  static const int kPri[4] = {0, 1, 2, 4};
  static const int kSec[3] = {0, 1, 2};
  const bool mono = p->mono != 0;
  const int nu = g.uc * g.ur;
  const int64_t margin = 40, gate = 15000;
  out->bits = -1;
  out->damping = 3 + std::min(p->base_q_idx / 64, 3);
  out->n_strengths = 0;
  out->unit_cols = g.uc;
  out->unit_rows = g.ur;
  memset(out->strengths, 0, sizeof(out->strengths));
  ustr.assign((size_t)nu * 4, 0);
  if (grid_out) memset(grid_out, 0, nu);
  std::vector<char> signaled(nu);
  int n_sig = 0, n_trusted = 0;
  for (int u = 0; u < nu; u++) {
    signaled[u] = dv_cnt[u] > 0;
    n_sig += signaled[u];
    if (gate == 0 || dv_sum[u] / std::max<int64_t>(dv_cnt[u], 1) >= gate) n_trusted++;
  }
  if (n_sig == 0) return;
  auto col = [](int pri, int sec) {
    int pi = 0, si = 0;
    for (int i = 0; i < 4; i++)
      if (kPri[i] == pri) pi = i;
    for (int i = 0; i < 3; i++)
      if (kSec[i] == sec) si = i;
    return si * 4 + pi;
  };
  auto off_of = [&](int64_t off) { return off - sat_mul(off, margin) / 1000; };
  // Candidate list.
  std::vector<std::pair<int, int>> cands = {{0, 0}};
  if (p->slow) {
    const int pri_list[3] = {1, 2, 4};
    std::vector<std::pair<int64_t, int>> ranked;
    for (int i = 0; i < 3; i++) {
      int64_t gsum = 0;
      const int c = col(pri_list[i], 0), c0 = col(0, 0);
      for (int u = 0; u < nu; u++) {
        const int64_t off = ltab[u * kNCand + c0], on = ltab[u * kNCand + c];
        gsum += on < off_of(off) ? off - on : 0;
      }
      ranked.push_back({gsum, i});
      cands.push_back({pri_list[i], 0});
    }
    std::stable_sort(ranked.begin(), ranked.end(), [](const std::pair<int64_t, int>& a, const std::pair<int64_t, int>& b) {
      return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    for (int sec : {1, 2}) {
      cands.push_back({0, sec});
      for (size_t r = 0; r < ranked.size() && r < 4; r++)
        if (ranked[r].first > 0) cands.push_back({pri_list[ranked[r].second], sec});
    }
  } else {
    for (int pri : {0, 1, 2, 4})
      for (int sec : {0, 1, 2})
        if (pri || sec) cands.push_back({pri, sec});
  }
  const size_t nl = cands.size();
  const size_t nc = mono ? 1 : nl;
  // ly[i][u], lc[i][u] flattened.
  std::vector<int64_t> ly(nl * nu), lc(nc * nu);
  for (size_t i = 0; i < nl; i++) {
    const int c = col(cands[i].first, cands[i].second);
    for (int u = 0; u < nu; u++) ly[i * nu + u] = ltab[u * kNCand + c];
  }
  for (size_t i = 0; i < nc; i++) {
    if (mono) {
      for (int u = 0; u < nu; u++) lc[u] = 0;
      break;
    }
    const int c = col(cands[i].first, cands[i].second);
    for (int u = 0; u < nu; u++) lc[i * nu + u] = utab[u * kNCand + c] + vtab[u * kNCand + c];
  }
  std::vector<int64_t> d_off(nu), thr(nu);
  int64_t total_off = 0;
  for (int u = 0; u < nu; u++) {
    d_off[u] = ly[u] + lc[u];
    thr[u] = off_of(d_off[u]);
    total_off += d_off[u];
  }
  const size_t n_pairs = nl * nc;
  // d_pair(p, u) for every pair, row-major by pair (n_pairs x nu).
  std::vector<int64_t> dp(n_pairs * nu);
  for (size_t pp = 0; pp < n_pairs; pp++) {
    const int64_t* a = &ly[(pp / nc) * nu];
    const int64_t* b = &lc[(pp % nc) * nu];
    int64_t* r = &dp[pp * nu];
    for (int u = 0; u < nu; u++) r[u] = a[u] + b[u];
  }
  auto d_pair = [&](size_t pp, int u) { return dp[pp * nu + u]; };
  // Units that never signal contribute d_off whatever the entry.
  std::vector<int> sig_units;
  int64_t unsig_off = 0;
  for (int u = 0; u < nu; u++) {
    if (signaled[u])
      sig_units.push_back(u);
    else
      unsig_off += d_off[u];
  }
  size_t global_entry = 0;
  int64_t prefix[4] = {INT64_MAX, INT64_MAX, INT64_MAX, INT64_MAX};
  for (size_t pp = 0; pp < n_pairs; pp++) {
    const int64_t* r = &dp[pp * nu];
    int64_t t = unsig_off;
    for (int u : sig_units) t += r[u];
    if (t < prefix[0]) {
      prefix[0] = t;
      global_entry = pp;
    }
  }
  // Greedy set construction on the signalled units (compacted copies).
  const size_t ns = sig_units.size();
  std::vector<int64_t> cm(ns), th(ns), off(ns), dps(n_pairs * ns);
  for (size_t k = 0; k < ns; k++) {
    const int u = sig_units[k];
    cm[k] = d_off[u];
    th[k] = thr[u];
    off[k] = d_off[u];
  }
  for (size_t pp = 0; pp < n_pairs; pp++)
    for (size_t k = 0; k < ns; k++) dps[pp * ns + k] = dp[pp * nu + sig_units[k]];
  std::vector<size_t> entries = {0};
  while (entries.size() < 8) {
    size_t best_p = 0;
    int64_t best_tot = INT64_MAX;
    for (size_t pp = 0; pp < n_pairs; pp++) {
      const int64_t* r = &dps[pp * ns];
      int64_t tot = unsig_off;
      for (size_t k = 0; k < ns; k++) {
        const int64_t b = cm[k] < r[k] ? cm[k] : r[k];
        tot += b >= th[k] ? off[k] : b;
      }
      if (tot < best_tot) {
        best_tot = tot;
        best_p = pp;
      }
    }
    entries.push_back(best_p);
    const int64_t* r = &dps[best_p * ns];
    for (size_t k = 0; k < ns; k++) cm[k] = std::min(cm[k], r[k]);
    const size_t n = entries.size();
    if ((n & (n - 1)) == 0) prefix[__builtin_ctzll(n)] = best_tot;
  }
  auto pair_strengths = [&](size_t pp, int s[4]) {
    s[0] = cands[pp / nc].first;
    s[1] = cands[pp / nc].second;
    s[2] = mono ? 0 : cands[pp % nc].first;
    s[3] = mono ? 0 : cands[pp % nc].second;
  };
  auto assign = [&](const size_t* set, size_t nset, std::vector<uint8_t>& grid) -> int64_t {
    int z = -1;
    for (size_t e = 0; e < nset; e++)
      if (set[e] == 0) {
        z = (int)e;
        break;
      }
    int64_t total = 0;
    grid.assign(nu, 0);
    for (int u = 0; u < nu; u++) {
      if (!signaled[u]) {
        total += d_off[u];
        continue;
      }
      bool have = false;
      int pm = 0;
      int64_t pd = 0, rb_d = INT64_MAX;
      size_t pe = 0, rb_e = 0;
      for (size_t e = 0; e < nset; e++) {
        const int64_t d = d_pair(set[e], u);
        if (d < rb_d) {
          rb_d = d;
          rb_e = e;
        }
        if (d < thr[u]) {
          int s[4];
          pair_strengths(set[e], s);
          const int mag = s[0] + s[1] + s[2] + s[3];
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
        grid[u] = (uint8_t)pe;
      } else if (z >= 0) {
        total += d_off[u];
        grid[u] = (uint8_t)z;
      } else {
        total += rb_d;
        grid[u] = (uint8_t)rb_e;
      }
    }
    return total;
  };
  const float lambda = frame_lambda_d(p->base_q_idx, p->bd, p->sub_x, p->sub_y, dc_q);
  const float cost_off = (float)total_off;
  const float per_entry_bits = mono ? 6.0f : 12.0f;
  int best_bits = -1;
  float best_cost = cost_off;
  std::vector<uint8_t> grid;
  for (int b = 0; b <= 3; b++) {
    const int nb = 1 << b;
    const int64_t total = b == 0 ? prefix[0] : assign(entries.data(), nb, grid);
    if (total == INT64_MAX) continue;
    if (b == 0 && (global_entry == 0 || n_trusted * 4 < n_sig * 3 || total >= off_of(total_off))) continue;
    volatile float e_bits = per_entry_bits * (float)(nb - 1);
    volatile float u_bits = (float)b * (float)n_sig;
    volatile float bits_f = e_bits + u_bits;
    volatile float lb = lambda * bits_f;
    const float cost = (float)total + lb;
    if (cost < best_cost) {
      best_cost = cost;
      best_bits = b;
    }
  }
  if (best_bits < 0) return;
  std::vector<size_t> set;
  if (best_bits == 0)
    set = {global_entry};
  else
    set.assign(entries.begin(), entries.begin() + (1 << best_bits));
  grid.assign(nu, 0);
  if (best_bits > 0) assign(set.data(), set.size(), grid);
  out->bits = best_bits;
  out->n_strengths = (int)set.size();
  for (size_t e = 0; e < set.size(); e++) {
    int s[4];
    pair_strengths(set[e], s);
    for (int k = 0; k < 4; k++) out->strengths[e][k] = (uint8_t)s[k];
  }
  if (grid_out && best_bits > 0) memcpy(grid_out, grid.data(), nu);
  for (int u = 0; u < nu; u++)
    for (int k = 0; k < 4; k++) ustr[(size_t)u * 4 + k] = out->strengths[grid[u]][k];
}

}  // namespace

extern "C" {

int mt_quant_init(uint8_t base_q_idx, uint8_t bd, uint8_t qm_level, mt_quant* out);

int mt_cdef_tables_device(const uint16_t* d_y, const uint16_t* d_u, const uint16_t* d_v, const uint16_t* d_src_y,
                          const uint16_t* d_src_u, const uint16_t* d_src_v, const uint8_t* d_skip8,
                          const mt_cdef_params* prm, uint8_t* d_dirs, int32_t* d_vars, int64_t* d_luma_tab,
                          int64_t* d_u_tab, int64_t* d_v_tab, void* stream) {
  int rc = check_params(prm);
  if (rc != MT_OK) return rc;
  const bool mono = prm->mono != 0;
  if (!d_y || !d_src_y || !d_skip8 || !d_dirs || !d_vars || !d_luma_tab) return MT_ERR_INVALID_INPUT;
  if (!mono && (!d_u || !d_v || !d_src_u || !d_src_v || !d_u_tab || !d_v_tab)) return MT_ERR_INVALID_INPUT;
  const Geo g = make_geo(prm);
  return launch_tables(d_y, d_u, d_v, d_src_y, d_src_u, d_src_v, d_skip8, g, mono, d_dirs, d_vars, d_luma_tab,
                       d_u_tab, d_v_tab, nullptr, nullptr, reinterpret_cast<cudaStream_t>(stream));
}

size_t mt_cdef_scratch_bytes(const mt_cdef_params* prm) {
  if (check_params(prm) != MT_OK) return 0;
  return make_layout(make_geo(prm), prm->mono != 0).total;
}

int mt_cdef_frame_device(uint16_t* d_y, uint16_t* d_u, uint16_t* d_v, const uint16_t* d_src_y,
                         const uint16_t* d_src_u, const uint16_t* d_src_v, const uint8_t* d_skip8,
                         const mt_cdef_params* prm, void* d_scratch, mt_cdef_decision* out, uint8_t* grid,
                         void* stream) {
  int rc = check_params(prm);
  if (rc != MT_OK) return rc;
  const bool mono = prm->mono != 0;
  if (!d_y || !d_src_y || !d_skip8 || !d_scratch || !out) return MT_ERR_INVALID_INPUT;
  if (!mono && (!d_u || !d_v || !d_src_u || !d_src_v)) return MT_ERR_INVALID_INPUT;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const Geo g = make_geo(prm);
  const Layout L = make_layout(g, mono);
  uint8_t* s = static_cast<uint8_t*>(d_scratch);
  const size_t nu = (size_t)g.uc * g.ur;
  uint8_t* dirs = s + L.dirs;
  int32_t* vars = reinterpret_cast<int32_t*>(s + L.vars);
  int64_t* tabs = reinterpret_cast<int64_t*>(s + L.tabs);
  unsigned long long* dv_sum = reinterpret_cast<unsigned long long*>(s + L.dv_sum);
  int* dv_cnt = reinterpret_cast<int*>(s + L.dv_cnt);
  mth::cdef_last_launches = 0;
  rc = launch_tables(d_y, d_u, d_v, d_src_y, d_src_u, d_src_v, d_skip8, g, mono, dirs, vars, tabs, tabs + nu * kNCand,
                     tabs + 2 * nu * kNCand, dv_sum, dv_cnt, st);
  if (rc != MT_OK) return rc;
  mth::cdef_last_launches = 2;
  // Read the tables back (one copy) for the host search.
  std::vector<uint8_t> host(L.read_bytes);
  if (cudaMemcpyAsync(host.data(), s + L.tabs, L.read_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MT_ERR_DEVICE;
  const int64_t* h_tabs = reinterpret_cast<const int64_t*>(host.data());
  const int64_t* h_dv_sum = reinterpret_cast<const int64_t*>(host.data() + (L.dv_sum - L.tabs));
  const int32_t* h_dv_cnt = reinterpret_cast<const int32_t*>(host.data() + (L.dv_cnt - L.tabs));
  mt_quant q;
  if (mt_quant_init((uint8_t)prm->base_q_idx, (uint8_t)prm->bd, 15, &q) != MT_OK) return MT_ERR_INVALID_INPUT;
  std::vector<uint8_t> ustr;
  decide(prm, g, h_tabs, h_tabs + nu * kNCand, h_tabs + 2 * nu * kNCand, h_dv_sum, h_dv_cnt, (float)q.dc_q, out, grid,
         ustr);
  if (out->bits < 0) return MT_OK;
  bool any_y = false, any_uv = false;
  for (size_t u = 0; u < nu; u++) {
    any_y |= (ustr[u * 4] | ustr[u * 4 + 1]) != 0;
    any_uv |= (ustr[u * 4 + 2] | ustr[u * 4 + 3]) != 0;
  }
  if (!any_y && (mono || !any_uv)) return MT_OK;
  if (cudaMemcpyAsync(s + L.ustr, ustr.data(), nu * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return MT_ERR_DEVICE;
  ApplyArgs aa;
  aa.rec[0] = d_y;
  aa.rec[1] = d_u;
  aa.rec[2] = d_v;
  aa.snap[0] = reinterpret_cast<uint16_t*>(s + L.snap_y);
  aa.snap[1] = reinterpret_cast<uint16_t*>(s + L.snap_u);
  aa.snap[2] = reinterpret_cast<uint16_t*>(s + L.snap_v);
  const size_t ny = (size_t)g.w8 * g.h8 * 2, nc = (size_t)g.cw8 * g.ch8 * 2;
  if (cudaMemcpyAsync(s + L.snap_y, d_y, ny, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MT_ERR_DEVICE;
  if (!mono) {
    if (cudaMemcpyAsync(s + L.snap_u, d_u, nc, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MT_ERR_DEVICE;
    if (cudaMemcpyAsync(s + L.snap_v, d_v, nc, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return MT_ERR_DEVICE;
  }
  cdef_apply_kernel<<<dim3(g.nbx, g.nby, mono ? 1 : 3), 64, 0, st>>>(aa, g, d_skip8, dirs, vars, s + L.ustr);
  mth::cdef_last_launches = 3;
  // The strengths were staged from pageable host memory; keep the buffer alive
  // until the copy has been consumed.
  if (cudaStreamSynchronize(st) != cudaSuccess) return MT_ERR_DEVICE;
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

int mt_cdef_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint16_t* src_y, const uint16_t* src_u,
                  const uint16_t* src_v, const uint8_t* skip8, const mt_cdef_params* prm, mt_cdef_decision* out,
                  uint8_t* grid) {
  int rc = check_params(prm);
  if (rc != MT_OK) return rc;
  const bool mono = prm->mono != 0;
  if (!y || !src_y || !skip8 || !out) return MT_ERR_INVALID_INPUT;
  if (!mono && (!u || !v || !src_u || !src_v)) return MT_ERR_INVALID_INPUT;
  const Geo g = make_geo(prm);
  const size_t ny = (size_t)g.w8 * g.h8 * 2, nc = mono ? 0 : (size_t)g.cw8 * g.ch8 * 2, nsk = (size_t)g.nbx * g.nby;
  const size_t scratch = mt_cdef_scratch_bytes(prm);
  const size_t o_y = 0, o_sy = up256(ny), o_u = o_sy + up256(ny), o_v = o_u + up256(nc), o_su = o_v + up256(nc),
               o_sv = o_su + up256(nc), o_sk = o_sv + up256(nc), o_scr = o_sk + up256(nsk);
  uint8_t* d = nullptr;
  if (cudaMalloc(&d, o_scr + scratch) != cudaSuccess) return MT_ERR_ALLOC;
  cudaError_t e = cudaMemcpy(d + o_y, y, ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_sy, src_y, ny, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + o_sk, skip8, nsk, cudaMemcpyHostToDevice);
  if (!mono) {
    if (e == cudaSuccess) e = cudaMemcpy(d + o_u, u, nc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_v, v, nc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_su, src_u, nc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + o_sv, src_v, nc, cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) {
    rc = mt_cdef_frame_device((uint16_t*)(d + o_y), mono ? nullptr : (uint16_t*)(d + o_u),
                              mono ? nullptr : (uint16_t*)(d + o_v), (const uint16_t*)(d + o_sy),
                              mono ? nullptr : (const uint16_t*)(d + o_su), mono ? nullptr : (const uint16_t*)(d + o_sv),
                              d + o_sk, prm, d + o_scr, out, grid, nullptr);
    if (rc == MT_OK) {
      e = cudaMemcpy(y, d + o_y, ny, cudaMemcpyDeviceToHost);
      if (!mono && e == cudaSuccess) e = cudaMemcpy(u, d + o_u, nc, cudaMemcpyDeviceToHost);
      if (!mono && e == cudaSuccess) e = cudaMemcpy(v, d + o_v, nc, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(d);
  if (rc != MT_OK) return rc;
  return e == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
}

}  // extern "C"
