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
//   the strength search   the staged search over the unit tables
//                        (src/coder/frame_cdef.rs:116-520) as a chain of small
//                        kernels, so that tables, search and apply run back to
//                        back on the stream and the host reads the decision
//                        once at the end.
#include <cuda_runtime.h>
#include <limits.h>
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

constexpr int kMaxPairs = 144;  // 12 luma x 12 chroma candidates
constexpr long long kMargin = 40, kGate = 15000;
constexpr int kGreedySteps = 7;  // entries 2 .. 8
constexpr int kSearchThreads = 256;

struct SearchState {
  // the decision
  int32_t bits, n_strengths;
  uint8_t strengths[8][4];
  // unit statistics: signalling units, trusted units, distortion sums
  unsigned long long n_sig, n_trusted, total_off, unsig_off, gsum[3];
  // candidates: (pri, sec) and the table column of each
  int32_t nl, nc, np;
  uint8_t cand[12][2];
  int8_t col[12];
  // pass totals: [0] the single-entry pass, [1] and [2] alternate in the greedy passes
  unsigned long long tot[3][kMaxPairs];
  long long prefix[4];
  int32_t global_entry, nentries;
  int32_t entries[8];
  unsigned long long assign_total[4];  // the 2-, 4- and 8-entry sets at [1..3]
};

// Scratch layout of mt_cdef_frame_device (256-byte aligned pieces).
struct Layout {
  size_t dirs, vars, tabs, dv_sum, dv_cnt, ustr, snap_y, snap_u, snap_v, total;
  size_t state, d_off, thr, cm, sig, grids, grid;  // the strength search
  size_t tab_bytes;  // one plane's table
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
  o = up256(o);
  L.ustr = o;
  o += up256(nu * 4);
  L.state = o;
  o += up256(sizeof(SearchState));
  L.d_off = o;
  o += up256(nu * 8);
  L.thr = o;
  o += up256(nu * 8);
  L.cm = o;
  o += up256(nu * 8);
  L.sig = o;
  o += up256(nu);
  L.grids = o;
  o += up256(3 * nu);
  L.grid = o;
  o += up256(nu);
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
// direction and table kernels, the strength search's kernels and the apply
// kernel).
thread_local int cdef_last_launches = 0;
// Bytes mt_cdef_frame_device reads back to the host: the search's state
// (decision and statistics) and, when asked for, the per-unit grid.
void cdef_frame_transfer_bytes(const mt_cdef_params* p, size_t* d2h, size_t* h2d) {
  const Geo g = make_geo(p);
  *d2h = sizeof(SearchState) + (size_t)g.uc * g.ur;
  *h2d = 0;
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

// ---------------------------------------------------------------------------
// The staged strength search (src/coder/frame_cdef.rs:116-520) on the device,
// as a chain of small kernels on the stream (no host round trip): the unit
// statistics, the candidate list, the single-entry pass, seven greedy entry
// passes, the assignment of the 2-, 4- and 8-entry sets to the units, the rate
// decision and the per-unit strengths the apply kernel reads.  Integer sums
// are 64-bit atomics (order-free, exact); every choice is the first minimum in
// the reference's order, and the rate arithmetic is the reference's f32
// operations one by one.

struct SearchArgs {
  const long long* ltab;
  const long long* utab;
  const long long* vtab;
  const unsigned long long* dv_sum;
  const int* dv_cnt;
  int nu, mono, slow;
  float lambda;      // the frame lambda_d pricing the CDEF bits
  SearchState* S;
  long long* d_off;  // distortion with CDEF off, per unit
  long long* thr;    // its margin threshold
  long long* cm;     // the greedy set's best distortion so far
  uint8_t* sig;      // the unit signals a strength index (a non-skip block)
  uint8_t* grids;    // 3 x nu: the entry of each unit for the 2-, 4- and 8-entry sets
  uint8_t* grid;     // nu: the chosen set's entry per unit (0 unless bits > 0)
  uint8_t* ustr;     // nu x 4: the unit's strengths for the apply kernel
};

__host__ __device__ __forceinline__ long long sat_mul_pos(long long a, long long b) {  // b > 0
  if (a > LLONG_MAX / b) return LLONG_MAX;
  if (a < LLONG_MIN / b) return LLONG_MIN;
  return a * b;
}
__host__ __device__ __forceinline__ long long off_of(long long off) { return off - sat_mul_pos(off, kMargin) / 1000; }
__host__ __device__ __forceinline__ int cand_col(int pri, int sec) {  // sec_idx * 4 + pri_idx
  return sec * 4 + (pri == 4 ? 3 : pri);
}

__device__ __forceinline__ long long d_pair(const SearchArgs& a, const SearchState& S, int pp, int u) {
  long long d = a.ltab[(size_t)u * kNCand + S.col[pp / S.nc]];
  if (!a.mono) {
    const int c = S.col[pp % S.nc];
    d += a.utab[(size_t)u * kNCand + c] + a.vtab[(size_t)u * kNCand + c];
  }
  return d;
}

// The four strengths of pair pp (luma pri, sec, chroma pri, sec).
__device__ __forceinline__ void pair_strengths(const SearchState& S, int mono, int pp, int s[4]) {
  s[0] = S.cand[pp / S.nc][0];
  s[1] = S.cand[pp / S.nc][1];
  s[2] = mono ? 0 : S.cand[pp % S.nc][0];
  s[3] = mono ? 0 : S.cand[pp % S.nc][1];
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sums of v[0..N) over the CTA into dst[0..N) with one atomic each
// (kSearchThreads threads).
template <int N>
__device__ __forceinline__ void block_add(unsigned long long (&v)[N], unsigned long long* const (&dst)[N]) {
  __shared__ unsigned long long part[N][kSearchThreads / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < N; k++) {
    const unsigned long long s = warp_sum(v[k]);
    if (l == 0) part[k][w] = s;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < N; k++) {
      unsigned long long s = l < kSearchThreads / 32 ? part[k][l] : 0ull;
      s = warp_sum(s);
      if (l == 0 && s) atomicAdd(dst[k], s);
    }
  }
}

// Per unit: the signalling and trust flags (directional-variance gate), the
// CDEF-off distortion and its threshold, and the luma gains of pri 1 / 2 / 4
// that rank the Slow candidate list.
__global__ void __launch_bounds__(kSearchThreads) cdef_unit_stats_kernel(SearchArgs a) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  SearchState& S = *a.S;
  unsigned long long v[7] = {0, 0, 0, 0, 0, 0, 0};  // n_sig, n_trusted, total_off, unsig_off, gsum[3]
  if (u < a.nu) {
    const bool sg = a.dv_cnt[u] > 0;
    const long long cnt = a.dv_cnt[u] > 1 ? a.dv_cnt[u] : 1;
    const long long* lt = a.ltab + (size_t)u * kNCand;
    const long long lo = lt[0];
    const long long off = lo + (a.mono ? 0 : a.utab[(size_t)u * kNCand] + a.vtab[(size_t)u * kNCand]);
    a.d_off[u] = off;
    a.thr[u] = off_of(off);
    a.cm[u] = off;
    a.sig[u] = sg;
    v[0] = sg;
    v[1] = (long long)a.dv_sum[u] / cnt >= kGate;
    v[2] = (unsigned long long)off;
    v[3] = sg ? 0ull : (unsigned long long)off;
    const long long lim = off_of(lo);
#pragma unroll
    for (int i = 0; i < 3; i++) {  // pri 1, 2, 4 at sec 0: columns 1..3
      const long long on = lt[1 + i];
      v[4 + i] = on < lim ? (unsigned long long)(lo - on) : 0ull;
    }
  }
  unsigned long long* const dst[7] = {&S.n_sig, &S.n_trusted, &S.total_off, &S.unsig_off,
                                      &S.gsum[0], &S.gsum[1], &S.gsum[2]};
  block_add<7>(v, dst);
}

// The candidate list (one thread): Slow ranks pri 1 / 2 / 4 by their gains
// and pairs the useful ones with sec 1 and 2; otherwise all 12.
__global__ void cdef_plan_kernel(SearchArgs a) {
  SearchState& S = *a.S;
  int n = 0;
  auto push = [&](int pri, int sec) {
    S.cand[n][0] = (uint8_t)pri;
    S.cand[n][1] = (uint8_t)sec;
    S.col[n] = (int8_t)cand_col(pri, sec);
    ++n;
  };
  push(0, 0);
  if (a.slow) {
    const int pri_list[3] = {1, 2, 4};
    int r[3] = {0, 1, 2};  // stable: larger gain first, then list order
    for (int i = 1; i < 3; i++)
      for (int j = i; j > 0 && S.gsum[r[j]] > S.gsum[r[j - 1]]; j--) {
        const int t = r[j];
        r[j] = r[j - 1];
        r[j - 1] = t;
      }
    for (int i = 0; i < 3; i++) push(pri_list[i], 0);
    for (int sec = 1; sec <= 2; sec++) {
      push(0, sec);
      for (int k = 0; k < 3; k++)
        if (S.gsum[r[k]] > 0) push(pri_list[r[k]], sec);
    }
  } else {
    const int pl[4] = {0, 1, 2, 4};
    for (int i = 0; i < 4; i++)
      for (int sec = 0; sec <= 2; sec++)
        if (pl[i] || sec) push(pl[i], sec);
  }
  S.nl = n;
  S.nc = a.mono ? 1 : n;
  S.np = n * S.nc;
  for (int k = 0; k < 4; k++) S.prefix[k] = LLONG_MAX;
  S.entries[0] = 0;
  S.nentries = 1;
}

// Per (pair, chunk of units): the pair's total over the signalling units.
// Pass 0 (the single-entry pass): its distortion.  Greedy passes: the set
// extended by the pair, each unit at the better of the set and the pair, or
// at CDEF off when that is within the margin.
__global__ void __launch_bounds__(kSearchThreads) cdef_pair_sum_kernel(SearchArgs a, int buf) {
  const SearchState& S = *a.S;
  const int pp = blockIdx.y;
  if (S.n_sig == 0 || pp >= S.np) return;
  unsigned long long v[1] = {0};
  for (int u = blockIdx.x * kSearchThreads + threadIdx.x; u < a.nu; u += gridDim.x * kSearchThreads) {
    if (!a.sig[u]) continue;
    const long long r = d_pair(a, S, pp, u);
    if (buf == 0) {
      v[0] += (unsigned long long)r;
    } else {
      const long long b = a.cm[u] < r ? a.cm[u] : r;
      v[0] += (unsigned long long)(b >= a.thr[u] ? a.d_off[u] : b);
    }
  }
  unsigned long long* const dst[1] = {&a.S->tot[buf][pp]};
  block_add<1>(v, dst);
}

// First minimum over the pairs of unsig_off + tot[buf][pair].
__device__ __forceinline__ int first_min(const SearchState& S, int buf, long long* best) {
  int bp = 0;
  long long bt = LLONG_MAX;
  for (int pp = 0; pp < S.np; pp++) {
    const long long t = (long long)(S.unsig_off + S.tot[buf][pp]);
    if (t < bt) {
      bt = t;
      bp = pp;
    }
  }
  *best = bt;
  return bp;
}

// The single-entry pass's best pair (one thread).
__global__ void cdef_global_entry_kernel(SearchArgs a) {
  SearchState& S = *a.S;
  if (S.n_sig == 0) return;
  long long bt;
  S.global_entry = first_min(S, 0, &bt);
  S.prefix[0] = bt;
}

// One greedy step: every CTA finds the pass's best pair (the same one) and
// lowers its units' set distortion to it; CTA 0 records the entry and clears
// the other pass buffer for the next step.
__global__ void __launch_bounds__(kSearchThreads) cdef_greedy_step_kernel(SearchArgs a, int buf) {
  SearchState& S = *a.S;
  if (S.n_sig == 0) return;
  __shared__ int s_best;
  __shared__ long long s_tot;
  if (threadIdx.x == 0) {
    long long bt;
    s_best = first_min(S, buf, &bt);
    s_tot = bt;
  }
  __syncthreads();
  const int bp = s_best;
  if (blockIdx.x == 0) {
    const int other = buf == 1 ? 2 : 1;
    for (int pp = threadIdx.x; pp < kMaxPairs; pp += blockDim.x) S.tot[other][pp] = 0;
    if (threadIdx.x == 0) {
      const int n = S.nentries + 1;
      S.entries[n - 1] = bp;
      S.nentries = n;
      if ((n & (n - 1)) == 0) S.prefix[__ffs(n) - 1] = s_tot;
    }
  }
  for (int u = blockIdx.x * kSearchThreads + threadIdx.x; u < a.nu; u += gridDim.x * kSearchThreads) {
    if (!a.sig[u]) continue;
    const long long r = d_pair(a, S, bp, u);
    if (r < a.cm[u]) a.cm[u] = r;
  }
}

// The 2-, 4- and 8-entry sets' per-unit entries and totals: a unit takes the
// smallest-magnitude entry within its margin (ties by distortion, then list
// order), else the zero entry at CDEF off, else its best entry.
__global__ void __launch_bounds__(kSearchThreads) cdef_assign_kernel(SearchArgs a) {
  const SearchState& S = *a.S;
  if (S.n_sig == 0) return;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v[3] = {0, 0, 0};
  if (u < a.nu) {
    for (int b = 1; b <= 3; b++) {
      const int nset = 1 << b;
      uint8_t g = 0;
      if (!a.sig[u]) {
        v[b - 1] = (unsigned long long)a.d_off[u];
      } else {
        int z = -1;
        for (int e = 0; e < nset; e++)
          if (S.entries[e] == 0) {
            z = e;
            break;
          }
        bool have = false;
        int pm = 0, pe = 0, rb_e = 0;
        long long pd = 0, rb_d = LLONG_MAX;
        for (int e = 0; e < nset; e++) {
          const long long d = d_pair(a, S, S.entries[e], u);
          if (d < rb_d) {
            rb_d = d;
            rb_e = e;
          }
          if (d < a.thr[u]) {
            int s[4];
            pair_strengths(S, a.mono, S.entries[e], s);
            const int mag = s[0] + s[1] + s[2] + s[3];
            if (!have || mag < pm || (mag == pm && d < pd)) {
              have = true;
              pm = mag;
              pd = d;
              pe = e;
            }
          }
        }
        long long t;
        if (have) {
          t = pd;
          g = (uint8_t)pe;
        } else if (z >= 0) {
          t = a.d_off[u];
          g = (uint8_t)z;
        } else {
          t = rb_d;
          g = (uint8_t)rb_e;
        }
        v[b - 1] = (unsigned long long)t;
      }
      a.grids[(size_t)(b - 1) * a.nu + u] = g;
    }
  }
  unsigned long long* const dst[3] = {&a.S->assign_total[1], &a.S->assign_total[2], &a.S->assign_total[3]};
  block_add<3>(v, dst);
}

// The rate decision (one thread): CDEF off, the single entry, or 2 / 4 / 8
// entries, each priced as distortion + lambda_d x (entry bits + index bits).
__global__ void cdef_decide_kernel(SearchArgs a) {
  SearchState& S = *a.S;
  S.bits = -1;
  S.n_strengths = 0;
  for (int e = 0; e < 8; e++)
    for (int k = 0; k < 4; k++) S.strengths[e][k] = 0;
  if (S.n_sig == 0) return;
  const long long total_off = (long long)S.total_off;
  const float per_entry_bits = a.mono ? 6.0f : 12.0f;
  const int n_sig = (int)S.n_sig, n_trusted = (int)S.n_trusted;
  int best_bits = -1;
  float best_cost = __ll2float_rn(total_off);
  for (int b = 0; b <= 3; b++) {
    const int nb = 1 << b;
    const long long total = b == 0 ? S.prefix[0] : (long long)S.assign_total[b];
    if (total == LLONG_MAX) continue;
    if (b == 0 && (S.global_entry == 0 || n_trusted * 4 < n_sig * 3 || total >= off_of(total_off))) continue;
    const float e_bits = __fmul_rn(per_entry_bits, __int2float_rn(nb - 1));
    const float u_bits = __fmul_rn(__int2float_rn(b), __int2float_rn(n_sig));
    const float bits_f = __fadd_rn(e_bits, u_bits);
    const float lb = __fmul_rn(a.lambda, bits_f);
    const float cost = __fadd_rn(__ll2float_rn(total), lb);
    if (cost < best_cost) {
      best_cost = cost;
      best_bits = b;
    }
  }
  if (best_bits < 0) return;
  const int n = 1 << best_bits;
  S.bits = best_bits;
  S.n_strengths = n;
  for (int e = 0; e < n; e++) {
    int s[4];
    pair_strengths(S, a.mono, best_bits == 0 ? S.global_entry : S.entries[e], s);
    for (int k = 0; k < 4; k++) S.strengths[e][k] = (uint8_t)s[k];
  }
}

// Each unit's entry and strengths under the decision (all zero when CDEF is
// off: the apply kernel then leaves the planes as they are).
__global__ void __launch_bounds__(kSearchThreads) cdef_unit_strengths_kernel(SearchArgs a) {
  const SearchState& S = *a.S;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= a.nu) return;
  const int g = S.bits > 0 ? a.grids[(size_t)(S.bits - 1) * a.nu + u] : 0;
  a.grid[u] = (uint8_t)g;
#pragma unroll
  for (int k = 0; k < 4; k++) a.ustr[(size_t)u * 4 + k] = S.bits >= 0 ? S.strengths[g][k] : 0;
}

// The search's launches on the stream, after the tables.
constexpr int kSearchLaunches = 7 + 2 * kGreedySteps;

int launch_search(const SearchArgs& a, cudaStream_t st) {
  if (cudaMemsetAsync(a.S, 0, sizeof(SearchState), st) != cudaSuccess) return MT_ERR_DEVICE;
  const int ublocks = (a.nu + kSearchThreads - 1) / kSearchThreads;
  const int chunks = std::min(ublocks, 16);  // unit chunks per pair in the pass sums
  cdef_unit_stats_kernel<<<ublocks, kSearchThreads, 0, st>>>(a);
  cdef_plan_kernel<<<1, 1, 0, st>>>(a);
  cdef_pair_sum_kernel<<<dim3(chunks, kMaxPairs), kSearchThreads, 0, st>>>(a, 0);
  cdef_global_entry_kernel<<<1, 1, 0, st>>>(a);
  for (int k = 0; k < kGreedySteps; k++) {
    const int buf = 1 + (k & 1);
    cdef_pair_sum_kernel<<<dim3(chunks, kMaxPairs), kSearchThreads, 0, st>>>(a, buf);
    cdef_greedy_step_kernel<<<std::min(ublocks, 64), kSearchThreads, 0, st>>>(a, buf);
  }
  cdef_assign_kernel<<<ublocks, kSearchThreads, 0, st>>>(a);
  cdef_decide_kernel<<<1, 1, 0, st>>>(a);
  cdef_unit_strengths_kernel<<<ublocks, kSearchThreads, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_DEVICE;
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
  // the strength search on the stream
  mt_quant q;
  if (mt_quant_init((uint8_t)prm->base_q_idx, (uint8_t)prm->bd, 15, &q) != MT_OK) return MT_ERR_INVALID_INPUT;
  SearchArgs sa;
  sa.ltab = reinterpret_cast<const long long*>(tabs);
  sa.utab = reinterpret_cast<const long long*>(tabs + nu * kNCand);
  sa.vtab = reinterpret_cast<const long long*>(tabs + 2 * nu * kNCand);
  sa.dv_sum = dv_sum;
  sa.dv_cnt = dv_cnt;
  sa.nu = (int)nu;
  sa.mono = mono;
  sa.slow = prm->slow != 0;
  sa.lambda = frame_lambda_d(prm->base_q_idx, prm->bd, prm->sub_x, prm->sub_y, (float)q.dc_q);
  sa.S = reinterpret_cast<SearchState*>(s + L.state);
  sa.d_off = reinterpret_cast<long long*>(s + L.d_off);
  sa.thr = reinterpret_cast<long long*>(s + L.thr);
  sa.cm = reinterpret_cast<long long*>(s + L.cm);
  sa.sig = s + L.sig;
  sa.grids = s + L.grids;
  sa.grid = s + L.grid;
  sa.ustr = s + L.ustr;
  if ((rc = launch_search(sa, st)) != MT_OK) return rc;
  mth::cdef_last_launches += kSearchLaunches;
  // the filter from a pre-CDEF snapshot, with each unit's strengths (all zero:
  // the planes stay as they are)
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
  mth::cdef_last_launches += 1;
  // the decision back to the host, once, at the end
  SearchState hs;
  if (cudaMemcpyAsync(&hs, s + L.state, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess) return MT_ERR_DEVICE;
  if (grid && cudaMemcpyAsync(grid, s + L.grid, nu, cudaMemcpyDeviceToHost, st) != cudaSuccess) return MT_ERR_DEVICE;
  if (cudaStreamSynchronize(st) != cudaSuccess) return MT_ERR_DEVICE;
  out->bits = hs.bits;
  out->damping = 3 + std::min(prm->base_q_idx / 64, 3);
  out->n_strengths = hs.n_strengths;
  out->unit_cols = g.uc;
  out->unit_rows = g.ur;
  memcpy(out->strengths, hs.strengths, sizeof(out->strengths));
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
