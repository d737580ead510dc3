// Frame-level rate-distortion parameters of the shipped Slow operating point:
// quality -> base qindex (src/avif.rs:637-666 quality_to_q), the quantisation-
// matrix level laws (src/quant.rs:122-167) and the decision lambdas
// (src/cost.rs:115-148, :269-292, src/partition_rd.rs:30-71,
// src/coder/lossy_state.rs:1681-1684, :1769-1788, :1864-1871, :2385-2409).
// Host code only; the values are inputs of the batched kernels.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../../include/maroontree_b200.h"

namespace {

// Shipped tuning constants these laws read (src/tuning.rs:750-784, :854-857,
// :913-915) and the model constants of src/cost.rs:93, :269-280.
constexpr float kTrellisLambda0 = 0.05f;
constexpr float kModeAomCalib = 0.009005174719460433f;
constexpr float kPartLambda = 2.775f;
constexpr float kMlamScale420 = 0.8f, kMlamScale422 = 0.65f, kMlamScale444 = 0.6f;
constexpr float kModeLambdaLoFloor = 0.0f, kModeLambdaLoFull = 72.0f, kModeLambdaLoW = 3.0f;
constexpr float kSatdBase = 1.25f, kSatdTop = 2.921556f, kSatdKneeLo = 20.0f, kSatdKneeHi = 48.0f;
constexpr float kProxyLumaScale = 7.130643f;
constexpr float kTopEase = 1.0f;
constexpr float kQmHqKnee = 12.0f, kQmHqWidth = 5.0f;

float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

// util.rs:36-59 fast_round on x86-64: add one ulp, then round to nearest even
// through the 1.5 * 2^23 magic constant.
float fast_round(float v) {
  uint32_t b;
  memcpy(&b, &v, 4);
  b += 1;
  float u;
  memcpy(&u, &b, 4);
  const volatile float magic = (float)((1u << 23) + (1u << 22));
  volatile float s = u + magic;
  return s - magic;
}

// Rust f32::round (half away from zero) of a non-negative value.
float round_half_away(float v) { return roundf(v); }

uint8_t qm_level_law(uint8_t q, int sub) {
  const bool subsampled = sub != 0;
  const float hi = 48.0f, lo = 128.0f;
  const float qi = (float)q;
  if (qi <= 20.0f) return subsampled ? 8 : 15;
  if (qi <= hi) {
    const float top = subsampled ? 8.0f : 15.0f;
    volatile float t = (8.0f - top) * (qi - 20.0f);
    t = t / (hi - 20.0f);
    return (uint8_t)fast_round(top + t);
  }
  if (qi >= lo) return 0;
  volatile float t = 8.0f * (lo - qi);
  t = t / (lo - hi);
  return (uint8_t)fast_round(t);
}

uint8_t qm_chroma_level_law(uint8_t q, int sub) {
  if (sub != 0) return qm_level_law(q, sub);
  const uint8_t top = 2;
  const uint8_t l = qm_level_law(q, sub);
  const uint8_t pinned = top < l ? top : l;
  const float hq = clampf((kQmHqKnee - (float)q) / kQmHqWidth, 0.0f, 1.0f);
  const float t = kTopEase * hq;
  if (t > 0.0f) {
    volatile float v = (15.0f - (float)pinned) * t;
    return (uint8_t)round_half_away((float)pinned + v);
  }
  return pinned;
}

// aom_ssimulacra2_rdmult_weight (src/cost.rs:122-126).
float ssim_rdmult_weight(uint8_t q) {
  int w = ((255 - (int)q) * 3) / 4;
  w = w < 0 ? 0 : (w > 72 ? 72 : w);
  return (float)(w + 128) * (1.0f / 128.0f);
}

// mode_lambda_weight (src/cost.rs:128-148).
float mode_lambda_weight(uint8_t q, int sub) {
  const float scale = sub == 2 ? kMlamScale420 : (sub == 1 ? kMlamScale422 : kMlamScale444);
  const float w = ssim_rdmult_weight(q);
  if (sub == 1 || kModeLambdaLoFull <= kModeLambdaLoFloor) return w * scale;
  volatile float r = ((float)q - kModeLambdaLoFloor) / (kModeLambdaLoFull - kModeLambdaLoFloor);
  const float rc = clampf(r, 0.0f, 1.0f);
  volatile float m = (w - kModeLambdaLoW) * rc;
  volatile float s = kModeLambdaLoW + m;
  return s * scale;
}

// mode_lambda_q (src/cost.rs:286-292): left-to-right f32 products.
float mode_lambda_q(float dc_q, uint8_t bd) {
  const int sh = (bd > 8 ? bd : 8) - 8;
  const float dc_q8 = dc_q / (float)(1u << sh);
  volatile float kf = 0.0015f * dc_q8;
  const float mult = 3.3f + kf;
  volatile float l = kModeAomCalib * 1.0f;
  l = l * dc_q;
  l = l * dc_q;
  return l * mult;
}

// luma_satd_scale (src/partition_rd.rs:30-49).
float luma_satd_scale(uint8_t q, bool subsampled) {
  if (subsampled) return kSatdBase;
  const float qi = (float)q;
  if (qi <= kSatdKneeLo) return kSatdTop;
  if (qi >= kSatdKneeHi) return kSatdBase;
  volatile float d = (kSatdBase - kSatdTop) * (qi - kSatdKneeLo);
  d = d / fmaxf(kSatdKneeHi - kSatdKneeLo, 1.0f);
  return kSatdTop + d;
}

// k_satd (src/partition_rd.rs:54-71).
float k_satd(uint8_t q, bool subsampled) {
  const float qi_[3] = {28.0f, 81.0f, 140.0f};
  const float k444[3] = {35.0f, 21.2f, 18.1f}, k420[3] = {24.5f, 21.3f, 18.2f};
  const float* k = subsampled ? k420 : k444;
  const float qi = (float)q;
  if (qi <= qi_[0]) return k[0];
  if (qi >= qi_[2]) return k[2];
  volatile float d;
  if (qi <= qi_[1]) {
    d = (k[1] - k[0]) * (qi - qi_[0]);
    d = d / (qi_[1] - qi_[0]);
    return k[0] + d;
  }
  d = (k[2] - k[1]) * (qi - qi_[1]);
  d = d / (qi_[2] - qi_[1]);
  return k[1] + d;
}

}  // namespace

extern "C" uint8_t mt_quality_to_q(uint8_t quality) {
  static const uint8_t anchors[14][2] = {{1, 215}, {30, 140}, {40, 116}, {50, 91}, {60, 70}, {70, 53}, {80, 35},
                                         {85, 28}, {90, 17}, {93, 12}, {96, 7}, {98, 5}, {99, 3}, {100, 1}};
  const int q = quality < 1 ? 1 : (quality > 100 ? 100 : quality);
  int l0 = anchors[0][0], q0 = anchors[0][1];
  for (int k = 1; k < 14; ++k) {
    const int l1 = anchors[k][0], q1 = anchors[k][1];
    if (q <= l1) {
      const int t = q - l0;
      const int den = (l1 - l0) > 1 ? (l1 - l0) : 1;
      int v = q0 + (q1 - q0) * t / den;
      v = v < 1 ? 1 : (v > 255 ? 255 : v);
      return (uint8_t)v;
    }
    l0 = l1;
    q0 = q1;
  }
  return 1;
}

extern "C" int mt_qm_levels(uint8_t base_q_idx, int32_t sub, uint8_t* y_level, uint8_t* uv_level) {
  if (sub < 0 || sub > 2 || !y_level || !uv_level) return MT_ERR_INVALID_INPUT;
  *y_level = qm_level_law(base_q_idx, sub);
  *uv_level = qm_chroma_level_law(base_q_idx, sub);
  return MT_OK;
}

extern "C" int mt_rd_lambdas_init(uint8_t base_q_idx, int32_t dc_q, int32_t sub, uint8_t bd, mt_rd_lambdas* out) {
  if (!out || sub < 0 || sub > 2 || dc_q <= 0) return MT_ERR_INVALID_INPUT;
  if (bd != 8) return MT_ERR_UNSUPPORTED;  // hbd_trellis_scale's 10/12-bit ramps are not carried
  const bool subsampled = sub != 0;
  out->mode_lambda = mode_lambda_q((float)dc_q, bd) * mode_lambda_weight(base_q_idx, sub);
  volatile float ld = out->mode_lambda / kPartLambda;
  out->lambda_d = ld;
  out->trellis_lambda0 = kTrellisLambda0;
  out->satd_scale = luma_satd_scale(base_q_idx, subsampled);
  volatile float b = kPartLambda / k_satd(base_q_idx, subsampled);
  out->satd_bridge = b * kProxyLumaScale;
  return MT_OK;
}
