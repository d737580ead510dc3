// The encode configuration of the drop-in boundary: EncodeConfig's fields and
// defaults (src/avif.rs:257-344), its validation (src/avif.rs:577-592
// EncodeConfig::validate, :593-635 validate_dims / validate_quality /
// validate_buf / checked_buffer_size) and the input checks of encode_rgb8
// (src/avif.rs:915-923), with one negative code per EncodeError variant
// (src/err.rs:33-62).  Host code only.
#include <stdint.h>
#include <string.h>

#include "../../include/maroontree_b200.h"

extern "C" int mt_encode_config_default(mt_encode_config* cfg) {
  if (!cfg) return MT_ERR_INVALID_INPUT;
  memset(cfg, 0, sizeof(*cfg));
  cfg->quality = 80;
  cfg->chroma = MT_CHROMA_420;
  cfg->color_present = 1;  // Cicp::srgb_ycbcr (src/color.rs:251-259)
  cfg->primaries = 1;
  cfg->transfer = 13;
  cfg->matrix = 6;
  cfg->full_range = 1;
  cfg->chroma_sample_position = 0;
  cfg->threads = 0;  // all available cores
  cfg->speed = MT_SPEED_SLOW;
  cfg->updating_cdf = 1;
  cfg->adaptive_quant = 1;
  cfg->variance_boost = 1;
  cfg->dark_aq = 1;
  cfg->cdef = 0;
  cfg->wiener = 0;
  cfg->quantization_matrices = 1;
  cfg->screen_content = 1;
  cfg->intrabc = 1;
  cfg->qmatrix_level = -1;
  cfg->alpha_quality = -1;
  cfg->orientation = 1;
  return MT_OK;
}

extern "C" int mt_encode_config_validate(const mt_encode_config* cfg) {
  if (!cfg) return MT_ERR_INVALID_INPUT;
  if (cfg->quality > 100) return MT_ERR_INVALID_QUALITY;
  if (cfg->alpha_quality > 100) return MT_ERR_INVALID_QUALITY;
  if (cfg->qmatrix_level > 15) return MT_ERR_INVALID_QUALITY;
  if (cfg->chroma < MT_CHROMA_420 || cfg->chroma > MT_CHROMA_MONO) return MT_ERR_INVALID_INPUT;
  if (cfg->speed < MT_SPEED_EXTRA_SLOW || cfg->speed > MT_SPEED_FAST) return MT_ERR_INVALID_INPUT;
  if (cfg->orientation < 1 || cfg->orientation > 8) return MT_ERR_INVALID_INPUT;
  if ((cfg->icc_len && !cfg->icc) || (cfg->exif_len && !cfg->exif)) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

extern "C" int mt_validate_rgb8_input(uint32_t width, uint32_t height, size_t rgb_len) {
  // validate_dims (src/avif.rs:593-598): 1..=16383 on both axes
  if (width < 1 || height < 1 || width > 16383 || height > 16383) return MT_ERR_INVALID_DIMENSIONS;
  // checked_buffer_size (src/avif.rs:614-632): w * h * channels must not overflow
  const unsigned __int128 n = (unsigned __int128)width * height * 3;
  if (n > (unsigned __int128)INT64_MAX) return MT_ERR_DIMENSION_TOO_LARGE;
  // PlanarImage::from_interleaved_rgb (src/encoder.rs:171-205): len must be w * h * 3
  if ((unsigned __int128)rgb_len != n) return MT_ERR_INVALID_INPUT;
  return MT_OK;
}

extern "C" int mt_encode_config_effective(const mt_encode_config* cfg, mt_encode_plan* out) {
  int rc = mt_encode_config_validate(cfg);
  if (rc != MT_OK) return rc;
  if (!out) return MT_ERR_INVALID_INPUT;
  memset(out, 0, sizeof(*out));
  out->base_q_idx = mt_quality_to_q((uint8_t)cfg->quality);
  const int sub = cfg->chroma == MT_CHROMA_420 ? 2 : (cfg->chroma == MT_CHROMA_422 ? 1 : 0);
  out->sub = sub;
  // EncodeConfig::vb (src/avif.rs:543-575): QM levels from the laws, a forced
  // uniform level, or flat (15) without matrices.
  if (!cfg->quantization_matrices) {
    out->qm_y = out->qm_u = out->qm_v = 15;
  } else if (cfg->qmatrix_level >= 0) {
    out->qm_y = out->qm_u = out->qm_v = (uint8_t)cfg->qmatrix_level;
  } else {
    uint8_t y = 15, uv = 15;
    mt_qm_levels(out->base_q_idx, sub, &y, &uv);
    out->qm_y = y;
    out->qm_u = out->qm_v = uv;
  }
  // cdef_enabled (src/avif.rs:449-451): Slow and ExtraSlow force CDEF on.
  out->cdef = cfg->cdef || cfg->speed == MT_SPEED_SLOW || cfg->speed == MT_SPEED_EXTRA_SLOW;
  out->aq = cfg->adaptive_quant != 0;
  out->variance_boost = cfg->variance_boost != 0;
  out->dark_aq = cfg->dark_aq != 0;
  return MT_OK;
}
