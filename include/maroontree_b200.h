/*
 * maroontree_b200 — C ABI of the B200 intra rate-distortion core.
 *
 * These entry points are what a host encoder's FFI crate binds in place of the
 * reference's CPU kernel dispatch tables.  Every function takes plain pointers
 * and sizes; no torch or CUDA types appear in the signatures.  Device entry
 * points (mt_*_device) take device pointers and a cudaStream_t passed as
 * `void*` (NULL = legacy default stream); host entry points (mt_* without the
 * suffix) take host buffers and do the copies themselves.
 *
 * Reference interfaces replaced (paths inside awxkee/maroontree):
 *   mt_quant_init / mt_quant_init_chroma  src/quant.rs:351-418  Quant::new_with_qm /
 *                                         Quant::new_chroma_with_delta_qm
 *   mt_coef_costs_build                   src/rate.rs:58-80 CoefCostTables::build +
 *                                         src/cost.rs:156-190 cdf_cost_with_table
 *   mt_qcat / mt_coef_cdfs_default        src/coef_q.rs:31-41 qcat, src/coder/cdfs.rs:401-629
 *                                         Cdfs::new (the coefficient slices)
 *   mt_range_encoder_* / mt_cdfs_default  src/odec.rs:35-615 OdEcEncoder, src/coder/cdfs.rs:193-629
 *   mt_pack_tile                          src/coder/wavefront.rs:617-657 pack_wavefront_tile
 *   mt_pack_tile_filtered                 the same, with replay_tile_with_filters folded in
 *   mt_emit_coeffs[_device] / mt_cdf_layout  src/coeffs.rs:34-2520 the square coefficient coders
 *   mt_replay_tile_with_filters           src/coder/tile_encode.rs:404-466 replay_tile_with_filters
 *   mt_sequence_header / mt_frame_header  src/obu.rs:46-771 sequence / frame headers, OBU framing
 *   mt_assemble_frame_obus / mt_av1_stream src/coder/frame_encode.rs:436-525, src/dispatch.rs:239-256
 *   mt_wrap_av1_image                     src/isobmff.rs:210-494 wrap_av1_image, src/avif.rs:676-740
 *   mt_encode_config_* / mt_validate_rgb8_input  src/avif.rs:257-344 EncodeConfig, :577-635, :915-923
 *   mt_quality_to_q / mt_qm_levels /      src/avif.rs:637-666 quality_to_q, src/quant.rs:122-167
 *   mt_rd_lambdas_init                    QM level laws, src/cost.rs + src/partition_rd.rs lambdas
 *   mt_candidate_chain[_device]           the per-candidate chain of the luma mode
 *                                         search, src/coder/partition_search.rs:467-530
 *                                         (predict_nd -> residual_pred -> DctDispatch ->
 *                                         trellis_optimize -> IdctDispatch ->
 *                                         luma_partition_distortion + luma_bits + mode bits
 *                                         -> partition_rd::rd_cost), batched over candidates
 *   mt_fwd_txfm_quant[_device]            src/dct.rs:2416-2950 DctDispatch::*_t
 *   mt_inv_txfm_dequant[_device]          src/idct.rs:90-160 IdctDispatch
 *   mt_trellis_optimize[_device]          src/trellis.rs:944-1030 trellis_optimize
 *   mt_intra_predict[_device]             src/intrapred.rs:322-398 IntraPredDispatch::predict_nd_ad,
 *                                         src/intrapred.rs:1740-1790 dc_pred
 *   mt_rdo_level8[_device]                the batched form of the same chain over a whole
 *                                         partition level: the per-block candidate loops of
 *                                         src/coder/partition_search.rs:467-530 (and the
 *                                         emitter's mode x type trials, e.g. :4320-4390) with
 *                                         their "if cost < best" selection
 */
#ifndef MAROONTREE_B200_H
#define MAROONTREE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (src/err.rs:146-173 EncodeError, one negative code per variant
 * this boundary can raise, plus device failures). */
#define MT_OK 0
#define MT_ERR_INVALID_INPUT (-2)
#define MT_ERR_UNSUPPORTED (-3)
#define MT_ERR_TOO_LARGE (-4)
#define MT_ERR_DEVICE (-10)
#define MT_ERR_ALLOC (-11)
/* The EncodeError variants of the encode boundary (src/err.rs:33-62). */
#define MT_ERR_INVALID_DIMENSIONS (-20)    /* InvalidDimensions: not 1..=16383 */
#define MT_ERR_DIMENSION_TOO_LARGE (-21)   /* DimensionTooLarge: buffer size overflows */
#define MT_ERR_INVALID_QUALITY (-22)       /* InvalidQuality: quality > 100, QM level > 15 */
#define MT_ERR_UNSUPPORTED_CHROMA_FORMAT (-23)
#define MT_ERR_UNSUPPORTED_BIT_DEPTH (-24) /* UnsupportedChromaBitDepth */

/* Intra prediction modes, AV1 numbering (src/intrapred.rs:54-79). */
#define MT_DC_PRED 0
#define MT_V_PRED 1
#define MT_H_PRED 2
#define MT_D45_PRED 3
#define MT_D135_PRED 4
#define MT_D113_PRED 5
#define MT_D157_PRED 6
#define MT_D203_PRED 7
#define MT_D67_PRED 8
#define MT_SMOOTH_PRED 9
#define MT_SMOOTH_V_PRED 10
#define MT_SMOOTH_H_PRED 11
#define MT_PAETH_PRED 12

/* Transform types in the 7-type intra set index order used by the reference
 * (src/cost.rs:100-103: IDTX=0, DCT_DCT=1, V_DCT=2, H_DCT=3, ADST_ADST=4,
 * ADST_DCT=5, DCT_ADST=6).  ADST_DCT = ADST down the columns, DCT along rows. */
#define MT_TX_IDTX 0
#define MT_TX_DCT_DCT 1
#define MT_TX_V_DCT 2
#define MT_TX_H_DCT 3
#define MT_TX_ADST_ADST 4
#define MT_TX_ADST_DCT 5
#define MT_TX_DCT_ADST 6

/* Quantiser state of one plane (src/quant.rs:327-343 Quant). */
typedef struct mt_quant {
  int32_t dc_q, ac_q;           /* dequant steps */
  int32_t q_mult_dc, q_mult_ac; /* round(65536 / step) */
  int32_t rmin, rmax, cmin, cmax, cf_max; /* inverse-transform clips */
  int32_t qm_level;             /* 0..14, 15 = flat */
  int32_t qm_chroma;
  int32_t qidx;
} mt_quant;

/* One (transform class, plane) slice of an immutable decision CDF snapshot
 * (src/coder/cdfs.rs Cdfs fields), AV1 inverse-CDF form: entry s is
 * 32768 * P(symbol > s); the last entry of each CDF is 0. */
typedef struct mt_coef_cdfs {
  uint16_t txb_skip[13][2];
  uint16_t base_tok[42][4];
  uint16_t br_tok[21][4];
  uint16_t eob_base[4][3];
  uint16_t eob_hi[11][2];
  uint16_t eob_bin[11];   /* eob_pt CDF of this size; unused tail = 0 */
  uint16_t dc_sign[3][2];
  uint16_t txtp[13][16];  /* intra tx-type CDF per y mode; unused tail = 0 */
  uint16_t eob_bin_1d[11]; /* eob_pt CDF of the 1-D classes (V_DCT / H_DCT) of this size
                            * (eob_bin_16_l1d / eob_bin_64_l1d); unused tail = 0 */
} mt_coef_cdfs;

/* Bit costs of the same slice, each entry cdf_cost_with_table(cdf, s)
 * (src/cost.rs:184-190) and br_cum the cumulative base-range ladder
 * (src/cost.rs:214-241).  Built on the host by mt_coef_costs_build. */
typedef struct mt_coef_costs {
  float txb_skip[13][2];
  float base_tok[42][4];
  float br_cum[21][13];
  float eob_base[4][3];
  float eob_hi[11][2];
  float eob_bin[11];
  float dc_sign[3][2];
  float txtp[13][16];
  float eob_bin_1d[11];
} mt_coef_costs;

/* One candidate of the batched chain: block position, intra mode (+ angle
 * delta), transform type and neighbour availability. */
typedef struct mt_candidate {
  uint16_t px, py;       /* luma sample position of the block */
  uint8_t mode;          /* MT_*_PRED */
  int8_t angle_delta;    /* -3..3, directional modes only */
  uint8_t tx_type;       /* MT_TX_* */
  uint8_t flags;         /* bit0 have_tr, bit1 have_bl, bit2 filter_type, bit3 no trellis */
  uint8_t dcs_ctx;       /* dc_sign context 0..2 */
  uint8_t skip_ctx;      /* txb_skip context 0..12 */
  uint16_t reserved;
  float mode_bits;       /* LossyTile::mode_bits(px, py, mode) of the caller */
  float extra_bits;      /* more signalling bits, added after mode_bits: bits = (luma_bits +
                          * mode_bits) + extra_bits; the angle-delta symbol of the proxy's delta
                          * pass, cdf_cost(angle_delta cdf of the mode, delta + 3)
                          * (src/coder/partition_search.rs:576-578); 0 adds nothing */
} mt_candidate;

#define MT_CAND_HAVE_TR 1u
#define MT_CAND_HAVE_BL 2u
#define MT_CAND_FILTER_TYPE 4u
/* Price the levels as quantised, without trellis_optimize: the reference's
 * 4x4 IDTX trial in the SPLIT4 pricing (src/coder/lossy_state.rs:2229-2236). */
#define MT_CAND_NO_TRELLIS 8u

/* Batch-wide parameters of the chain. */
typedef struct mt_chain_params {
  int32_t tx_size;        /* square luma transform size: 8, or 4 / 16 for the 4x4 / 16x16 levels */
  int32_t bd;             /* bit depth (8) */
  int32_t frame_w, frame_h; /* padded plane size, also the prediction frame bounds */
  int32_t stride;         /* samples per row of src and recon */
  float trellis_lambda0;  /* lambda0 * prdo of trellis_optimize; <= 0 disables */
  float mode_lambda;      /* mlam * prdo, the rd_cost lambda */
  float satd_scale;       /* partition_rd::luma_satd_scale(base_q, subsampled) */
  float satd_bridge;      /* K_PART_LAMBDA / k_satd * proxy_luma_scale; 0 = bridge off */
  int32_t use_skip_bits;  /* 1: skip_bits below replace the txb_skip CDF cost */
  float skip_bits[2];     /* (all_zero = 1, all_zero = 0) */
  int32_t vis_w, vis_h;   /* displayed luma size; samples past it carry no distortion (the
                           * reference's SrcBlock masking, src/rd_sse.rs:61-167, :630-655);
                           * 0 = frame_w / frame_h */
} mt_chain_params;

/* eob value of a candidate the kernel rejected (block outside the frame, or a
 * mode / type / context index out of range); its other outputs are zero. */
#define MT_EOB_INVALID (-2)

/* Per-candidate outputs. */
typedef struct mt_candidate_result {
  float distortion;       /* luma_partition_distortion */
  float bits;             /* luma_bits + mode_bits */
  float cost;             /* rd_cost(distortion, mode_lambda, bits) */
  uint32_t satd;          /* raw SATD of the reconstruction */
  int32_t eob;            /* last nonzero scan index after trellis, -1 if none */
  uint32_t reserved[3];
} mt_candidate_result;

/* One block of an RDO level (8x8 for mt_rdo_level8*, 4x4 for mt_rdo_level4*):
 * position, neighbour availability, contexts and the caller's
 * mode-signalling bits for each of the 13 luma modes. */
typedef struct mt_block8 {
  uint16_t px, py;
  uint8_t flags;          /* MT_CAND_* bits */
  uint8_t dcs_ctx;        /* dc_sign context 0..2 */
  uint8_t skip_ctx;       /* txb_skip context 0..12 */
  uint8_t reserved;
  float mode_bits[13];    /* LossyTile::mode_bits(px, py, m) for m = 0..12 */
} mt_block8;

/* One (mode, angle delta, transform type) candidate of every block. */
typedef struct mt_combo {
  uint8_t mode;
  int8_t angle_delta;
  uint8_t tx_type;
  uint8_t flags;          /* MT_COMBO_NO_TRELLIS */
  float bits;             /* extra_bits of this combo's candidates (the angle-delta symbol) */
} mt_combo;
#define MT_COMBO_NO_TRELLIS 1u

/* Per-block winner of a level: the lowest rd cost over the combos, ties to
 * the earlier combo (the reference's strict-< scan in candidate order). */
typedef struct mt_block_best {
  int32_t combo;          /* index into the combo list, -1 if none evaluated */
  float cost, distortion, bits;
  uint32_t satd;
  int32_t eob;
  uint32_t reserved[2];
} mt_block_best;

/* ---- host-side helpers ---------------------------------------------------- */

/* Quant::new_with_qm(base_q_idx, bd, qm_level) for 8-bit luma. */
int mt_quant_init(uint8_t base_q_idx, uint8_t bd, uint8_t qm_level, mt_quant* out);
/* Quant::new_chroma_with_delta_qm(base_q_idx, dc_delta, ac_delta, bd, qm_level). */
int mt_quant_init_chroma(uint8_t base_q_idx, int32_t dc_delta, int32_t ac_delta, uint8_t bd,
                         uint8_t qm_level, mt_quant* out);
/* Inverse QM weight row for a w x h transform (qm_row, src/quant.rs:83-89), or
 * NULL when the level is flat.  Points into a static table. */
const uint8_t* mt_qm_row(int32_t qm_level, int32_t chroma, int32_t w, int32_t h);
/* Default diagonal scan of a square transform of size n (4, 8, 16, 32). */
const uint16_t* mt_default_scan(int32_t n);
/* CoefCostTables-style bit costs of one CDF slice. */
int mt_coef_costs_build(const mt_coef_cdfs* cdfs, mt_coef_costs* out);
/* Decision lambdas of a frame (8-bit): the luma proxy's and the emitters'
 * mode lambda mlam = mode_lambda_q(dc_q) x tune_weight (src/cost.rs:128-148,
 * :286-292, src/coder/lossy_state.rs:1769-1771, :1864-1871), the decision
 * lambda lambda_d = mlam / K_PART_LAMBDA (:1787-1789), the trellis lambda0
 * (src/cost.rs:93, :110-112), and the SATD proxy's scale and bridge
 * (src/partition_rd.rs:30-71, src/coder/lossy_state.rs:2396-2408:
 * luma_satd_scale, K_PART_LAMBDA / k_satd x proxy_luma_scale). */
typedef struct mt_rd_lambdas {
  float mode_lambda;
  float lambda_d;
  float trellis_lambda0;
  float satd_scale;
  float satd_bridge;
} mt_rd_lambdas;

/* quality 0..100 -> base qindex (src/avif.rs:637-666 quality_to_q). */
uint8_t mt_quality_to_q(uint8_t quality);
/* Default quantisation-matrix levels of a base qindex: qm_level_law (luma) and
 * qm_chroma_level_law (src/quant.rs:122-167); sub 0 = 4:4:4, 1 = 4:2:2,
 * 2 = 4:2:0. */
int mt_qm_levels(uint8_t base_q_idx, int32_t sub, uint8_t* y_level, uint8_t* uv_level);
/* The lambdas above for base qindex base_q_idx (the frame's; the SATD laws
 * read the AQ base qindex, equal to it without AQ), the DC quantiser step dc_q
 * of the block's qindex, chroma subsampling sub (0 4:4:4, 1 4:2:2, 2 4:2:0)
 * and bit depth bd (8 only: MT_ERR_UNSUPPORTED otherwise). */
int mt_rd_lambdas_init(uint8_t base_q_idx, int32_t dc_q, int32_t sub, uint8_t bd, mt_rd_lambdas* out);
/* Coefficient CDF q context of a base qindex: qcat (src/coef_q.rs:31-41). */
int mt_qcat(int32_t base_q_idx);
/* The (transform class, plane) slice of the default decision snapshot
 * Cdfs::new(qctx) (src/coder/cdfs.rs:401-629) for a tx_w x tx_h transform
 * (4..64, at most 1:4): skip / base / br / eob_base / eob_hi rows of the AV1
 * class (the mean of the square sizes below and above), dc_sign of the plane,
 * the eob_pt CDF of the transform's coefficient count (and the luma 1-D form
 * at 16 / 64 / 128 coefficients), and for luma transforms without a 32-point
 * side the intra tx-type CDFs per y mode (INTRA1 at TX_4X4 / TX_8X8, INTRA2 at
 * TX_16X16).  plane: 0 luma, 1 chroma (no chroma 64-point class). */
int mt_coef_cdfs_default(int32_t qctx, int32_t tx_w, int32_t tx_h, int32_t plane, mt_coef_cdfs* out);

/* ---- batched kernels ------------------------------------------------------ */

/* The candidate chain over n candidates.  src/recon: u16 planes of
 * frame_h x stride samples.  qm_row: inverse QM weights of the transform size
 * (tx_size^2 bytes, column-major rc = x*h + y) or NULL when flat.
 * levels_out (optional, n * tx_size^2 int32): final quantised levels,
 * column-major.  recon_out (optional, n * tx_size^2 int32): reconstructed
 * samples (prediction + inverse residual, clamped), row-major. */
int mt_candidate_chain(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm,
                       const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                       const mt_candidate* cands, int32_t n, mt_candidate_result* results,
                       int32_t* levels_out, int32_t* recon_out);
/* Device form.  d_scratch (optional, mt_candidate_chain_scratch_bytes(n)
 * bytes) lets the launch bucket the candidates by code path first; results
 * are identical with or without it. */
int mt_candidate_chain_device(const uint16_t* d_src, const uint16_t* d_recon,
                              const mt_chain_params* prm, const mt_quant* quant,
                              const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                              const mt_candidate* d_cands, int32_t n,
                              mt_candidate_result* d_results, int32_t* d_levels_out,
                              int32_t* d_recon_out, void* d_scratch, void* stream);
size_t mt_candidate_chain_scratch_bytes(int32_t n);

/* One batched RDO level: every combo of every block (ncombos * nblocks chain
 * evaluations in one launch) and the per-block best.  Host form: host
 * buffers in and out; results_out (optional) receives all
 * ncombos * nblocks results, combo-major (index combo * nblocks + block).
 * Consecutive combos with the same (mode, angle delta) share one prediction,
 * so list each mode's transform types together.  At most MT_LEVEL_MAX_COMBOS
 * combos (13 modes x 7 deltas x 16 types is 1456), else MT_ERR_TOO_LARGE. */
#define MT_LEVEL_MAX_COMBOS 2048
int mt_rdo_level8(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm,
                  const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                  const mt_block8* blocks, int32_t nblocks, const mt_combo* combos,
                  int32_t ncombos, mt_block_best* best_out, mt_candidate_result* results_out);
/* Device form: d_results (ncombos * nblocks records) and d_scratch
 * (mt_rdo_level8_scratch_bytes: the per-block argmin keys, the run table and
 * one 64-byte prediction per (mode, delta, block)) are caller-provided;
 * d_best receives the winners. */
int mt_rdo_level8_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos,
                         int32_t ncombos, mt_block_best* d_best, mt_candidate_result* d_results,
                         void* d_scratch, void* stream);
size_t mt_rdo_level8_scratch_bytes(int32_t nblocks, int32_t ncombos);

/* The same batched level for 4x4 luma blocks (prm->tx_size = 4): the per-4x4
 * chain the reference's SPLIT4 pricing runs (src/coder/lossy_state.rs:
 * 2148-2290: predict_nd from the pre-block reconstruction, dct4x4_t /
 * adst4x4_t / idtx4x4_t, trellis_optimize over SCAN_4X4 -- skipped for combos
 * flagged MT_COMBO_NO_TRELLIS, as its IDTX trial does --, the 4x4 inverse,
 * luma_partition_distortion and luma_bits over the TX_4X4 class).  Blocks are
 * mt_block8 records on the 4-sample grid; qm_row is the 16-entry 4x4 row;
 * costs the TX_4X4 luma slice; d_scratch is mt_rdo_level4_scratch_bytes
 * (the per-block argmin keys). */
int mt_rdo_level4(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm,
                  const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                  const mt_block8* blocks, int32_t nblocks, const mt_combo* combos,
                  int32_t ncombos, mt_block_best* best_out, mt_candidate_result* results_out);
int mt_rdo_level4_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos,
                         int32_t ncombos, mt_block_best* d_best, mt_candidate_result* d_results,
                         void* d_scratch, void* stream);
size_t mt_rdo_level4_scratch_bytes(int32_t nblocks, int32_t ncombos);

/* The batched 16x16 level: the 16x16 arm of rd_cost_square
 * (src/coder/partition_search.rs:620-673 and its proxy_ad / ADST refinement
 * passes) for every (block, combo) pair -- predict_nd (DC via dc_pred_16x16)
 * -> dct16x16_t / adst16x16_t / adstdct16x16_t / dctadst16x16_t (+QM) or
 * idtx16x16_t -> trellis_optimize over SCAN_16X16 -> the 16x16 inverse ->
 * luma_partition_distortion -> TX_16X16 luma_bits + mode bits (+ the combo's
 * bits) -> rd_cost.  prm->tx_size = 16; blocks are 16x16 at multiples of 16
 * (an MT_CAND_* flags byte per block as for 8x8); qm_row is the 256-entry
 * TX_16X16 row of the level (NULL: flat); costs is the TX_16X16 slice.
 * Transform types DCT_DCT, ADST_ADST, ADST_DCT, DCT_ADST, IDTX (V/H_DCT give
 * MT_EOB_INVALID). */
int mt_rdo_level16(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_block8* blocks, int32_t nblocks,
                   const mt_combo* combos, int32_t ncombos, mt_block_best* best_out,
                   mt_candidate_result* results_out);
int mt_rdo_level16_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos, int32_t ncombos,
                          mt_block_best* d_best, mt_candidate_result* d_results, void* d_scratch, void* stream);
size_t mt_rdo_level16_scratch_bytes(int32_t nblocks, int32_t ncombos);

/* Allocation-free form of mt_rdo_level8_device.  No counterpart in the
 * reference: it exists for callers that cannot give this library device
 * memory on demand (a fixed GPU-memory budget owned by another framework's
 * pool, or a real-time thread that must not call the driver's allocator).
 * The caller passes only inputs and the per-block output; the call allocates
 * nothing and needs no working storage: its per-block argmin keys live in a
 * file-scope device array of MT_NOALLOC_MAX_BLOCKS entries (1 MiB held on
 * every device that loads the library until exit), and each block's winner is
 * re-evaluated to fill d_best, which equals mt_rdo_level8_device's d_best.
 * Its input checks and error codes are mt_rdo_level8_device's; beyond them,
 * more than MT_NOALLOC_MAX_BLOCKS blocks returns MT_ERR_TOO_LARGE.  Every call
 * looks up that array's device address with the device current (the first
 * call on a device may load the module, so make it before any stream
 * capture).  All calls share the array: calls that overlap on the GPU race
 * and must not be issued. */
#define MT_NOALLOC_MAX_BLOCKS 131072
int mt_rdo_level8_device_noalloc(const uint16_t* d_src, const uint16_t* d_recon,
                                 const mt_chain_params* prm, const mt_quant* quant,
                                 const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                                 const mt_block8* d_blocks, int32_t nblocks, const mt_combo* d_combos,
                                 int32_t ncombos, mt_block_best* d_best, void* stream);

/* ---- The proxy's mode beam ----
 * proxy_mode_beam's ranking (src/coder/partition_search.rs:187-238): for every
 * N x N block (N = prm->tx_size: 4, 8 or 16), the 11 nd_modes (DC, V, H, D45,
 * D135, D113, D157, D203, D67, SMOOTH, PAETH; src/intrapred.rs:1712-1729)
 * predicted at angle delta 0 from the reconstruction, each scored by
 * satd_sad_proxy (SAD + SATD/4 over 4x4 Hadamard tiles of src - pred,
 * src/rd_sse.rs:559-589, :1143-1176; samples past the displayed frame count as
 * the prediction), sorted by (score, mode).  The caller keeps the first
 * proxy_mode_beam_len of them (Slow 4:4:4 keeps {DC, PAETH} without ranking).
 * scores / modes: nblocks x MT_BEAM_MODES, ascending.  A block outside the
 * frame gets scores of all ones and mode 255. */
#define MT_BEAM_MODES 11
int mt_mode_beam_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_chain_params* prm,
                        const mt_block8* d_blocks, int32_t nblocks, uint64_t* d_scores, uint8_t* d_modes,
                        void* stream);
/* Host-buffer form of mt_mode_beam_device (scores may be NULL). */
int mt_mode_beam(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm, const mt_block8* blocks,
                 int32_t nblocks, uint64_t* scores, uint8_t* modes);

/* ---- Decision distortion of reconstructed blocks ----
 * sse_recon (src/rd_sse.rs:449-475) of n w x h luma blocks (w, h multiples of
 * 4 up to 64): the error src - clamp(pred + resid, 0, 2^bd - 1) over the part
 * of each block inside the displayed plane (vis_w x vis_h samples; a block
 * wholly outside scores 0).  wsse_scale 0: the plain SSE; > 0: the reference's
 * weighted decision distortion round(weighted_sse(err) * wsse_scale), half away
 * from zero, err zero-padded to whole 4x4 tiles of the displayed part
 * (src/rd_sse.rs:244-271; the 4x4-DCT weighted SSE in the pinned AVX2 order,
 * src/avx/rd.rs:767-848).  pos: (px, py) u16 pairs; pred / resid: n blocks of
 * w*h int32 packed row-major (resid may be NULL: zero). */
int mt_sse_recon_device(const uint16_t* d_src, int32_t stride, int32_t vis_w, int32_t vis_h, int32_t bd,
                        const uint16_t* d_pos, const int32_t* d_pred, const int32_t* d_resid, int32_t n, int32_t w,
                        int32_t h, float wsse_scale, int64_t* d_out, void* stream);
/* Host-buffer form (the source plane is stride x plane_h samples). */
int mt_sse_recon(const uint16_t* src, int32_t stride, int32_t plane_h, int32_t vis_w, int32_t vis_h, int32_t bd,
                 const uint16_t* pos, const int32_t* pred, const int32_t* resid, int32_t n, int32_t w, int32_t h,
                 float wsse_scale, int64_t* out);

/* ---- Context-aware trellis ----
 * trellis_optimize_ctx (src/trellis.rs:55-942) of n TX_8X8 luma blocks
 * (class 1, plane 0) against the decision-CDF costs: the per-coefficient
 * RD-best level in reverse scan order with the real base/range token costs,
 * then the EOB position by the eob_pt / eob_base costs, with quantisation-
 * matrix weighting (w/32, squared from QM level 5) and the tile's band tilt
 * (distortion of coefficients with |target| < 2 divided by
 * 1 + tilt * index / 64).  Shipped tuning: no dead zone, the DC-only terminal
 * in context 0, skip priced at 1 bit.  d_levels (column-major int32, 64 per
 * block) are updated in place; d_dcs_ctx: the dc_sign context of each block.
 * lambda0 <= 0 leaves the levels unchanged. */
int mt_trellis_optimize_ctx_device(int32_t* d_levels, const float* d_targets, const uint8_t* d_dcs_ctx, int32_t n,
                                   const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                                   float lambda0, float band_tilt, void* stream);

/* ---- The 16x16 leaf's TX_8X8 split trial ----
 * split16_luma_try (src/coder/partition_search.rs:4235-4428) of a batch of
 * (16x16 block, luma mode) jobs: the four 8x8 quadrants in raster order, each
 * predicted from the reconstruction with the quadrants already trial-coded
 * (edge flags (py > 0, px > 0), (have_tr, 0), (1, have_bl), (0, 0)), DCT_DCT
 * with trellis_optimize_ctx, the dav1d inverse and sse_recon; with tx_search
 * the 4:4:4 type trials ADST_ADST, ADST_DCT, DCT_ADST (trellised), IDTX,
 * V_DCT, H_DCT (not trellised), each gated on its SSE (the ADST family within
 * tx_guard of the DCT's) and priced only when the gate passes: the 2-D types by
 * real_block_bits_bounded (src/rate.rs:149-291) in the quadrant's progressive
 * txb_skip / dc_sign contexts, V/H by luma_bits_1d_8x8 (src/coder/
 * lossy_state.rs:876-1008); the lowest rd_cost_i64 wins, ties to the earlier
 * type.  The winner's coefficient result context (lossy_state.rs:630-648)
 * feeds the next quadrant's contexts, its reconstruction the next quadrant's
 * prediction. */
typedef struct mt_split16_params {
  int32_t frame_w, frame_h; /* padded plane size, also the prediction frame bounds */
  int32_t stride;           /* samples per row of src and recon */
  int32_t bd;               /* bit depth (8) */
  int32_t vis_w, vis_h;     /* displayed luma size; 0 = frame_w / frame_h */
  float trellis_lambda0;    /* lam of trellis_optimize_ctx; <= 0 disables */
  float rd_lambda;          /* rd_lam of the type gates and the bits bound (the caller's mlam) */
  float band_tilt;          /* Cdfs::band_tilt of the tile (src/coder/lossy_state.rs:351-359) */
  float wsse_scale;         /* sse_recon: 0 plain SSE, > 0 the scaled weighted SSE */
  int32_t tx_search;        /* 1: the 4:4:4 type search; 0: DCT_DCT only (4:2:0, 4:2:2, mono) */
  int32_t tx_guard_shift;   /* Tuning::tx_guard_shift (4) / tx_guard_shift_444 (5); >= 63: no slack */
  int32_t use_skip_bits;    /* 1: skip_bits replace the txb_skip CDF cost of the 2-D walks */
  float skip_bits[13][2];   /* skip_price of class TX_8X8 per context: (all_zero = 1, all_zero = 0) */
} mt_split16_params;

typedef struct mt_split16_job {
  uint16_t px, py;          /* 16x16 block origin (luma samples) */
  uint8_t mode;             /* MT_*_PRED */
  int8_t angle_delta;       /* -3..3, directional modes only */
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL / FILTER_TYPE of the 16x16 block */
  uint8_t reserved;
  uint8_t a_coef[4];        /* above coefficient contexts of the block's four 4-sample columns */
  uint8_t l_coef[4];        /* left coefficient contexts of its four 4-sample rows */
} mt_split16_job;

typedef struct mt_split16_result {
  int64_t sse;              /* sum of the quadrants' sse_recon */
  float bits;               /* sum of the quadrants' coefficient bits, quadrant order */
  uint8_t tx_types[4];      /* winning MT_TX_* per quadrant; all 255 for a rejected job */
} mt_split16_result;

/* Device form.  d_cf (optional): n x 256 int32, quadrant q's levels at
 * [q*64, q*64 + 64) column-major; d_rec (optional): n x 256 u16, the 16x16
 * trial reconstruction row-major.  A job outside the frame, or with a mode /
 * delta out of range, is rejected (tx_types 255, sse 0, bits 0). */
int mt_split16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                           const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                           const mt_split16_job* d_jobs, int32_t n, mt_split16_result* d_results, int32_t* d_cf,
                           uint16_t* d_rec, void* stream);
/* ---- The 16x16 leaf's depth-2 trial: sixteen TX_4X4 ----
 * split16_depth2_try (src/coder/partition_search.rs:4524-4642): the sixteen
 * 4x4 transform blocks of each job in raster order, each predicted from the
 * reconstruction with the blocks already trial-coded (edge flags: top row
 * (py > 0 && (i < 3 || have_tr)), others (i < 3); left column
 * (px > 0 && (j < 3 || have_bl)), others none), DCT_DCT with
 * trellis_optimize, then ADST_ADST (trellised), IDTX, V_DCT, H_DCT, each taken
 * when its sse_recon is within tx_guard of the DCT's and its rd cost is lower
 * (ties keep the earlier type).  The 2-D types are priced by
 * real_block_bits_bounded in txb_skip context 0 and the dc_sign context of the
 * job's own above / left bytes for that column and row (the trial leaves the
 * coefficient contexts alone), V / H by luma_bits_1d_4x4.  costs / qm_row:
 * the TX_4X4 class slice and 4x4 row.  Of mt_split16_params, skip_bits[0]
 * is the TX_4X4 class's context-0 pair (all_zero = 1, all_zero = 0) when
 * use_skip_bits is set; tx_search and band_tilt are not used (this trial
 * always tries its four types, with the plain trellis). */
typedef struct mt_split16_d2_result {
  int64_t sse;              /* sum of the sixteen sse_recon */
  float bits;               /* sum of their coefficient bits, raster order */
  uint8_t tx_types[16];     /* winning MT_TX_* per 4x4 in raster order; all 255 for a rejected job */
  uint8_t reserved[4];
} mt_split16_d2_result;

/* d_cf (optional): n x 256 int32, 4x4 block t's levels at [t*16, t*16 + 16)
 * column-major; d_rec (optional): n x 256 u16, the trial reconstruction
 * row-major.  Rejected jobs as in mt_split16_luma_device. */
int mt_split16_depth2_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                             const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                             const mt_split16_job* d_jobs, int32_t n, mt_split16_d2_result* d_results,
                             int32_t* d_cf, uint16_t* d_rec, void* stream);
int mt_split16_depth2(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                      const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                      mt_split16_d2_result* results, int32_t* cf_out, uint16_t* rec_out);

/* ---- The 8x8 leaf's TX_4X4 split trial ----
 * split4tx_try (src/coder/block8.rs:157-286): the four 4x4 transform blocks of
 * an 8x8 job in raster order (edge flags (py > 0, px > 0), (have_tr, 0),
 * (1, have_bl), (0, 0)), DCT_DCT with trellis_optimize, then ADST_ADST
 * (trellised) and IDTX, each taken when its sse_recon is within tx_guard of
 * the DCT's and its rd cost is lower, priced like the depth-2 trial
 * (real_block_bits_bounded in txb_skip context 0 and the dc_sign context of
 * the job's bytes a_coef[i] / l_coef[j], i, j in 0..1).  The job's px, py
 * address an 8x8 block; costs / qm_row: the TX_4X4 slice and 4x4 row; the
 * params as for mt_split16_depth2.  d_cf (optional): n x 64 int32, 4x4 block
 * q's levels at [q*16, q*16 + 16); d_rec (optional): n x 64 u16. */
int mt_split4tx_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                       const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                       const mt_split16_job* d_jobs, int32_t n, mt_split16_result* d_results, int32_t* d_cf,
                       uint16_t* d_rec, void* stream);
int mt_split4tx(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out);

/* ---- The 8x8 leaf's luma search (pick_block8, src/coder/block8.rs:689-1420) ----
 * mt_leaf8_luma: the Slow mode loop's candidates -- each (block, mode, delta)
 * predicted from the reconstruction, DCT_DCT (+ QM) with the per-candidate
 * trellis_optimize_ctx in the block's dc_sign context, the dav1d inverse,
 * sse_recon, luma_bits in txb_skip context 0, and
 * cost = rd_cost_i64(sse, rd_lambda, bits + syntax_bits) (block8.rs:738-808;
 * syntax_bits is the caller's luma_intra_syntax_bits).  trellis_lambda0 <= 0
 * prices the plain quantised levels (the Medium / Fast loop).
 * mt_leaf8_tx_refine: the winner's transform-type refinement
 * (block8.rs:1183-1404): the DCT baseline as above, then ADST_ADST (taken when
 * within tx_guard of the DCT's SSE and below the DCT's rd cost), ADST_DCT and
 * DCT_ADST (within tx_guard of the DCT's SSE, below the current best), IDTX
 * (within tx_guard of the current best's SSE, unbounded rate), and unless
 * tx_search is 0 (4:2:0) V_DCT and H_DCT (at most the current best's SSE);
 * the ADST family trellised, priced by the bounded 2-D walk, V / H by the 1-D
 * walk.  Params as mt_split16_params with skip_bits[0] the TX_8X8 class's
 * context-0 pair; band_tilt the tile's.  Rejected jobs (outside the frame, a
 * bad mode / delta / context) get sse 0, bits and cost +inf, tx_type 255. */
typedef struct mt_leaf8_job {
  uint16_t px, py;          /* 8x8 block origin */
  uint8_t mode;             /* MT_*_PRED */
  int8_t angle_delta;
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL / FILTER_TYPE */
  uint8_t dcs_ctx;          /* dc_sign_ctx of the block, 0..2 */
  float syntax_bits;        /* luma_intra_syntax_bits(px, py, 8, 8, mode, delta) */
} mt_leaf8_job;
typedef struct mt_leaf8_result {
  int64_t sse;              /* sse_recon of the chosen levels */
  float bits;               /* coefficient bits (without the syntax bits) */
  float cost;               /* mt_leaf8_luma: rd_cost_i64(sse, rd_lambda, bits + syntax_bits);
                             * mt_leaf8_tx_refine: rd_cost_i64(sse, rd_lambda, bits) */
  uint8_t tx_type;          /* MT_TX_* (DCT_DCT from mt_leaf8_luma) */
  uint8_t reserved[7];
} mt_leaf8_result;
/* d_cf (optional): n x 64 int32 levels column-major; d_rec (optional): n x 64
 * u16 reconstruction. */
int mt_leaf8_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                         const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                         const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                         uint16_t* d_rec, void* stream);
int mt_leaf8_tx_refine_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                              const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                              const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                              uint16_t* d_rec, void* stream);
/* The 16x16 leaf (pick_luma16, src/coder/partition_search.rs): the mode
 * loop's candidates (:4802-4880) as mt_leaf8_luma_device at 16x16 -- DCT_DCT
 * (+ QM) with trellis_optimize_ctx of class TX_16X16, sse_recon, luma_bits in
 * txb_skip context 0 with the txtp16 symbol -- and the winner's refinement
 * (:5252-5474): ADST_ADST (within tx_guard of the DCT's SSE, below the DCT's
 * rd cost, bounded rate), ADST_DCT and DCT_ADST (within tx_guard of the DCT's
 * SSE, below the current best, unbounded rate), IDTX (within tx_guard of the
 * current best's SSE); no V / H.  Jobs address 16x16 blocks; the costs / qm
 * row are the TX_16X16 slice and 16x16 row; d_cf / d_rec are n x 256. */
int mt_leaf16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                          uint16_t* d_rec, void* stream);
int mt_leaf16_tx_refine_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                               const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                               const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                               uint16_t* d_rec, void* stream);
/* Host-buffer form; refine = 0: the candidates, 1: the refinement. */
int mt_leaf16(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);
/* Host-buffer forms; refine = 0: mt_leaf8_luma, 1: mt_leaf8_tx_refine. */
int mt_leaf8(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
             const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
             mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);
/* The 32x32 leaf (pick_luma32, src/coder/block32.rs:728-836): the mode loop's
 * candidates as mt_leaf8_luma_device at 32x32 -- the prediction at 32x32, the
 * TX_32X32 DCT_DCT (the only intra type of that size; the reference's 64-bit
 * rounded forward transform, src/dct.rs:589-736) with the 32x32 QM,
 * trellis_optimize_ctx of class TX_32X32, the dav1d inverse with the TX_32X32
 * dequantisation (src/idct.rs:2130-2320), sse_recon, luma_bits in txb_skip
 * context 0 with no tx-type symbol, and
 * cost = rd_cost_i64(sse, rd_lambda, bits + syntax_bits).  Jobs address 32x32
 * blocks; the costs / qm row are the TX_32X32 slice and 32x32 row (1024
 * weights); skip_bits[0] the TX_32X32 class's context-0 pair; d_cf / d_rec
 * are n x 1024. */
int mt_leaf32_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_leaf8_job* d_jobs, int32_t n, mt_leaf8_result* d_results, int32_t* d_cf,
                          uint16_t* d_rec, void* stream);
/* Host-buffer form of mt_leaf32_luma_device. */
int mt_leaf32(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
              const uint8_t* qm_row, const mt_coef_costs* costs, const mt_leaf8_job* jobs, int32_t n,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);

/* The 64x64 leaf's four-TX_32X32 leg (rd_pick_luma64's candidate loop,
 * src/coder/block64.rs:1906-1958; the shipped tuning leaves TX_64X64 off): for
 * each (64x64 block, mode, delta) the four quadrants in raster order, each
 * predicted at 32x32 from the block's running reconstruction with the
 * per-transform edge flags (quad_edges, :2731-2745: the first from the rows /
 * columns around the block, the second with the block's top-right flag, the
 * third with top-right and the block's bottom-left flag, the fourth with
 * neither), TX_32X32 DCT_DCT with the QM and trellis_optimize_ctx in the
 * quadrant's dc_sign context, the inverse, the decision distortion sse_recon
 * x K_PART_LAMBDA (luma64_wsse, src/coder/lossy_state.rs:2363-2382) and
 * luma_bits in txb_skip context 0; the quadrant's reconstruction is written
 * back before the next.  total = rd_lambda x mode_bits (+ rd_lambda x
 * delta_bits for a directional mode) + the quadrants' sse x 2.775 +
 * rd_lambda x bits, f32 in that order.  Params as for the 32x32 leaf
 * (trellis_lambda0: the trellis lambda with the perceptual scale;
 * rd_lambda: mlam x prdo).  Rejected jobs (outside the frame, a bad mode /
 * delta / context) get total and bits +inf, sse 0. */
typedef struct mt_quad32_job {
  uint16_t px, py;          /* 64x64 block origin */
  uint8_t mode;             /* MT_*_PRED */
  int8_t angle_delta;       /* -3..3, directional modes only */
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL of the 64x64 block, MT_CAND_FILTER_TYPE */
  uint8_t reserved;
  uint8_t dcs_ctx[4];       /* dc_sign_ctx_32 of each quadrant, raster order */
  float mode_bits;          /* mode_bits(px, py, mode) */
  float delta_bits;         /* the angle-delta symbol's bits (read for directional modes) */
} mt_quad32_job;
typedef struct mt_quad32_result {
  float total;              /* the candidate's total cost */
  float bits[4];            /* each quadrant's coefficient bits */
  uint32_t reserved;
  int64_t sse[4];           /* each quadrant's sse_recon */
} mt_quad32_result;
int mt_quad32_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_quad32_job* d_jobs, int32_t n, mt_quad32_result* d_results, void* stream);
/* Host-buffer form of mt_quad32_luma_device. */
int mt_quad32_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_quad32_job* jobs, int32_t n,
                   mt_quad32_result* results);

/* The 64x64 leaf's sixteen-TX_16X16 leg (rd_pick_luma64's tx_depth-2 trial,
 * src/coder/block64.rs:1983-2010, on in the shipped tuning as tx64_depth2,
 * through grid16_luma_pass, :1670-1805): for the winning (mode, delta) of a
 * 64x64 block, the sixteen 16x16 transforms in raster order, each predicted at
 * 16x16 from the block's running reconstruction with the per-transform edge
 * flags (first row: top-right when the block has a row above and the
 * transform is not the last column or the block has its top-right; other
 * rows: not the last column; first column: bottom-left when the block has a
 * column on its left and the transform is not the last row or the block has
 * its bottom-left; other columns: none), TX_16X16 DCT_DCT with the QM and
 * trellis_optimize_ctx in the dc_sign context of the transform's four above
 * and four left coefficient-context bytes (dc_sign_ctx_span), the inverse,
 * the distortion sse_recon x K_PART_LAMBDA, and luma_bits_ctx_bounded in the
 * txb_skip context skip_ctx_split of the same bytes with the DCT_DCT symbol
 * (1 in the TX_16X16 intra set) of the mode's tx-type CDF; the transform's
 * coef_res_ctx then fills its four above and four left bytes.  dist and bits
 * are f32 sums in raster order; total = (rd_lambda x mode_bits [+ rd_lambda x
 * delta_bits]) + (dist + rd_lambda x bits) + rd_lambda x depth_bits.  Costs /
 * qm row: the TX_16X16 slice and 16x16 row; skip_bits[ctx]: the TX_16X16
 * class's pair per txb_skip context.  Rejected jobs (outside the frame, a bad
 * mode / delta) get total, dist and bits +inf, sse 0. */
typedef struct mt_grid16_job {
  uint16_t px, py;          /* 64x64 block origin */
  uint8_t mode;             /* MT_*_PRED */
  int8_t angle_delta;       /* -3..3, directional modes only */
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL of the 64x64 block, MT_CAND_FILTER_TYPE */
  uint8_t reserved;
  uint8_t a_coef[16];       /* above coefficient contexts of the block's sixteen 4-sample columns */
  uint8_t l_coef[16];       /* left coefficient contexts of its sixteen 4-sample rows */
  float mode_bits;          /* mode_bits(px, py, mode) */
  float delta_bits;         /* the angle-delta symbol's bits (read for directional modes) */
  float depth_bits;         /* tx_depth64_bits(2) - tx_depth64_bits(1) */
} mt_grid16_job;
typedef struct mt_grid16_result {
  float total;              /* the tx_depth-2 total */
  float dist;               /* sum of the transforms' sse x K_PART_LAMBDA */
  float bits;               /* sum of their coefficient bits */
  uint32_t reserved;
  int64_t sse;              /* sum of their sse_recon */
} mt_grid16_result;
/* Device form.  d_cf (optional): n x 4096 int32, transform t's levels
 * (column-major, as the 16x16 leaf's) at t * 256, raster order. */
int mt_grid16_luma_device(const uint16_t* d_src, const uint16_t* d_recon, const mt_split16_params* prm,
                          const mt_quant* quant, const uint8_t* d_qm_row, const mt_coef_costs* d_costs,
                          const mt_grid16_job* d_jobs, int32_t n, mt_grid16_result* d_results, int32_t* d_cf,
                          void* stream);
/* Host-buffer form of mt_grid16_luma_device. */
int mt_grid16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                   const uint8_t* qm_row, const mt_coef_costs* costs, const mt_grid16_job* jobs, int32_t n,
                   mt_grid16_result* results, int32_t* cf_out);

/* ---- Chroma RD ----
 * uv_mode_bits (src/coder/lossy_state.rs:1302-1349) prices a chroma mode from
 * the decision CDFs: the CfL-allowed uv_mode CDF of the luma mode, the
 * angle-delta CDF at delta 0 for a directional mode, and for CfL the joint
 * sign and the per-plane alpha magnitudes (contexts by the other plane's
 * sign); CfL with both alphas 0 is priced as DC.  CDFs in the inverse form of
 * mt_coef_cdfs (one entry per symbol, the last 0). */
#define MT_UV_CFL_PRED 13
typedef struct mt_uv_mode_cdfs {
  uint16_t uv_mode[13][14];    /* uv_mode with CfL allowed, per y mode */
  uint16_t angle_delta[8][7];  /* per directional mode, V_PRED..D67_PRED */
  uint16_t cfl_sign[8];
  uint16_t cfl_alpha[6][16];
} mt_uv_mode_cdfs;
typedef struct mt_uv_mode_costs {  /* cdf_cost_with_table of every symbol of the same CDFs */
  float uv_mode[13][14];
  float angle_delta[8][7];
  float cfl_sign[8];
  float cfl_alpha[6][16];
} mt_uv_mode_costs;
/* The decision snapshot's CDFs (Cdfs::new, src/coder/cdfs.rs; the mode CDFs
 * do not depend on the quantiser). */
int mt_uv_mode_cdfs_default(mt_uv_mode_cdfs* out);
int mt_uv_mode_costs_build(const mt_uv_mode_cdfs* cdfs, mt_uv_mode_costs* out);
/* uv_mode_bits(y_mode, uv_mode, cfl ? Some([alpha_u, alpha_v]) : None). */
float mt_uv_mode_bits(const mt_uv_mode_costs* costs, int32_t y_mode, int32_t uv_mode, int32_t cfl, int32_t alpha_u,
                      int32_t alpha_v);

/* The 16x16 leaf's 4:2:0 chroma search (pick_uv16_420,
 * src/coder/block16.rs:980-1381, with the shipped tuning: uv16_joint on,
 * uv8_joint_k 4, cfl_alpha_rd_steps 0) over n 16x16 leaves, each with an 8x8
 * chroma block at (px / 2, py / 2):
 *   1. DC: per plane the DC prediction, DCT_DCT with the QM, the chroma
 *      trellis (trellis_optimize_ctx, coefficient class TX_8X8, chroma CDFs,
 *      the dc_sign context of the plane's two above / two left bytes),
 *      preserve_dc, the inverse, sse_recon and chroma_bits (txb_skip context
 *      7 + above non-zero + left non-zero, no tx-type symbol); total = the
 *      planes' rd_cost_i64 in f32, with no mode bits;
 *   2. CfL: the AC of the 16x16 luma reconstruction (cfl_ac_sub 4:2:0), each
 *      plane's closed-form alpha (cfl_best_alpha over the displayed part),
 *      its prediction through DCT_DCT, trellis, inverse, sse and bits (no
 *      preserve_dc); total = the planes' costs + rd_lambda x
 *      uv_mode_bits(CfL, alphas) - rd_lambda x uv_mode_bits(DC); taken when an
 *      alpha is non-zero and the total is below the best;
 *   3. the joint shortlist: SMOOTH_V, PAETH, SMOOTH, SMOOTH_H, V, H, D135,
 *      D113, D157, D45, D67, D203, the directional ones at deltas -3..3 when
 *      angle_deltas is set, each scored by the two planes' satd_sad_proxy,
 *      sorted by (score, mode, delta); the first joint_k are priced: rd_lambda
 *      x (uv_mode_bits + the delta's angle-delta bits over delta 0's), then
 *      per plane the prediction with the leaf's edge flags, the mode's
 *      transform (dav1d's uv-mode map: ADST_ADST, ADST_DCT, DCT_ADST or
 *      DCT_DCT) with the QM, trellis, preserve_dc, inverse, sse and bits,
 *      stopping after U when the total already reaches the best; taken when
 *      below the best.
 * Params: mt_split16_params of the chroma planes (frame_w / frame_h the
 * chroma plane's size, stride its stride, vis_w / vis_h its displayed size,
 * trellis_lambda0 the trellis lambda, rd_lambda the chroma mode lambda
 * (emit_mlam_c), band_tilt of the chroma quantiser, wsse_scale, skip_bits[ctx]
 * the TX_8X8 class's chroma pairs when use_skip_bits); quant the chroma
 * quantiser; qm row the 8x8 chroma weights (NULL: flat); costs the chroma
 * TX_8X8 slice (mt_coef_cdfs_default(qctx, 8, 8, 1)). */
typedef struct mt_uv16_params {
  int32_t luma_stride;   /* stride of the luma reconstruction the CfL AC reads */
  int32_t joint_k;       /* 4:2:0: shortlist length, clamped to 1..12 (uv8_joint_k) */
  int32_t angle_deltas;  /* try_angle_deltas_av1(16, base_q_idx) */
  float dir_lambda;      /* 4:4:4: the directional stage's lambda (emit_mlam: uv16_444_mlam_c is off) */
} mt_uv16_params;
typedef struct mt_uv16_job {
  uint16_t px, py;          /* 16x16 luma leaf origin */
  uint8_t y_mode;           /* the luma winner's mode */
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL of the leaf, MT_CAND_FILTER_TYPE: chroma filter type */
  uint8_t a_coef[2][2];     /* above coefficient contexts of the chroma block's two 4-sample columns, U then V */
  uint8_t l_coef[2][2];     /* left contexts of its two 4-sample rows */
  uint8_t reserved[2];
} mt_uv16_job;
typedef struct mt_uv16_result {
  float total;              /* the winner's total (the picker's best_total) */
  float dc_total;           /* the DC path's total */
  float cfl_total;          /* the CfL path's total */
  uint8_t uv_mode;          /* MT_*_PRED or MT_UV_CFL_PRED; 255 for a rejected job */
  int8_t angle_delta;
  int8_t cfl_alpha[2];      /* the closed-form alphas (U, V) */
} mt_uv16_result;
/* Device form.  d_luma: the luma reconstruction (luma_stride); d_src_u /
 * d_src_v and d_rec_u / d_rec_v: the chroma source and reconstruction planes
 * (prm->stride).  d_cf (optional): n x 128 int32, the winner's U then V
 * levels; d_rec (optional): n x 128 uint16, its U then V reconstruction
 * (clamp(prediction + inverse)).  Rejected jobs (chroma block outside the
 * plane, a bad mode) get uv_mode 255 and total +inf. */
int mt_pick_uv16_420_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv16_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream);
/* Host-buffer form: chroma planes prm->stride x prm->frame_h, the luma
 * reconstruction luma_stride x 2 frame_h. */
int mt_pick_uv16_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv16_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out);

/* The 16x16 leaf's 4:4:4 chroma search (pick_uv16_444,
 * src/coder/block16.rs:437-978, shipped tuning: no palette outside screen
 * content, uv16_444_mlam_c off, cfl_alpha_rd_steps 0) on the leaf's 16x16
 * chroma blocks (the luma position):
 *   1. DC: per plane DCT_DCT with the QM, the plain trellis_optimize (the
 *      4:4:4 chroma_rect_trellis), preserve_dc, the inverse, sse_recon and
 *      chroma_bits (coefficient class TX_16X16, txb_skip context 7 + above
 *      non-zero + left non-zero over four bytes each, dc_sign over 4 + 4);
 *   2. CfL: the 4:4:4 AC of the leaf's luma reconstruction, each plane's
 *      cfl_best_alpha, the same chain without preserve_dc; taken when an
 *      alpha is non-zero and rd_cost_i64(sse_u + sse_v, rd_lambda, bits_u +
 *      bits_v + uv_mode_bits(CfL)) is below DC's (with uv_mode_bits(DC));
 *   3. with dir_lambda: the current choice's total rd_lambda' x mode bits +
 *      the planes' rd_cost_i64, then the 12 modes at delta 0 ranked by the two
 *      planes' satd_sad_proxy, the 3 best (DirectionalTopK: strict insertion,
 *      ties to the earlier mode) priced in list order with the mode's
 *      transform, the trellis, preserve_dc; a winner that is directional with
 *      angle_deltas set then tries its zone-2 deltas (V: 1..3, H: -3..-1,
 *      D113 / D135 / D157: +-1..3) predicted with no top-right / bottom-left.
 * Params as for mt_pick_uv16_420 with the chroma planes at the luma size
 * (luma_stride may equal prm->stride), the 16x16 chroma QM row (256 weights)
 * and the chroma TX_16X16 cost slice (mt_coef_cdfs_default(qctx, 16, 16, 1));
 * rd_lambda is emit_mlam_c, uvp->dir_lambda emit_mlam.  d_cf / d_rec: n x
 * 512, U then V. */
typedef struct mt_uv16_444_job {
  uint16_t px, py;          /* 16x16 leaf origin (luma and chroma) */
  uint8_t y_mode;
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL of the leaf, MT_CAND_FILTER_TYPE: chroma filter type */
  uint8_t a_coef[2][4];     /* above coefficient contexts of the block's four 4-sample columns, U then V */
  uint8_t l_coef[2][4];
  uint8_t reserved[2];
} mt_uv16_444_job;
/* The 32x32 leaf's 4:4:4 chroma search (pick_uv32_444,
 * src/coder/block32.rs:2264-2720, shipped tuning) on its 32x32 chroma blocks:
 * as mt_pick_uv16_444 at 32x32, with every transform DCT_DCT (forced at
 * TX_32X32), the plain trellis_optimize over the 1024-entry scan, chroma_bits
 * of the chroma TX_32X32 class (contexts over eight above / eight left
 * bytes), and CfL taken when the planes' rd_cost_i64 summed plus rd_lambda x
 * uv_mode_bits(CfL) is below DC's sum plus rd_lambda x uv_mode_bits(DC).
 * uvp->dir_lambda is mlam_c x (emit_mlam / mlam) at 32.  QM row: the 32x32
 * chroma weights; costs: the chroma TX_32X32 slice (mt_coef_cdfs_default(qctx,
 * 32, 32, 1)).  d_cf / d_rec: n x 2048, U then V. */
typedef struct mt_uv32_444_job {
  uint16_t px, py;          /* 32x32 leaf origin (luma and chroma) */
  uint8_t y_mode;
  uint8_t flags;            /* MT_CAND_HAVE_TR / HAVE_BL of the leaf, MT_CAND_FILTER_TYPE: chroma filter type */
  uint8_t a_coef[2][8];     /* above coefficient contexts of the block's eight 4-sample columns, U then V */
  uint8_t l_coef[2][8];
  uint8_t reserved[2];
} mt_uv32_444_job;
int mt_pick_uv32_444_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv32_444_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream);
int mt_pick_uv32_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv32_444_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out);

/* The 32x32 leaf's 4:2:0 chroma search (pick_uv32_420,
 * src/coder/block32.rs:2797-3120, shipped tuning: uv_ad and uv_ad32 on,
 * cfl_alpha_rd_steps 0) on the leaf's 16x16 chroma blocks at (px / 2, py / 2):
 * DC (DCT_DCT with the QM, trellis_optimize_ctx of the chroma TX_16X16 class
 * in the dc_sign context of the plane's four above / four left bytes,
 * preserve_dc); CfL from the 4:2:0 AC of the 32x32 luma reconstruction,
 * taken when an alpha is non-zero and body + rd_lambda x (uv_mode_bits(CfL) -
 * uv_mode_bits(DC)), f32 as the reference orders it, is below DC's; the 12
 * modes at delta 0 ranked by SATD into a top-3 priced in list order (each
 * winner clearing CfL); when CfL did not win and angle_deltas is set, a
 * directional winner's zone-2 deltas with no top-right / bottom-left.  Every
 * total on rd_lambda (emit_mlam_c at 32).  Jobs: mt_uv16_444_job's layout
 * with px / py the 32x32 leaf origin and the contexts those of the 16x16
 * chroma block.  Params, QM row and costs as for the 4:4:4 search (16x16 chroma
 * weights, the chroma TX_16X16 slice); the luma reconstruction luma_stride x
 * 2 frame_h.  d_cf / d_rec: n x 512, U then V. */
typedef mt_uv16_444_job mt_uv32_420_job;
int mt_pick_uv32_420_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv32_420_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream);
int mt_pick_uv32_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv32_420_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out);
int mt_pick_uv16_444_device(const uint16_t* d_src_u, const uint16_t* d_src_v, const uint16_t* d_rec_u,
                            const uint16_t* d_rec_v, const uint16_t* d_luma, const mt_split16_params* prm,
                            const mt_uv16_params* uvp, const mt_quant* quant, const uint8_t* d_qm_row,
                            const mt_coef_costs* d_costs, const mt_uv_mode_costs* d_mode_costs,
                            const mt_uv16_444_job* d_jobs, int32_t n, mt_uv16_result* d_results, int32_t* d_cf,
                            uint16_t* d_rec, void* stream);
int mt_pick_uv16_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* prm, const mt_uv16_params* uvp,
                     const mt_quant* quant, const uint8_t* qm_row, const mt_coef_costs* costs,
                     const mt_uv_mode_costs* mode_costs, const mt_uv16_444_job* jobs, int32_t n,
                     mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out);

/* Host-buffer form (planes stride x frame_h; costs and qm row on the host). */
int mt_split16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* prm, const mt_quant* quant,
                    const uint8_t* qm_row, const mt_coef_costs* costs, const mt_split16_job* jobs, int32_t n,
                    mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out);

/* ---- Filter-intra shortlist ----
 * rank_filter_intra_modes (src/coder/superblock.rs:356-400) over n luma blocks
 * of w x h (4, 8, 16 or 32 each) at pos[2b], pos[2b+1]: each of the five
 * filter-intra modes (DC, V, H, D157, PAETH in that order) predicted by the
 * recursive 4x2-cell filter (filter_intra_predict, src/intrapred.rs:473-565:
 * the above row of w samples, the left column of h samples and the corner,
 * with the reference's fills when an edge is missing; no above-right), scored
 * by satd_sad_proxy (samples past the displayed window count as the
 * prediction), and sorted by (score, mode order); the caller keeps the first
 * `budget`.  scores / modes: n x MT_FILTER_INTRA_MODES ascending; preds
 * (optional): n x 5 x w*h int16, row-major, in mode order.  A block outside
 * the frame gets scores of all ones and modes 255. */
#define MT_FILTER_INTRA_MODES 5
int mt_filter_intra_beam_device(const uint16_t* d_src, const uint16_t* d_recon, int32_t stride, int32_t frame_w,
                                int32_t frame_h, int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h,
                                const uint16_t* d_pos, int32_t n, uint64_t* d_scores, uint8_t* d_modes,
                                int16_t* d_preds, void* stream);
/* Host-buffer form (planes stride x frame_h; scores and preds may be NULL). */
int mt_filter_intra_beam(const uint16_t* src, const uint16_t* recon, int32_t stride, int32_t frame_w, int32_t frame_h,
                         int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h, const uint16_t* pos,
                         int32_t n, uint64_t* scores, uint8_t* modes, int16_t* preds);

/* ---- Chroma-from-luma alpha search ----
 * For n chroma blocks of cw x ch samples (4, 8, 16 or 32 each): the luma AC of
 * the co-located reconstructed luma (cfl_ac_sub, src/intrapred.rs:1133-1172:
 * each chroma position sums its 1, 2 or 4 luma samples, scaled to the <<3
 * range, then the rounded block mean is removed; cfl_ac_444 is the unsampled
 * case) and, for each of the U and V planes, the alpha of cfl_best_alpha
 * (src/intrapred.rs:1211-1258): the analytic least-squares optimum
 * round(64 num / den) clamped to [-16, 16], then the candidate in its +-3
 * neighbourhood (inside [-16, 16]) with the lowest SSE of src - cfl_pred
 * (dc + sign(alpha ac) ((|alpha ac| + 32) >> 6), clamped), first minimum; 0
 * when the AC has no energy.  Only the displayed part of each block
 * (vis_cw x vis_ch chroma samples of the plane; 0 = the whole block) is
 * measured, as the reference's SrcBlock does.  sub_x / sub_y: the chroma
 * subsampling (1, 1) 4:2:0, (1, 0) 4:2:2, (0, 0) 4:4:4.  dc: the DC_PRED value
 * of the block in each plane, which the caller computes from its chroma
 * reconstruction (dc_pred).  alpha: n x 2 (U, V); ac (optional): n x cw*ch
 * int32 row-major, the AC the prediction uses. */
typedef struct mt_cfl_block {
  uint16_t cx, cy;          /* chroma sample position */
  int16_t dc[2];            /* DC_PRED of the U and V planes at the block */
} mt_cfl_block;
int mt_cfl_alpha_device(const uint16_t* d_luma, int32_t luma_stride, const uint16_t* d_src_u, const uint16_t* d_src_v,
                        int32_t chroma_stride, int32_t sub_x, int32_t sub_y, int32_t cw, int32_t ch, int32_t vis_cw,
                        int32_t vis_ch, int32_t bd, const mt_cfl_block* d_blocks, int32_t n, int8_t* d_alpha,
                        int32_t* d_ac, void* stream);
/* Host-buffer form: luma is luma_stride x luma_h samples, the chroma planes
 * chroma_stride x chroma_h. */
int mt_cfl_alpha(const uint16_t* luma, int32_t luma_stride, int32_t luma_h, const uint16_t* src_u,
                 const uint16_t* src_v, int32_t chroma_stride, int32_t chroma_h, int32_t sub_x, int32_t sub_y,
                 int32_t cw, int32_t ch, int32_t vis_cw, int32_t vis_ch, int32_t bd, const mt_cfl_block* blocks,
                 int32_t n, int8_t* alpha, int32_t* ac);

/* ---- Lossy luma palette candidates (src/coder/palette.rs) ----
 * Per w x h block (w, h in 4..64, powers of two): block_color_histogram
 * (:651-706: distinct values ascending with counts; no candidate when the
 * block has < 2 or > 64 distinct values), then fourteen candidate slots:
 * slot s < 7 is sel = s + 2 colours with palette_centers' exact values
 * (colours == distinct) or dp_palette_center_sets' optimal centres
 * (:728-869, the shipped palette_dp_centers), slot s >= 7 is sel = s + 3
 * (s - 5 colours) with top_palette_centers' dominant colours (:708-726, only
 * when colours < distinct).  Each candidate's index map is built by
 * lossy_luma_palette_from_centers (:1218-1265): the row Viterbi
 * (viterbi_map_core, :1028-1172) when viterbi_lambda > 0, else
 * luma_nearest_indices (src/kmeans.rs:71-101) + smooth_palette_map
 * (:1173-1216) when smooth_t > 0; then palette_index_bits (:1911-1925). */
#define MT_PALETTE_SLOTS 14

typedef struct mt_palette_opts {
  int32_t smooth_t;             /* palette_smooth tolerance in sample units; 0 = off */
  int32_t smooth_guard;         /* palette_smooth_guard: keep samples the nearest centre hits exactly */
  float viterbi_lambda;         /* > 0: the Viterbi map with this lambda (mlam x palette_viterbi_*) */
  float color_costs[7][5][8];   /* palette_y_color bits [colours - 2][ctx][symbol] (pal_y_cost_tables) */
} mt_palette_opts;

typedef struct mt_palette_cand {
  int16_t colors[8];  /* ascending centres, n_colors valid, the rest 0 */
  uint8_t n_colors;   /* 0: no candidate in this slot */
  uint8_t sel;        /* 2..8 (exact / optimal centres) or 10..16 (dominant colours) */
  uint8_t hist_len;   /* the block's distinct values; 0 when the histogram gate rejects it */
  uint8_t reserved;
  float index_bits;   /* palette_index_bits of the map; 0 for an empty slot */
} mt_palette_cand;

/* d_pos: n (x, y) uint16 pairs; d_cands: n x MT_PALETTE_SLOTS; d_maps:
 * n x MT_PALETTE_SLOTS x w x h indices (zero for an empty slot).  A block
 * outside frame_w x frame_h, or with a sample above (1 << bd) - 1, gets
 * empty slots. */
int mt_luma_palette_device(const uint16_t* d_src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd,
                           int32_t w, int32_t h, const uint16_t* d_pos, int32_t n, const mt_palette_opts* opts,
                           mt_palette_cand* d_cands, uint8_t* d_maps, void* stream);
/* Host-buffer form; maps may be NULL. */
int mt_luma_palette(const uint16_t* src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd, int32_t w,
                    int32_t h, const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_palette_cand* cands,
                    uint8_t* maps);

/* ---- UV palette candidates (4:4:4 screen content: the palette leg of
 * pick_uv16_444 / pick_uv32_444, src/coder/block16.rs:813-860) ----
 * Per w x h chroma block (w, h in 4..32): exact_uv_palette
 * (src/coder/palette.rs:199-262) when the block holds 2..8 distinct (U, V)
 * pairs -- slot 0, exact = 1, the pairs in lexicographic order and the map
 * of each sample's pair; otherwise lossy_uv_palette_from_hist (:315-431) over
 * uv_pair_histogram (:264-309, the block's pairs sorted and counted) in
 * slots 0..3 for (8 colours, k-means), (4, k-means), (8, dominant pairs),
 * (4, dominant pairs): all pairs when the histogram holds exactly that many,
 * the most frequent pairs (count descending, pair ascending), or eight Lloyd
 * passes from weighted-quantile starts with integer rounded means, a slot
 * left empty when the centres collapse or the histogram is too small.  The
 * centres are sorted; the index map is viterbi_uv_palette_map (:1053-1076:
 * the row Viterbi on the squared (U, V) distance with opts->color_costs, the
 * palette_uv_color bits, and opts->viterbi_lambda) when viterbi_lambda > 0,
 * else uv_nearest_indices (src/kmeans.rs:37-68). */
#define MT_UV_PALETTE_SLOTS 4
typedef struct mt_uv_palette_cand {
  uint8_t n_colors;   /* 0: no candidate in this slot */
  uint8_t exact;      /* 1: exact_uv_palette's */
  uint8_t reserved[2];
  int16_t u[8];       /* the centres in (U, V) lexicographic order, n_colors valid */
  int16_t v[8];
} mt_uv_palette_cand;
/* d_pos: n (x, y) uint16 block origins in the chroma planes (stride);
 * d_cands: n x MT_UV_PALETTE_SLOTS; d_maps: n x MT_UV_PALETTE_SLOTS x w x h
 * (zero for an empty slot).  opts->smooth_t is not used. */
int mt_uv_palette_device(const uint16_t* d_src_u, const uint16_t* d_src_v, int32_t stride, int32_t w, int32_t h,
                         const uint16_t* d_pos, int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* d_cands,
                         uint8_t* d_maps, void* stream);
/* Host-buffer form: planes stride x rows (rows covering every block). */
int mt_uv_palette(const uint16_t* src_u, const uint16_t* src_v, int32_t stride, int32_t rows, int32_t w, int32_t h,
                  const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* cands,
                  uint8_t* maps);

/* Forward transform + quantisation of n residual blocks (row-major int32,
 * tx_size^2 each) with one tx type per block: levels (column-major int32) and
 * f32 quantisation targets, with the QM applied as DctDispatch does. */
int mt_fwd_txfm_quant_device(const int32_t* d_resid, const uint8_t* d_tx_types, int32_t n,
                             int32_t tx_size, const mt_quant* quant, const uint8_t* d_qm_row,
                             int32_t* d_levels, float* d_targets, void* stream);
/* Inverse transform + dequantisation of n level blocks -> row-major residual. */
int mt_inv_txfm_dequant_device(const int32_t* d_levels, const uint8_t* d_tx_types, int32_t n,
                               int32_t tx_size, const mt_quant* quant, const uint8_t* d_qm_row,
                               int32_t* d_resid, void* stream);
/* trellis_optimize over n blocks in place (levels), one scan for all. */
int mt_trellis_optimize_device(int32_t* d_levels, const float* d_targets, int32_t n,
                               int32_t tx_size, float dc_q, float ac_q, float lambda0,
                               void* stream);
/* Intra prediction of n candidates (mode/angle/flags from the candidate
 * records) into pred_out (n * tx_size^2 int32, row-major). */
int mt_intra_predict_device(const uint16_t* d_recon, const mt_chain_params* prm,
                            const mt_candidate* d_cands, int32_t n, int32_t* d_pred_out,
                            void* stream);

/* Colour conversion + padding (src/encoder.rs:113-127, :370-410, :532-604
 * and src/dispatch.rs:113-131): interleaved 8-bit RGB (w x h x 3) -> the
 * coder's padded u16 planes.  sub = 0 (4:4:4) or 2 (4:2:0).  Padded sizes from
 * mt_padded_plane_dims: luma align8(w) x align8(h), chroma that >> sub. */
int mt_padded_plane_dims(int32_t w, int32_t h, int32_t sub, int32_t* pw, int32_t* ph, int32_t* pcw,
                         int32_t* pch);
int mt_csc_rgb8(const uint8_t* rgb, int32_t w, int32_t h, int32_t sub, uint16_t* y, uint16_t* cb,
                uint16_t* cr);
int mt_csc_rgb8_device(const uint8_t* d_rgb, int32_t w, int32_t h, int32_t sub, uint16_t* d_y,
                       uint16_t* d_cb, uint16_t* d_cr, void* stream);

/* Deblocking of one plane (src/loopfilter.rs:482-648 filter_plane_impl, with
 * the dav1d loop filter of src/loopfilter.rs:98-292), as src/coder/frame_deblock.rs
 * drives it per plane.  px: the padded plane (w x h u16, w and h multiples of 4),
 * filtered in place; only edges inside the visible vis_w x vis_h window are
 * filtered.  bw4 / bh4: block width / height in 4-sample units per 4x4 cell
 * (row-major, nc4 cells per row, ceil(vis_h/4) rows; entries >= 1).  vedge4 /
 * hedge4: 1 where a block starts at that cell column / row, or NULL for the
 * alignment rule (col % bw4 == 0, row % bh4 == 0).  level 0..63 (0 = no
 * filtering), sharp 0..7, is_luma selects the 4/8/16 (luma) or 4/6 (chroma)
 * widths.  bd must be 8. */
int mt_deblock_plane(uint16_t* px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* bw4,
                     const uint8_t* bh4, const uint8_t* vedge4, const uint8_t* hedge4, int32_t nc4, int32_t level,
                     int32_t sharp, int32_t is_luma, int32_t bd);
int mt_deblock_plane_device(uint16_t* d_px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* d_bw4,
                            const uint8_t* d_bh4, const uint8_t* d_vedge4, const uint8_t* d_hedge4, int32_t nc4,
                            int32_t level, int32_t sharp, int32_t is_luma, int32_t bd, void* stream);

/* Frame deblocking as src/coder/frame_deblock.rs:206-224 (frame_deblock)
 * drives it: luma from the luma TRANSFORM-block maps with explicit block-start
 * flags (16 4-rows per superblock), then, when luma is filtered and a chroma
 * level is non-zero, U and V from chroma geometry derived from the luma
 * PREDICTION-block maps (src/coder/frame_deblock.rs:87-152: size >> subsampling,
 * clamped to 1..8 cells, alignment-rule edges).  Maps: (h8/4) x (w8/4) u8 cells
 * of the luma grid.  Sharpness is the shipped 7. */
typedef struct mt_deblock_frame_params {
  int32_t w8, h8;          /* padded luma plane (multiples of 8) */
  int32_t disp_w, disp_h;  /* visible luma size */
  int32_t sub_x, sub_y;    /* chroma subsampling shifts */
  int32_t mono;
  int32_t bd;              /* 8 */
} mt_deblock_frame_params;
/* loop_filter_levels / loop_filter_sharpness (src/obu.rs:306-334, shipped
 * tuning): the frame's luma and chroma levels and the sharpness. */
int mt_loop_filter_levels(int32_t base_q_idx, int32_t sub_x, int32_t sub_y, int32_t* lvl_y, int32_t* lvl_uv,
                          int32_t* sharp);
/* Device working storage of the two device entries below (edge widths per
 * cell, the chroma geometry, and room for the unfiltered planes of an
 * in-place call). */
size_t mt_deblock_frame_scratch_bytes(const mt_deblock_frame_params* prm);
/* The frame deblocked in place on the stream: the planes are snapshotted into
 * the scratch, then each 64x64 tile is filtered from the snapshot (all
 * vertical, then all horizontal edges, in shared memory) and written once.
 * Maps whose edges have overlapping taps (no AV1 geometry has them) are
 * filtered by two frame-wide passes that keep the reference's order. */
int mt_deblock_frame_device(uint16_t* d_y, uint16_t* d_u, uint16_t* d_v, const uint8_t* d_blk4,
                            const uint8_t* d_blk4h, const uint8_t* d_blk4v, const uint8_t* d_blk4t,
                            const uint8_t* d_pblk4, const uint8_t* d_pblk4h, const mt_deblock_frame_params* prm,
                            int32_t lvl_y, int32_t lvl_u, int32_t lvl_v, void* d_scratch, void* stream);
/* The same from unfiltered planes d_in_* (left unchanged) into the planes
 * d_* (same sizes, separate buffers), without the snapshot.  No counterpart in
 * the reference, which filters in place. */
int mt_deblock_frame_device_to(const uint16_t* d_in_y, const uint16_t* d_in_u, const uint16_t* d_in_v, uint16_t* d_y,
                               uint16_t* d_u, uint16_t* d_v, const uint8_t* d_blk4, const uint8_t* d_blk4h,
                               const uint8_t* d_blk4v, const uint8_t* d_blk4t, const uint8_t* d_pblk4,
                               const uint8_t* d_pblk4h, const mt_deblock_frame_params* prm, int32_t lvl_y,
                               int32_t lvl_u, int32_t lvl_v, void* d_scratch, void* stream);
int mt_deblock_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint8_t* blk4, const uint8_t* blk4h,
                     const uint8_t* blk4v, const uint8_t* blk4t, const uint8_t* pblk4, const uint8_t* pblk4h,
                     const mt_deblock_frame_params* prm, int32_t lvl_y, int32_t lvl_u, int32_t lvl_v);

/* Frame CDEF (src/coder/frame_cdef.rs:49-520 frame_cdef, with the filter,
 * direction search and 12-strength candidate evaluation of src/cdef.rs), in
 * the configuration the encoder ships: weighted-SSE decision metric
 * (src/rd_sse.rs weighted_sse, AVX2 order src/avx/rd.rs:767-848, scale 1),
 * 40 per-mille margin, directional-variance gate 15000, chroma weight 1, CDEF
 * bits priced with the frame lambda_d.
 *
 * Planes: luma w8 x h8 (multiples of 8), chroma (w8 >> sub_x) x (h8 >> sub_y)
 * (absent when mono), all u16 row-major; recon planes are filtered in place.
 * skip8: one byte per luma 8x8 block ((w8/8) x (h8/8), 1 = skip block, which
 * CDEF leaves untouched).  The caller gates CDEF as the reference does (no
 * IntraBC, CDEF enabled, base_q_idx != 0). */
typedef struct mt_cdef_params {
  int32_t w8, h8;          /* padded luma plane */
  int32_t disp_w, disp_h;  /* visible luma size (w8 - 8 < disp_w <= w8) */
  int32_t sub_x, sub_y;    /* chroma subsampling shifts: (1,1) 4:2:0, (1,0) 4:2:2, (0,0) 4:4:4 */
  int32_t mono;            /* 1: luma only */
  int32_t base_q_idx;      /* 1..255 */
  int32_t bd;              /* 8 */
  int32_t slow;            /* 1: Speed::Slow or slower (two-stage strength search) */
} mt_cdef_params;

typedef struct mt_cdef_decision {
  int32_t bits;            /* cdef_bits 0..3, or -1: CDEF off for the frame (planes unchanged) */
  int32_t damping;         /* signalled damping 3..6 */
  int32_t n_strengths;     /* entries in strengths (1 << bits), 0 when bits == -1 */
  int32_t unit_cols, unit_rows;  /* the 64x64 unit grid */
  uint8_t strengths[8][4]; /* per entry: luma pri, luma sec, chroma pri, chroma sec */
} mt_cdef_decision;

/* Per-block directions / variances and the per-64x64-unit distortion of all
 * 12 strength pairs (index sec_idx * 4 + pri_idx over pri {0,1,2,4}, sec
 * {0,1,2}): src/coder/frame_cdef.rs:600-820 cdef_luma_unit_dists_all /
 * cdef_chroma_unit_sse_all.  dirs / vars: (h8/8) x (w8/8); tables:
 * unit_rows x unit_cols x 12 int64 (u / v tables ignored when mono). */
int mt_cdef_tables_device(const uint16_t* d_y, const uint16_t* d_u, const uint16_t* d_v, const uint16_t* d_src_y,
                          const uint16_t* d_src_u, const uint16_t* d_src_v, const uint8_t* d_skip8,
                          const mt_cdef_params* prm, uint8_t* d_dirs, int32_t* d_vars, int64_t* d_luma_tab,
                          int64_t* d_u_tab, int64_t* d_v_tab, void* stream);
/* Device working storage mt_cdef_frame_device needs. */
size_t mt_cdef_scratch_bytes(const mt_cdef_params* prm);
/* The whole frame CDEF on the stream: tables, the strength search and the
 * filter applied to the recon planes, back to back on the device; the stream
 * is synchronised once, at the end, to read the decision.  grid: host buffer
 * of unit_cols * unit_rows bytes (the per-unit strength index; zeros unless
 * bits > 0), may be NULL. */
int mt_cdef_frame_device(uint16_t* d_y, uint16_t* d_u, uint16_t* d_v, const uint16_t* d_src_y,
                         const uint16_t* d_src_u, const uint16_t* d_src_v, const uint8_t* d_skip8,
                         const mt_cdef_params* prm, void* d_scratch, mt_cdef_decision* out, uint8_t* grid,
                         void* stream);
/* Host-buffer form of mt_cdef_frame_device. */
int mt_cdef_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint16_t* src_y, const uint16_t* src_u,
                  const uint16_t* src_v, const uint8_t* skip8, const mt_cdef_params* prm, mt_cdef_decision* out,
                  uint8_t* grid);

/* ---- Adaptive quantisation: the per-superblock qindex grid ----
 * Replaces the frame pre-pass of the reference's tile encoder: for every tile,
 * tile_ref_activity / tile_ref_picked (src/coder/aq.rs:162-192) and
 * precompute_aq_grid -> aq_sb_target (src/coder/lossy_state.rs:3796-3963), with
 * Variance Boost (src/aq_common.rs:58-150), dark-structure protection
 * (src/aq_common.rs:216-345, DarkAq::on) and the relative step clamp
 * (src/coder/lossy_state.rs:133-154).  Shipped tuning: aq_slope 5, aq_max_delta
 * 28, aq_r 1.35, top_ease 1 / knee 20 / width 12, delta_q_res 2 (steps of 4
 * qindex, at most 12 per superblock).
 *
 * The luma plane is the padded source, w8 x h8 u16 row-major (stride w8).
 * Tiles follow the frame header's uniform spacing for the given log2 counts
 * (src/coder/tiling.rs:138-147); each tile has at most 64 superblock columns
 * and 2304 superblocks (the AV1 limits), else MT_ERR_INVALID_INPUT.  The chain
 * restarts at base_q_idx in every tile. */
typedef struct mt_aq_params {
  int32_t w8, h8;           /* padded luma size, multiples of 8, at most 16384 */
  int32_t tile_cols_log2;   /* the frame's tiling (see mt_tiling_spec_min) */
  int32_t tile_rows_log2;
  int32_t base_q_idx;       /* frame base qindex 0..255 */
  int32_t bd;               /* 8, 10 or 12 */
  int32_t variance_boost;   /* 1: Variance Boost (octile of the 8x8 variances); 0: classic whole-SB AQ */
  int32_t dark_aq;          /* 1: dark-structure protection (active from base qindex 90) */
  int32_t octile;           /* 1..8 (clamped), 6 by default */
  int32_t boost_only;       /* 1: never coarsen; 0 by default */
  float strength;           /* Variance Boost strength (negative clamps to 0), 1 by default */
} mt_aq_params;

/* One superblock of the grid (AqCell, src/coder/aq.rs:325-342). */
typedef struct mt_aq_cell {
  uint8_t prev;    /* raster-chain qindex before the superblock */
  uint8_t newq;    /* the superblock's qindex */
  int8_t steps;    /* signalled reducedDeltaQIndex, -12..12 */
  uint8_t target;  /* aq_sb_target, the qindex the steps move toward */
} mt_aq_cell;

/* The spec-minimum tiling the reference encodes with (plan_tiling with one
 * target tile, src/coder/tiling.rs:92-136). */
int mt_tiling_spec_min(int32_t w8, int32_t h8, int32_t* cols_log2, int32_t* rows_log2);
/* Device working storage mt_aq_grid_device needs. */
size_t mt_aq_grid_scratch_bytes(const mt_aq_params* prm);
/* The grid on the stream: d_cells holds (ceil(h8/64) x ceil(w8/64)) cells in
 * frame raster order; d_tile_refs (may be NULL) two floats per tile in raster
 * order of tiles: ref_act (tile mean whole-SB log-activity) and ref_pick (tile
 * mean log octile variance). */
int mt_aq_grid_device(const uint16_t* d_luma, const mt_aq_params* prm, mt_aq_cell* d_cells, float* d_tile_refs,
                      void* d_scratch, void* stream);
/* Host-buffer form of mt_aq_grid_device. */
int mt_aq_grid(const uint16_t* luma, const mt_aq_params* prm, mt_aq_cell* cells, float* tile_refs);
/* The dark-protection weight's power for each x: equal to the host C
 * library's powf(x, 1.2f) for every x in (1, 4.5], the range the weight uses
 * (72 / (16 + mean) with mean >= 0, clamped to [1, 4.5] after the power);
 * elsewhere the binary64 power rounded once to binary32. */
int mt_dark_pow_device(const float* d_x, float* d_out, int64_t n, void* stream);

/* ---- Screen-content frame gate ----
 * Replaces screen_frame_gate (src/coder/screen_gate.rs:64-273): per 16x16 luma
 * block the distinct-value histogram (palette-exact / lenient counts,
 * src/coder/palette.rs:651-690), the repeats among the hashes of the aligned
 * non-flat 8x8 blocks, and, when that pre-screen passes, the IntraBC copy-gain
 * model over the hash index of every 8x8 window on the chroma-parity grid
 * (LossyIbcIndex, src/coder/block64.rs:92-330).  Shipped tuning: screen_few_share
 * 0.10, ibc_gate_prescreen 0.02, ibc_gate_dv 1, ibc_gate_beta 32.  The luma
 * plane is the padded source, w8 x h8 u16 row-major. */
typedef struct mt_screen_gate_params {
  int32_t w8, h8;          /* padded luma size, multiples of 8 */
  int32_t sub_x, sub_y;    /* chroma subsampling shifts (the index grid's step) */
  int32_t bd;              /* 8, 10 or 12 */
  int32_t base_q_idx;      /* frame base qindex */
} mt_screen_gate_params;

typedef struct mt_screen_gate_result {
  int32_t ibc_pays;        /* IntraBC is expected to save more than the loop filters it costs */
  int32_t few_colour;      /* enough palette-exact 16x16 blocks for the text palette tools */
  int32_t copy_stage;      /* 1: the pre-screen passed and the copy gains were measured */
  uint32_t blocks16;       /* 16x16 blocks counted, (w8 / 16) * (h8 / 16) */
  uint32_t few16;          /* palette-exact 16x16 blocks (2..8 values spanning >= 64 << (bd - 8)) */
  uint32_t lenient16;      /* 16x16 blocks of 2..16 values with that span */
  uint32_t nonflat8;       /* aligned non-flat 8x8 blocks inside the 16x16 grid */
  uint32_t dup8;           /* of those, hashes already seen */
  uint32_t copied;         /* 16x16 blocks whose best earlier copy gains */
  uint32_t reserved;
  uint64_t gain;           /* summed copy gain (gradient energy units) */
  uint64_t photo;          /* photo-like 8x8 blocks priced as lost deblocking */
} mt_screen_gate_result;

/* At most this many index windows ((w8 - 7) x (h8 - 7) on the chroma-parity
 * grid), else MT_ERR_TOO_LARGE. */
#define MT_SCREEN_MAX_WINDOWS (1u << 26)
/* Device working storage mt_screen_gate_device needs. */
size_t mt_screen_gate_scratch_bytes(const mt_screen_gate_params* prm);
/* The gate on the stream: the block pass, one read of its four counters (the
 * stream is synchronised), the copy stage when the pre-screen passes (a second
 * synchronisation), and the verdicts into the host struct *out. */
int mt_screen_gate_device(const uint16_t* d_luma, const mt_screen_gate_params* prm, void* d_scratch,
                          mt_screen_gate_result* out, void* stream);
/* Host-buffer form. */
int mt_screen_gate(const uint16_t* luma, const mt_screen_gate_params* prm, mt_screen_gate_result* out);

/* Library version string. */
const char* mt_version(void);


/* ---- Entropy coding, tile packing and filter replay (host) ----------------
 * The AV1 multi-symbol range coder of src/odec.rs:35-615 (OdEcEncoder): CDFs
 * are inverse-form u16 arrays whose last entry is the adaptation counter
 * (src/tables.rs:31-35 icdf); a CDF of len entries codes len symbols.
 * mt_range_encoder_* replace OdEcEncoder::{new, encode_bool, encode_symbol,
 * encode_symbol_noupdate, encode_literal, encode_signed_subexp_with_ref, done}
 * (src/odec.rs:236-253, :427-600). */
typedef struct mt_range_encoder mt_range_encoder;
mt_range_encoder* mt_range_encoder_new(int32_t updating_cdf);
void mt_range_encoder_free(mt_range_encoder* e);
int mt_range_encode_bool(mt_range_encoder* e, int32_t value, uint16_t f);
/* adapt != 0: encode_symbol (adapts cdf in place when the encoder updates
 * CDFs); adapt == 0: encode_symbol_noupdate. */
int mt_range_encode_symbol(mt_range_encoder* e, int32_t s, uint16_t* cdf, int32_t len, int32_t adapt);
int mt_range_encode_literal(mt_range_encoder* e, uint32_t value, uint32_t bits);
int mt_range_encode_signed_subexp_with_ref(mt_range_encoder* e, int32_t v, int32_t low, int32_t high, uint32_t k,
                                           int32_t r);
/* Flushes, returns the bytes (free with mt_free) and frees the encoder. */
int mt_range_encoder_done(mt_range_encoder* e, uint8_t** out, size_t* out_len);

/* The frame-initial CDF set Cdfs::new(qctx) (src/coder/cdfs.rs:401-629) as
 * slots in Cdfs::semantic_slots order (src/coder/cdfs.rs:193-355): slot i is
 * data[offsets[i] .. offsets[i] + lens[i]).  With all three arrays NULL only
 * the sizes are returned. */
int32_t mt_cdf_slot_count(void);
/* First slot of each CDF group in that order: a CDF with context k of group g
 * is slot g + k (two-level groups row-major, e.g. kf_y + above * 5 + left,
 * part_split + level * 4 + ctx, uv_mode + cfl_allowed * 13 + y_mode,
 * txsz + cat * 3 + ctx).  Groups a class or plane lacks are -1.  eob_bin is
 * the first of the seventeen eob_pt CDFs in the order 16c 16l 32c 32l 64l
 * 16l1d 64l1d 128l1d 64c 256l 256c 128c 128l 1024l 1024c 512c 512l. */
typedef struct mt_cdf_slot_layout {
  int32_t skip, intrabc, part_bl8, part_split, kf_y, uv_mode, angle_delta, filter_intra, filter_intra_mode;
  int32_t palette_y_mode, palette_y_size, palette_uv_mode, cfl_sign, cfl_alpha, txsz, txtp8, txtp4, txtp16;
  int32_t txb_skip[5];
  int32_t base_tok[5][2], br_tok[4][2], eob_base[5][2], eob_hi[5][2];
  int32_t dc_sign[2];
  int32_t eob_bin, delta_q, wiener_restore, nslots;
} mt_cdf_slot_layout;
int mt_cdf_layout(mt_cdf_slot_layout* out);
int mt_cdfs_default(int32_t qctx, uint16_t* data, size_t data_cap, uint32_t* offsets, uint16_t* lens,
                    int32_t slots_cap, size_t* data_len, int32_t* nslots);

/* One tile's packer: pack_wavefront_tile (src/coder/wavefront.rs:617-657).
 * The superblocks' semantic token streams (EntropyTokens, src/odec.rs:96-108:
 * two tag bits, adaptive symbol (slot << 8 | s), bool (f << 1 | v), gathered
 * partition bool (slot << 2 | split << 1 | top), non-adapting symbol) are
 * replayed in raster order against Cdfs::new(qcat(base_q_idx)) (replay_semantic,
 * src/odec.rs:315-360).  Superblock i's tokens are ops[sb_start[i] ..
 * sb_start[i + 1]) (sb_start has nsb + 1 entries); sb_cdef_point[i] is the
 * index within them of its read_cdef() point, or -1 (NULL: none).  Returns
 * the payload (free with mt_free) and, when trace is non-NULL, the symbol
 * trace the filter replay needs (free with mt_tile_trace_free).  A token that
 * names no slot or a symbol outside its CDF returns MT_ERR_INVALID_INPUT. */
typedef struct mt_tile_trace mt_tile_trace;
int mt_pack_tile(uint8_t base_q_idx, int32_t updating_cdf, const uint32_t* ops, const uint32_t* sb_start,
                 const int32_t* sb_cdef_point, int32_t nsb, uint8_t** payload, size_t* payload_len,
                 mt_tile_trace** trace);
void mt_tile_trace_free(mt_tile_trace* t);
/* replay_tile_with_filters (src/coder/tile_encode.rs:404-466) without loop
 * restoration: the trace re-emitted superblock by superblock in raster order
 * over the tile (x0, y0, w, h), with the 64x64 unit's cdef_idx (cdef_grid,
 * unit_cols per row, cdef_bits wide) as a raw literal at each recorded
 * read_cdef() point; cdef_grid NULL replays the trace as is. */
int mt_replay_tile_with_filters(const mt_tile_trace* t, int32_t tile_x0, int32_t tile_y0, int32_t tile_w,
                                int32_t tile_h, const uint8_t* cdef_grid, int32_t unit_cols, int32_t grid_len,
                                int32_t cdef_bits, int32_t updating_cdf, uint8_t** out, size_t* out_len);
/* mt_pack_tile followed by mt_replay_tile_with_filters in one pass, for a
 * caller that knows each superblock's cdef_idx before packing (the frame's
 * filters already decided): superblock i's sb_cdef_idx[i] (< 2^cdef_bits) is
 * coded as a raw literal at its read_cdef() point, the symbol sequence
 * replay_tile_with_filters would produce over a tile whose 64x64 units are
 * its superblocks (same bytes), with no trace kept.  cdef_bits 0 packs as
 * mt_pack_tile does. */
int mt_pack_tile_filtered(uint8_t base_q_idx, int32_t updating_cdf, const uint32_t* ops, const uint32_t* sb_start,
                          const int32_t* sb_cdef_point, int32_t nsb, const uint8_t* sb_cdef_idx, int32_t cdef_bits,
                          uint8_t** payload, size_t* payload_len);
/* Frees a buffer this library returned. */
void mt_free(void* p);


/* ---- Headers and container (host) ----------------------------------------
 * src/bitwriter.rs leb128, src/obu.rs wrap_obu / sequence_header_cicp(_ss) /
 * sequence_header_mono / frame_header_lossy_multitile(_th),
 * src/coder/frame_encode.rs:436-525 assemble_tilegroup / assemble_frame_obus,
 * src/coder/tiling.rs:63-136 the increment bits of a tiling, and
 * src/isobmff.rs:68-494 wrap_av1_image with src/avif.rs:676-740 make_av1c. */
typedef struct mt_sequence_header_params {
  uint32_t width, height;          /* displayed frame size */
  uint32_t profile;                /* 0 (4:2:0 / mono), 1 (4:4:4), 2 (4:2:2 or 12-bit) */
  uint32_t bit_depth;              /* 8, 10, 12 */
  int32_t monochrome;              /* 1: the monochrome header (sequence_header_mono) */
  int32_t color_present;           /* CICP colour description present */
  uint32_t primaries, transfer, matrix; /* CICP code points (matrix 0 = identity / RGB) */
  int32_t full_range;
  uint32_t chroma_sample_position; /* coded for 4:2:0 */
  uint32_t ss_x, ss_y;             /* chroma subsampling */
  int32_t enable_filter_intra, enable_intra_edge_filter;
} mt_sequence_header_params;

typedef struct mt_frame_header_params {
  int32_t w8, h8;                  /* padded frame size (for the tiling's increment bits) */
  int32_t tile_cols_log2, tile_rows_log2;
  uint32_t base_q_idx;             /* 1..255 (lossy) */
  uint32_t qm_y, qm_u, qm_v;       /* 0..15; all 15 = no quantisation matrices */
  int32_t uac_delta, udc_delta;    /* chroma AC / DC qindex deltas */
  int32_t monochrome;
  int32_t aq;                      /* superblock delta-q present */
  uint32_t delta_q_res_log2;
  int32_t allow_intrabc;
  int32_t updating_cdf;            /* 0: disable_cdf_update */
  int32_t lf_y, lf_u, lf_v, lf_sharpness; /* loop-filter levels and sharpness */
  int32_t cdef_bits;               /* -1: CDEF off (the no-op parameter set) */
  int32_t cdef_damping;            /* 3..6 */
  uint8_t cdef_strengths[8][4];    /* (y pri, y sec, uv pri, uv sec); sec 0, 1, 2 or 4 */
  int32_t lr_luma_wiener;          /* 1: luma RESTORE_WIENER */
} mt_frame_header_params;

typedef struct mt_avif_item_params {
  uint32_t width, height;
  uint8_t bit_depth, channels;     /* channels 3 colour, 1 monochrome */
  uint8_t seq_profile, seq_level_idx; /* av1C (mt_av1_level_for) */
  int32_t monochrome, chroma_sub_x, chroma_sub_y;
  int32_t color_present;           /* nclx colr box */
  uint16_t primaries, transfer, matrix;
  int32_t full_range;
  const uint8_t* icc; size_t icc_len;   /* prof colr box, or NULL */
  const uint8_t* exif; size_t exif_len; /* Exif item (TIFF bytes), or NULL */
  uint8_t irot_steps;              /* 0..3 anti-clockwise quarter turns */
  int32_t imir_axis;               /* -1 none, 0 vertical axis, 1 horizontal axis */
  int32_t clli_present;
  uint16_t max_content_light_level, max_pic_average_light_level;
} mt_avif_item_params;

/* leb128 bytes of value (out NULL: only the length). */
int mt_leb128(uint64_t value, uint8_t* out, size_t cap, size_t* len);
/* An OBU with obu_has_size_field = 1 around payload. */
int mt_wrap_obu(int32_t obu_type, const uint8_t* payload, size_t n, uint8_t** out, size_t* out_len);
/* The increment_tile_{cols,rows}_log2 bits (each at most 8) that signal a tiling. */
int mt_tiling_increments(int32_t w8, int32_t h8, int32_t tile_cols_log2, int32_t tile_rows_log2, uint8_t* cols_incr,
                         int32_t* ncols, uint8_t* rows_incr, int32_t* nrows);
/* The sequence header OBU. */
int mt_sequence_header(const mt_sequence_header_params* p, uint8_t** out, size_t* out_len);
/* The uncompressed frame header bits (with trailing bits when trailing != 0). */
int mt_frame_header(const mt_frame_header_params* p, int32_t trailing, uint8_t** out, size_t* out_len);
/* One OBU_FRAME for a single tile, else OBU_FRAME_HEADER + OBU_TILE_GROUP
 * (tile sizes as 4-byte little-endian tile_size_minus_1). */
int mt_assemble_frame_obus(const mt_frame_header_params* p, const uint8_t* const* tiles, const size_t* tile_lens,
                           int32_t ntiles, uint8_t** out, size_t* out_len);
/* temporal delimiter + sequence header + frame OBUs (src/dispatch.rs:239-256). */
int mt_av1_stream(const mt_sequence_header_params* sp, const mt_frame_header_params* fp, const uint8_t* const* tiles,
                  const size_t* tile_lens, int32_t ntiles, uint8_t** out, size_t* out_len);
/* seq_level_idx for a picture size (AV1 Table A.2 thresholds). */
uint8_t mt_av1_level_for(uint32_t width, uint32_t height);
/* The AVIF file around an AV1 stream (free with mt_free). */
int mt_wrap_av1_image(const uint8_t* obu, size_t obu_len, const mt_avif_item_params* p, uint8_t** out,
                      size_t* out_len);


/* ---- Encode configuration (the drop-in boundary's EncodeConfig) -----------
 * Every EncodeConfig field (src/avif.rs:257-316) except the gain map;
 * mt_encode_config_default gives EncodeConfig::default() (src/avif.rs:318-344:
 * quality 80, 4:2:0, sRGB-YCbCr CICP, all cores, Slow, adaptive CDFs, AQ with
 * Variance Boost and dark protection, CDEF flag off (Slow forces it on),
 * Wiener off, quantisation matrices on, screen content and IntraBC allowed). */
#define MT_CHROMA_420 0
#define MT_CHROMA_422 1
#define MT_CHROMA_444 2
#define MT_CHROMA_MONO 3
#define MT_SPEED_EXTRA_SLOW 0
#define MT_SPEED_SLOW 1
#define MT_SPEED_MEDIUM 2
#define MT_SPEED_FAST 3
typedef struct mt_encode_config {
  int32_t quality;                 /* 0..100 */
  int32_t chroma;                  /* MT_CHROMA_* */
  int32_t color_present;           /* color_encoding: Some(Cicp) */
  uint32_t primaries, transfer, matrix;
  int32_t full_range;
  uint32_t chroma_sample_position;
  const uint8_t* icc; size_t icc_len;
  int32_t orientation;             /* metadata: EXIF orientation 1..8 */
  int32_t clli_present;            /* metadata: content light level */
  uint16_t max_content_light_level, max_pic_average_light_level;
  const uint8_t* exif; size_t exif_len;
  int32_t threads;                 /* 0 = all cores */
  int32_t speed;                   /* MT_SPEED_* */
  int32_t updating_cdf, adaptive_quant, variance_boost, dark_aq, cdef, wiener;
  int32_t quantization_matrices, screen_content, intrabc;
  int32_t qmatrix_level;           /* -1 = None, else 0..15 */
  int32_t alpha_quality;           /* -1 = None, else 0..100 */
} mt_encode_config;

/* The frame-level settings a validated config resolves to: quality_to_q, the
 * QM levels of EncodeConfig::vb (src/avif.rs:543-575), cdef_enabled
 * (src/avif.rs:449-451), the AQ switches. */
typedef struct mt_encode_plan {
  uint8_t base_q_idx;
  uint8_t qm_y, qm_u, qm_v;
  int32_t sub;                     /* 0 4:4:4 / mono, 1 4:2:2, 2 4:2:0 */
  int32_t cdef, aq, variance_boost, dark_aq;
} mt_encode_plan;

int mt_encode_config_default(mt_encode_config* cfg);
/* EncodeConfig::validate (src/avif.rs:577-592): MT_ERR_INVALID_QUALITY for a
 * quality or alpha quality above 100 or a QM level above 15. */
int mt_encode_config_validate(const mt_encode_config* cfg);
/* encode_rgb8's input checks (src/avif.rs:915-923, :593-635): dimensions
 * 1..=16383 (MT_ERR_INVALID_DIMENSIONS), a buffer size that does not overflow
 * (MT_ERR_DIMENSION_TOO_LARGE), rgb_len == width * height * 3
 * (MT_ERR_INVALID_INPUT). */
int mt_validate_rgb8_input(uint32_t width, uint32_t height, size_t rgb_len);
int mt_encode_config_effective(const mt_encode_config* cfg, mt_encode_plan* out);


/* ---- Coefficient token emission (device) ----------------------------------
 * The square 2-D coefficient coders of src/coeffs.rs (encode_tx4_luma_coeffs_adapt
 * :2414, encode_4x4_chroma_coeffs :2310, encode_tx8_coeffs_adapt :583,
 * encode_tx16_coeffs_adapt :707) batched over transform blocks, writing the
 * semantic tokens mt_pack_tile replays (slots of mt_cdf_layout).  A block's
 * levels are cf[x * n + y] (column-major, the reference's layout) at
 * levels + cf_offset. */
typedef struct mt_coef_block {
  uint32_t cf_offset;   /* first of the n * n levels */
  uint8_t log2n;        /* 2, 3, 4: TX_4X4, TX_8X8, TX_16X16 */
  uint8_t plane;        /* 0 luma, 1 chroma */
  uint8_t skip_ctx;     /* txb_skip context 0..12 */
  uint8_t dcs_ctx;      /* dc_sign context 0..2 */
  uint8_t y_mode;       /* luma: the tx-type CDF row */
  uint8_t txtp;         /* luma: tx-type symbol in the class's intra set */
  uint8_t code_txtp;    /* luma: 1 codes the tx-type symbol (the 2-D class's) */
  uint8_t tx_class;     /* 0 the 2-D class; 1 V_DCT, 2 H_DCT (luma TX_4X4 / TX_8X8: encode_tx{4,8}_coeffs_1d,
                         * src/coeffs.rs:109-420, their own scan, contexts and eob CDF) */
} mt_coef_block;
/* Device form, two calls on the stream: with d_tokens NULL it counts each
 * block's tokens into d_counts and writes the n + 1 exclusive offsets
 * (d_offsets[n] = total); with d_tokens (>= total entries) it writes the
 * tokens of block i at d_tokens + d_offsets[i] and its coefficient context
 * byte (cul | dc-sign bits, 0x40 for an all-zero block) to d_res_ctx[i]. */
int mt_emit_coeffs_device(const int32_t* d_levels, const mt_coef_block* d_blocks, int32_t n, uint32_t* d_counts,
                          uint32_t* d_offsets, uint32_t* d_tokens, uint8_t* d_res_ctx, void* stream);
/* Host form: *tokens (free with mt_free) and offsets (n + 1 entries). */
int mt_emit_coeffs(const int32_t* levels, size_t nlevels, const mt_coef_block* blocks, int32_t n, uint32_t** tokens,
                   uint32_t* offsets, uint8_t* res_ctx);


/* ---- End-to-end encode ------------------------------------------------------
 * encode_rgb8 (src/avif.rs:915-940) for 8-bit RGB: the encode_rgb8 input
 * checks and EncodeConfig validation, Q13 colour conversion and padding, the
 * decisions below on the device, and the reference's coefficient and block
 * syntax, adaptive range coder, loop-filter levels, CDEF strength search with
 * its cdef_idx replay, sequence / frame headers and AVIF container.  The
 * decisions are NOT the reference's decode_sb search: every superblock is
 * split down to 8x8 blocks, each taking the lowest-RD-cost (13 intra modes at
 * angle delta 0) x (7 intra transform types) luma candidate of the candidate
 * chain, chroma UV_DC_PRED / DCT_DCT; the output is therefore a valid AVIF
 * with this library's own decisions, not the reference's bytes.  4:2:0 and
 * 4:4:4 (else MT_ERR_UNSUPPORTED_CHROMA_FORMAT).  The frame is coded in the
 * reference's spec-minimum uniform tiling (mt_tiling_spec_min: one tile up to
 * 64 superblocks wide and 2304 in area, e.g. 1 x 2 tiles at 4096x4096), the
 * tiles' decisions and range coding independent.  *out is freed with mt_free. */
int mt_encode_rgb8(const uint8_t* rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg, uint8_t** out,
                   size_t* out_len);
/* What one encode call did, for measurement: the bytes it copied between the
 * host and the device in each direction, the kernels of this library it
 * launched, the semantic tokens it range coded, and device times (CUDA events
 * on its stream) of the block-decision kernel and of the whole call. */
typedef struct mt_encode_stats {
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint32_t kernel_launches;
  uint32_t tokens;
  uint32_t blocks;          /* 8x8 blocks decided */
  uint32_t levels;          /* dependency levels of those blocks (the critical path) */
  float blocks_ms;
  float call_ms;
} mt_encode_stats;

/* The same, also returning the decoder's output planes (padded sizes of
 * mt_padded_plane_dims, after deblocking and CDEF) when recon_out is non-NULL
 * and the call's measurements when stats is non-NULL. */
int mt_encode_rgb8_ex(const uint8_t* rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg,
                      uint8_t** out, size_t* out_len, uint16_t* recon_out[3], mt_encode_stats* stats);
/* mt_encode_rgb8 with the interleaved RGB already in device memory (d_rgb,
 * width * height * 3 bytes); the AVIF comes back in host memory as from
 * mt_encode_rgb8.  No counterpart in the reference, whose input is always in
 * host memory. */
int mt_encode_rgb8_device(const uint8_t* d_rgb, uint32_t width, uint32_t height, const mt_encode_config* cfg,
                          uint8_t** out, size_t* out_len, mt_encode_stats* stats);
/* mt_encode_rgb8 of n images (1..64) in one call: each image set up on a
 * stream of its own, the 8x8 decisions of all of them in ONE persistent launch
 * (their blocks merged level by level into one dependency-ordered ticket
 * queue, so blocks of different images run side by side), then each image's
 * syntax, filters, range coding and container on a host thread of its own.
 * Image i's bytes are those of encoding it alone; rcs[i] (when non-NULL)
 * receives its code, and the call returns the first failing code or MT_OK.
 * Images may differ in size and configuration.  No counterpart in the
 * reference, which encodes one image per call. */
int mt_encode_rgb8_batch(int32_t n, const uint8_t* const* rgb, const uint32_t* widths, const uint32_t* heights,
                         const mt_encode_config* cfgs, uint8_t** outs, size_t* out_lens, int32_t* rcs,
                         mt_encode_stats* stats);
/* The encode calls of a device reuse its device buffers (one set per image
 * of the largest batch seen, each grown to the largest frame it carried; a
 * call that finds them taken by another thread's call allocates its own).  This frees every device's set; the next call
 * allocates again.  No counterpart in the reference, whose buffers are host
 * memory freed per call. */
void mt_encode_release_buffers(void);
/* The same encode from 8-bit Y, U, V planes (chroma at ((w + sx) >> sx) x
 * ((h + sy) >> sy)), without colour conversion: the planes are coded as
 * given and described by the config's CICP (e.g. identity for G, B, R). */
int mt_encode_yuv8(const uint8_t* y, const uint8_t* u, const uint8_t* v, uint32_t width, uint32_t height,
                   const mt_encode_config* cfg, uint8_t** out, size_t* out_len, uint16_t* recon_out[3]);

#ifdef __cplusplus
}
#endif
#endif /* MAROONTREE_B200_H */
