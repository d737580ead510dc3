/*
 * Oracle: CPU restatement of the reference's intra RD kernels, used ONLY as the
 * checker of the CUDA path (tests, smoke, the bench's CPU-baseline leg).  It is
 * test infrastructure, not part of the product; nothing in maroontree_b200/
 * links or calls it.
 *
 * Each function follows the reference (awxkee/maroontree) file:line named in
 * its comment, in the arithmetic order of the x86-64 build with AVX2+FMA
 * detected at run time (the AVX2 float sites are named where they differ from
 * the scalar Rust).  Integer arithmetic wraps (built with -fwrapv) like Rust
 * release builds; floats are IEEE binary32 without contraction
 * (-ffp-contract=off) except where the AVX2 reference uses an explicit FMA.
 */
#ifndef MT_ORACLE_H
#define MT_ORACLE_H
#include <stdint.h>
#include "../include/maroontree_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The CDF groups the coefficient coders touch, as semantic slot numbers. */
typedef struct or_emit_slots {
  int32_t txb_skip[4], base_tok[4][2], br_tok[4][2], eob_base[4][2], eob_hi[4][2], dc_sign[2];
  int32_t eob_bin, txtp4, txtp8, txtp16;
} or_emit_slots;
/* src/coeffs.rs coefficient coders over a block list (tokens of src/odec.rs:96-108). */
int or_emit_coeffs(const int32_t* levels, const mt_coef_block* blocks, int32_t n, const or_emit_slots* S,
                   uint32_t* tokens, size_t cap, uint32_t* offsets, uint8_t* res_ctx);

int or_quant_init(uint8_t base_q_idx, uint8_t bd, uint8_t qm_level, mt_quant* out);
int or_quant_init_chroma(uint8_t base_q_idx, int32_t dc_delta, int32_t ac_delta, uint8_t bd,
                         uint8_t qm_level, mt_quant* out);
const uint8_t* or_qm_row(int32_t qm_level, int32_t chroma, int32_t w, int32_t h);
const uint16_t* or_default_scan(int32_t n);

/* dct.rs: forward transform + quantisation of one n x n block (n = 8). */
void or_dct1d(int32_t* buf, int32_t n);
/* partition_search.rs proxy_mode_beam's ranking (11 nd_modes by satd_sad_proxy). */
int or_mode_beam(const uint16_t* src, const uint16_t* recon, const mt_chain_params* p, const mt_block8* blocks,
                 int32_t nblocks, uint64_t* scores, uint8_t* modes);
void or_fwd_txfm_quant(const int32_t* resid, int32_t tx_type, int32_t n, const mt_quant* q,
                       const uint8_t* qm_row, int32_t* levels, float* targets);
/* idct.rs: dequantisation + inverse transform of one block. */
void or_inv_txfm_dequant(const int32_t* levels, int32_t tx_type, int32_t n, const mt_quant* q,
                         const uint8_t* qm_row, int32_t* resid);
/* trellis.rs:944 trellis_optimize (AVX2 step-A order). */
void or_trellis_optimize(int32_t* cf, const float* tf, float dc_q, float ac_q,
                         const uint16_t* scan, int32_t n, float lambda0);
/* intrapred.rs:1357 intra_predict_nd_ad_impl (non-DC modes) and :1740 dc_pred. */
void or_intra_predict(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t bw,
                      int32_t bh, int32_t mode, int32_t angle_delta, int32_t have_tr,
                      int32_t have_bl, int32_t fw, int32_t fh, int32_t filter_type, int32_t bd,
                      int32_t* out);
int32_t or_dc_pred(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t w,
                   int32_t h, int32_t bd);
/* partition_rd.rs:86 luma_satd_scalar. */
uint64_t or_luma_satd(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w,
                      int32_t h, int32_t max_value, const int32_t* pred, const int32_t* resid);
/* cost.rs:156 cost_q_table / cdf_cost_with_table. */
float or_cdf_cost(const uint16_t* cdf, int32_t s);
/* rate.rs:149 real_block_bits_bounded (bound = +inf) for a square luma block. */
float or_real_block_bits(const int32_t* cf, const uint16_t* scan, int32_t n, int32_t cls,
                         const mt_coef_cdfs* cdfs, int32_t skip_ctx, int32_t dcs_ctx,
                         int32_t y_mode, int32_t txtp, int32_t use_skip_bits,
                         const float* skip_bits);
/* rate.rs:149 real_block_bits_bounded for any w x h (txtp_mode < 0: no txtp symbol). */
float or_real_block_bits_wh(const int32_t* cf, const uint16_t* scan, int32_t w, int32_t h,
                            const mt_coef_cdfs* cdfs, int32_t skip_ctx, int32_t dcs_ctx, int32_t txtp_mode,
                            int32_t txtp, int32_t use_skip_bits, const float* skip_bits);
/* rate.rs:58 CoefCostTables::build and the other per-symbol costs. */
void or_coef_costs_build(const mt_coef_cdfs* cdfs, mt_coef_costs* out);
/* The candidate chain of partition_search.rs:467-530, per candidate. */
int or_candidate_chain(const uint16_t* src, const uint16_t* recon, const mt_chain_params* prm,
                       const mt_quant* quant, const uint8_t* qm_row, const mt_coef_cdfs* cdfs,
                       const mt_candidate* cands, int32_t n, mt_candidate_result* results,
                       int32_t* levels_out, int32_t* recon_out, int32_t threads);

/* encoder.rs CSC + dispatch.rs padding: interleaved RGB -> padded Y/Cb/Cr
 * (sub 0 = 4:4:4, 2 = 4:2:0). */
int or_csc_rgb8(const uint8_t* rgb, int32_t w, int32_t h, int32_t sub, uint16_t* y, uint16_t* cb, uint16_t* cr);
/* loopfilter.rs filter_plane (scalar path, per superblock row order). */
int or_deblock_plane(uint16_t* px, int32_t w, int32_t h, int32_t vis_w, int32_t vis_h, const uint8_t* bw4,
                     const uint8_t* bh4, const uint8_t* vedge4, const uint8_t* hedge4, int32_t nc4, int32_t level,
                     int32_t sharp, int32_t is_luma, int32_t sb_rows4, int32_t bd);
void or_loop_filter_levels(int32_t base_q_idx, int32_t sub, int32_t* lvl_y, int32_t* lvl_uv, int32_t* sharp);
int or_deblock_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint8_t* blk4, const uint8_t* blk4h,
                     const uint8_t* blk4v, const uint8_t* blk4t, const uint8_t* pblk4, const uint8_t* pblk4h,
                     const mt_deblock_frame_params* g, int32_t lvl_y, int32_t lvl_u, int32_t lvl_v);
/* frame_cdef.rs frame_cdef: tables (optional outputs), decision, apply in place. */
int or_cdef_frame(uint16_t* y, uint16_t* u, uint16_t* v, const uint16_t* sy, const uint16_t* su, const uint16_t* sv,
                  const uint8_t* skip8, const mt_cdef_params* prm, mt_cdef_decision* out, uint8_t* grid,
                  int64_t* luma_tab, int64_t* u_tab, int64_t* v_tab, uint8_t* dirs, int32_t* vars);
float or_weighted_sse(const int32_t* err, int32_t w, int32_t h);
float or_cdef_frame_lambda(int32_t qidx, int32_t bd, int32_t sub_x, int32_t sub_y);
/* rd_sse.rs sse_recon (plain or weighted decision distortion) of n blocks. */
int or_sse_recon(const uint16_t* src, int32_t stride, int32_t vis_w, int32_t vis_h, int32_t bd, const uint16_t* pos,
                 const int32_t* pred, const int32_t* resid, int32_t n, int32_t w, int32_t h, float scale, int64_t* out);
/* aq_common.rs / coder/aq.rs / lossy_state.rs: the adaptive-quantisation grid and its pieces. */
float or_fast_round(float x);
float or_dirty_log1pf(float d);
void or_dark_pow(const float* x, float* out, int64_t n);
int32_t or_dark_protection(int32_t enabled, int32_t base_q, const uint16_t* yp, int32_t pw, int32_t sb_y, int32_t sb_x,
                           int32_t width, int32_t height, float scale);
int or_tiling_spec_min(int32_t w8, int32_t h8, int32_t* cols_log2, int32_t* rows_log2);
int or_aq_grid(const uint16_t* luma, const mt_aq_params* p, mt_aq_cell* cells, float* refs_out);
/* screen_gate.rs screen_frame_gate; block64.rs hash8. */
int or_screen_gate(const uint16_t* luma, const mt_screen_gate_params* p, mt_screen_gate_result* out);
uint32_t or_hash8(const uint16_t* luma, int32_t w, int32_t x, int32_t y);
/* trellis.rs:55 trellis_optimize_ctx (shipped tuning) of a square luma block. */
void or_trellis_optimize_ctx(int32_t* cf, const float* tf, float dc_q, float ac_q, const uint16_t* scan, int32_t w,
                             float lambda0, const mt_coef_cdfs* cdfs, int32_t dcs_ctx, const uint8_t* qm,
                             int32_t qm_level, float band_tilt);
/* rate.rs:149 real_block_bits_bounded with its exact abort bound. */
float or_real_block_bits_bounded(const int32_t* cf, const uint16_t* scan, int32_t w, int32_t h,
                                 const mt_coef_cdfs* cdfs, int32_t skip_ctx, int32_t dcs_ctx, int32_t txtp_mode,
                                 int32_t txtp, int32_t use_skip_bits, const float* skip_bits, float bound);
/* lossy_state.rs:876 / :1010 luma_bits_1d_8x8 / _4x4 (V_DCT, H_DCT). */
float or_luma_bits_1d(const int32_t* cf, int32_t w, int32_t vertical, const mt_coef_cdfs* cdfs, int32_t dcs,
                      int32_t y_mode);
/* lossy_state.rs:630 coef_res_ctx. */
uint8_t or_coef_res_ctx(const int32_t* cf, const uint16_t* scan, int32_t n);
/* partition_search.rs:4235 split16_luma_try over a batch of jobs. */
int or_split16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                    const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                    mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out, int32_t threads);
/* partition_search.rs:4524 split16_depth2_try over a batch of jobs. */
int or_split16_depth2(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                      const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                      mt_split16_d2_result* results, int32_t* cf_out, uint16_t* rec_out, int32_t threads);
/* intrapred.rs:1112-1258 cfl_ac_sub / cfl_ac_444 + cfl_best_alpha over a batch of chroma blocks. */
int or_cfl_alpha(const uint16_t* luma, int32_t luma_stride, const uint16_t* src_u, const uint16_t* src_v,
                 int32_t chroma_stride, int32_t sub_x, int32_t sub_y, int32_t cw, int32_t ch, int32_t vis_cw,
                 int32_t vis_ch, int32_t bd, const mt_cfl_block* blocks, int32_t n, int8_t* alpha, int32_t* ac_out);
/* intrapred.rs:473-565 filter_intra_predict; superblock.rs:356-400 rank_filter_intra_modes. */
void or_filter_intra_predict(const uint16_t* recon, int32_t stride, int32_t ox, int32_t oy, int32_t w, int32_t h,
                             int32_t mode, int32_t bd, int32_t* out);
int or_filter_intra_beam(const uint16_t* src, const uint16_t* recon, int32_t stride, int32_t frame_w, int32_t frame_h,
                         int32_t vis_w, int32_t vis_h, int32_t bd, int32_t w, int32_t h, const uint16_t* pos,
                         int32_t n, uint64_t* scores, uint8_t* modes, int16_t* preds);
/* block8.rs:157 split4tx_try over a batch of 8x8 jobs. */
int or_split4tx(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_split16_job* jobs, int32_t n,
                mt_split16_result* results, int32_t* cf_out, uint16_t* rec_out);
/* block8.rs:689-1404 pick_block8: the mode loop's candidates (refine 0) or the winner's type refinement (1). */
int or_leaf8(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
             const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
             mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);
/* partition_search.rs pick_luma16: the mode loop's candidates (refine 0, :4802-4880) or the winner's type
 * refinement (1, :5252-5474). */
int or_leaf16(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
              const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_leaf8_job* jobs, int32_t n, int32_t refine,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);
/* block64.rs rd_pick_luma64's four-TX_32X32 leg (:1906-1958) per (64x64 block, mode, delta). */
int or_quad32_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                   const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_quad32_job* jobs, int32_t n,
                   mt_quad32_result* results);
/* block64.rs rd_pick_luma64's tx_depth-2 trial (:1983-2010, grid16_luma_pass :1670-1805) per (64x64 block,
 * mode, delta); cf_out (optional): n x 4096, transform t's levels at t * 256. */
int or_grid16_luma(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
                   const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_grid16_job* jobs, int32_t n,
                   mt_grid16_result* results, int32_t* cf_out);
/* lossy_state.rs uv_mode_bits (:1302-1349) from the mode CDFs. */
float or_uv_mode_bits(const mt_uv_mode_cdfs* c, int32_t y_mode, int32_t uv_mode, int32_t cfl, int32_t alpha_u,
                      int32_t alpha_v);
/* block16.rs pick_uv16_420 (:980-1381) with the shipped tuning, per 16x16 leaf. */
int or_pick_uv16_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc, const mt_uv16_job* jobs,
                     int32_t n, mt_uv16_result* results, int32_t* cf_out, uint16_t* rec_out);
/* block16.rs pick_uv16_444 (:437-978) with the shipped tuning, per 16x16 leaf. */
int or_pick_uv16_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv16_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out);
/* block32.rs pick_uv32_420 (:2797-3120) with the shipped tuning, per 32x32 leaf. */
int or_pick_uv32_420(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv16_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out);
/* block32.rs pick_uv32_444 (:2264-2720) with the shipped tuning, per 32x32 leaf. */
int or_pick_uv32_444(const uint16_t* src_u, const uint16_t* src_v, const uint16_t* rec_u, const uint16_t* rec_v,
                     const uint16_t* luma, const mt_split16_params* p, const mt_uv16_params* u, const mt_quant* q,
                     const uint8_t* qm, const mt_coef_cdfs* cd, const mt_uv_mode_cdfs* mc,
                     const mt_uv32_444_job* jobs, int32_t n, mt_uv16_result* results, int32_t* cf_out,
                     uint16_t* rec_out);
/* palette.rs exact_uv_palette / uv_pair_histogram / lossy_uv_palette_from_hist + the UV index map. */
int or_uv_palette(const uint16_t* su, const uint16_t* sv, int32_t stride, int32_t w, int32_t h, const uint16_t* pos,
                  int32_t n, const mt_palette_opts* opts, mt_uv_palette_cand* cands, uint8_t* maps);
/* dct1d_32_i32 in place on 32 values. */
void or_dct1d_32(int32_t* buf);
/* block32.rs pick_luma32: the mode loop's candidates (:776-836, TX_32X32 DCT_DCT). */
int or_leaf32(const uint16_t* src, const uint16_t* recon, const mt_split16_params* p, const mt_quant* q,
              const uint8_t* qm, const mt_coef_cdfs* cdfs, const mt_leaf8_job* jobs, int32_t n,
              mt_leaf8_result* results, int32_t* cf_out, uint16_t* rec_out);
float or_scaled_trellis_lambda(float dc_q, float ac_q, float lambda0);
int or_edge_filter_strength(int w, int h, int filter_type, int delta);
int or_use_edge_upsample(int w, int h, int filter_type, int delta);

/* palette.rs / kmeans.rs lossy luma palette candidates and their parts (oracle_palette.cpp). */
int or_luma_palette(const uint16_t* src, int32_t stride, int32_t frame_w, int32_t frame_h, int32_t bd, int32_t w,
                    int32_t h, const uint16_t* pos, int32_t n, const mt_palette_opts* opts, mt_palette_cand* cands,
                    uint8_t* maps);
void or_block_color_histogram(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                              int32_t* vals, uint32_t* counts, int32_t* n_out);
void or_dp_palette_center_sets(const int32_t* vals, const uint32_t* counts, int32_t n, int32_t kmax, int32_t* sets,
                               int32_t* lens);
void or_luma_nearest_indices(const uint16_t* src, int32_t stride, int32_t px, int32_t py, int32_t w, int32_t h,
                             const int32_t* centers, int32_t n, uint8_t* out);
void or_palette_color_ctx_nb(int32_t l, int32_t u, int32_t ul, int32_t cur, int32_t* ctx, int32_t* sym);
void or_palette_color_ctx(const uint8_t* map, int32_t stride, int32_t y, int32_t x, int32_t* ctx, int32_t* sym);
float or_dirty_log2f(float d);

#ifdef __cplusplus
}
#endif
#endif
