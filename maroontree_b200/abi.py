"""ctypes mirror of ``include/maroontree_b200.h`` plus numpy record dtypes for the
batched arrays.  Loads the in-tree ``_lib/libmaroontree_b200.so``; there is no
fallback, a missing library raises."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libmaroontree_b200.so")

MT_OK = 0
MT_ERR_INVALID_INPUT = -2
MT_ERR_UNSUPPORTED = -3
MT_ERR_TOO_LARGE = -4
MT_NOALLOC_MAX_BLOCKS = 131072
MT_LEVEL_MAX_COMBOS = 2048
MT_ERR_INVALID_QUALITY = -22
MT_ERR_DIMENSION_TOO_LARGE = -21
MT_ERR_INVALID_DIMENSIONS = -20
MT_ERR_DEVICE = -10
MT_ERR_ALLOC = -11
MT_EOB_INVALID = -2

# intra modes (src/intrapred.rs:54-79)
DC_PRED, V_PRED, H_PRED, D45_PRED, D135_PRED, D113_PRED, D157_PRED, D203_PRED, D67_PRED = range(9)
SMOOTH_PRED, SMOOTH_V_PRED, SMOOTH_H_PRED, PAETH_PRED = 9, 10, 11, 12
# 7-type intra transform set order (src/cost.rs:100-103)
TX_IDTX, TX_DCT_DCT, TX_V_DCT, TX_H_DCT, TX_ADST_ADST, TX_ADST_DCT, TX_DCT_ADST = range(7)
TX_2D_SCAN_TYPES = (TX_IDTX, TX_DCT_DCT, TX_ADST_ADST, TX_ADST_DCT, TX_DCT_ADST)

CAND_HAVE_TR, CAND_HAVE_BL, CAND_FILTER_TYPE, CAND_NO_TRELLIS = 1, 2, 4, 8
COMBO_NO_TRELLIS = 1


class Quant(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "dc_q", "ac_q", "q_mult_dc", "q_mult_ac", "rmin", "rmax", "cmin", "cmax", "cf_max",
        "qm_level", "qm_chroma", "qidx")]


class CoefCdfs(C.Structure):
    _fields_ = [
        ("txb_skip", (C.c_uint16 * 2) * 13),
        ("base_tok", (C.c_uint16 * 4) * 42),
        ("br_tok", (C.c_uint16 * 4) * 21),
        ("eob_base", (C.c_uint16 * 3) * 4),
        ("eob_hi", (C.c_uint16 * 2) * 11),
        ("eob_bin", C.c_uint16 * 11),
        ("dc_sign", (C.c_uint16 * 2) * 3),
        ("txtp", (C.c_uint16 * 16) * 13),
        ("eob_bin_1d", C.c_uint16 * 11),
    ]


class CoefCosts(C.Structure):
    _fields_ = [
        ("txb_skip", (C.c_float * 2) * 13),
        ("base_tok", (C.c_float * 4) * 42),
        ("br_cum", (C.c_float * 13) * 21),
        ("eob_base", (C.c_float * 3) * 4),
        ("eob_hi", (C.c_float * 2) * 11),
        ("eob_bin", C.c_float * 11),
        ("dc_sign", (C.c_float * 2) * 3),
        ("txtp", (C.c_float * 16) * 13),
        ("eob_bin_1d", C.c_float * 11),
    ]


class ChainParams(C.Structure):
    _fields_ = [
        ("tx_size", C.c_int32), ("bd", C.c_int32), ("frame_w", C.c_int32), ("frame_h", C.c_int32),
        ("stride", C.c_int32), ("trellis_lambda0", C.c_float), ("mode_lambda", C.c_float),
        ("satd_scale", C.c_float), ("satd_bridge", C.c_float), ("use_skip_bits", C.c_int32),
        ("skip_bits", C.c_float * 2), ("vis_w", C.c_int32), ("vis_h", C.c_int32),
    ]


class Split16Params(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("frame_w", "frame_h", "stride", "bd", "vis_w", "vis_h")] + [
        (n, C.c_float) for n in ("trellis_lambda0", "rd_lambda", "band_tilt", "wsse_scale")] + [
        (n, C.c_int32) for n in ("tx_search", "tx_guard_shift", "use_skip_bits")] + [
        ("skip_bits", (C.c_float * 2) * 13)]


assert C.sizeof(Split16Params) == 156


class UvModeCdfs(C.Structure):
    """mt_uv_mode_cdfs."""
    _fields_ = [("uv_mode", (C.c_uint16 * 14) * 13), ("angle_delta", (C.c_uint16 * 7) * 8),
                ("cfl_sign", C.c_uint16 * 8), ("cfl_alpha", (C.c_uint16 * 16) * 6)]


class UvModeCosts(C.Structure):
    """mt_uv_mode_costs."""
    _fields_ = [("uv_mode", (C.c_float * 14) * 13), ("angle_delta", (C.c_float * 7) * 8),
                ("cfl_sign", C.c_float * 8), ("cfl_alpha", (C.c_float * 16) * 6)]


class Uv16Params(C.Structure):
    """mt_uv16_params."""
    _fields_ = [(n, C.c_int32) for n in ("luma_stride", "joint_k", "angle_deltas")] + [("dir_lambda", C.c_float)]


UV_CFL_PRED = 13
UV16_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("y_mode", "u1"), ("flags", "u1"),
                           ("a_coef", "u1", (2, 2)), ("l_coef", "u1", (2, 2)), ("reserved", "u1", (2,))])
UV16_RESULT_DTYPE = np.dtype([("total", "<f4"), ("dc_total", "<f4"), ("cfl_total", "<f4"), ("uv_mode", "u1"),
                              ("angle_delta", "i1"), ("cfl_alpha", "i1", (2,))])
assert C.sizeof(UvModeCdfs) == 2 * (13 * 14 + 8 * 7 + 8 + 6 * 16) and C.sizeof(UvModeCosts) == 4 * (13 * 14 + 8 * 7 + 8 + 6 * 16)
assert UV16_JOB_DTYPE.itemsize == 16 and UV16_RESULT_DTYPE.itemsize == 16
UV16_444_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("y_mode", "u1"), ("flags", "u1"),
                               ("a_coef", "u1", (2, 4)), ("l_coef", "u1", (2, 4)), ("reserved", "u1", (2,))])
assert UV16_444_JOB_DTYPE.itemsize == 24
UV32_444_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("y_mode", "u1"), ("flags", "u1"),
                               ("a_coef", "u1", (2, 8)), ("l_coef", "u1", (2, 8)), ("reserved", "u1", (2,))])
assert UV32_444_JOB_DTYPE.itemsize == 40

SPLIT16_JOB_DTYPE = np.dtype([
    ("px", "<u2"), ("py", "<u2"), ("mode", "u1"), ("angle_delta", "i1"), ("flags", "u1"), ("reserved", "u1"),
    ("a_coef", "u1", (4,)), ("l_coef", "u1", (4,)),
])
SPLIT16_RESULT_DTYPE = np.dtype([("sse", "<i8"), ("bits", "<f4"), ("tx_types", "u1", (4,))])
SPLIT16_D2_RESULT_DTYPE = np.dtype([("sse", "<i8"), ("bits", "<f4"), ("tx_types", "u1", (16,)),
                                    ("reserved", "u1", (4,))])
assert SPLIT16_JOB_DTYPE.itemsize == 16 and SPLIT16_RESULT_DTYPE.itemsize == 16
assert SPLIT16_D2_RESULT_DTYPE.itemsize == 32
LEAF8_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("mode", "u1"), ("angle_delta", "i1"), ("flags", "u1"),
                            ("dcs_ctx", "u1"), ("syntax_bits", "<f4")])
LEAF8_RESULT_DTYPE = np.dtype([("sse", "<i8"), ("bits", "<f4"), ("cost", "<f4"), ("tx_type", "u1"),
                               ("reserved", "u1", (7,))])
assert LEAF8_JOB_DTYPE.itemsize == 12 and LEAF8_RESULT_DTYPE.itemsize == 24
# mt_quad32_job / mt_quad32_result.
QUAD32_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("mode", "u1"), ("angle_delta", "i1"), ("flags", "u1"),
                             ("reserved", "u1"), ("dcs_ctx", "u1", (4,)), ("mode_bits", "<f4"),
                             ("delta_bits", "<f4")], align=True)
QUAD32_RESULT_DTYPE = np.dtype([("total", "<f4"), ("bits", "<f4", (4,)), ("reserved", "<u4"), ("sse", "<i8", (4,))],
                               align=True)
assert QUAD32_JOB_DTYPE.itemsize == 20 and QUAD32_RESULT_DTYPE.itemsize == 56
# mt_grid16_job / mt_grid16_result.
GRID16_JOB_DTYPE = np.dtype([("px", "<u2"), ("py", "<u2"), ("mode", "u1"), ("angle_delta", "i1"), ("flags", "u1"),
                             ("reserved", "u1"), ("a_coef", "u1", (16,)), ("l_coef", "u1", (16,)),
                             ("mode_bits", "<f4"), ("delta_bits", "<f4"), ("depth_bits", "<f4")], align=True)
GRID16_RESULT_DTYPE = np.dtype([("total", "<f4"), ("dist", "<f4"), ("bits", "<f4"), ("reserved", "<u4"),
                                ("sse", "<i8")], align=True)
assert GRID16_JOB_DTYPE.itemsize == 52 and GRID16_RESULT_DTYPE.itemsize == 24
CFL_BLOCK_DTYPE = np.dtype([("cx", "<u2"), ("cy", "<u2"), ("dc", "<i2", (2,))])
assert CFL_BLOCK_DTYPE.itemsize == 8

PALETTE_SLOTS = 14


class PaletteOpts(C.Structure):
    _fields_ = [("smooth_t", C.c_int32), ("smooth_guard", C.c_int32), ("viterbi_lambda", C.c_float),
                ("color_costs", (C.c_float * 8) * 5 * 7)]


PALETTE_CAND_DTYPE = np.dtype([("colors", "<i2", (8,)), ("n_colors", "u1"), ("sel", "u1"), ("hist_len", "u1"),
                               ("reserved", "u1"), ("index_bits", "<f4")])
assert PALETTE_CAND_DTYPE.itemsize == 24

UV_PALETTE_SLOTS = 4
UV_PALETTE_CAND_DTYPE = np.dtype([("n_colors", "u1"), ("exact", "u1"), ("reserved", "u1", (2,)),
                                  ("u", "<i2", (8,)), ("v", "<i2", (8,))])
assert UV_PALETTE_CAND_DTYPE.itemsize == 36


class DeblockFrameParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("w8", "h8", "disp_w", "disp_h", "sub_x", "sub_y", "mono", "bd")]


class CdefParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("w8", "h8", "disp_w", "disp_h", "sub_x", "sub_y", "mono", "base_q_idx",
                                         "bd", "slow")]


class CdefDecision(C.Structure):
    _fields_ = [
        ("bits", C.c_int32), ("damping", C.c_int32), ("n_strengths", C.c_int32), ("unit_cols", C.c_int32),
        ("unit_rows", C.c_int32), ("strengths", (C.c_uint8 * 4) * 8),
    ]


assert C.sizeof(CdefParams) == 40 and C.sizeof(CdefDecision) == 52


class AqParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("w8", "h8", "tile_cols_log2", "tile_rows_log2", "base_q_idx", "bd",
                                         "variance_boost", "dark_aq", "octile", "boost_only")] + [
        ("strength", C.c_float)]


assert C.sizeof(AqParams) == 44

AQ_CELL_DTYPE = np.dtype([("prev", "u1"), ("newq", "u1"), ("steps", "i1"), ("target", "u1")])


class ScreenGateParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("w8", "h8", "sub_x", "sub_y", "bd", "base_q_idx")]


class ScreenGateResult(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("ibc_pays", "few_colour", "copy_stage")] + [
        (n, C.c_uint32) for n in ("blocks16", "few16", "lenient16", "nonflat8", "dup8", "copied", "reserved")] + [
        ("gain", C.c_uint64), ("photo", C.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


assert C.sizeof(ScreenGateParams) == 24 and C.sizeof(ScreenGateResult) == 56

BLOCK8_DTYPE = np.dtype([
    ("px", "<u2"), ("py", "<u2"), ("flags", "u1"), ("dcs_ctx", "u1"), ("skip_ctx", "u1"), ("reserved", "u1"),
    ("mode_bits", "<f4", (13,)),
])
COMBO_DTYPE = np.dtype([("mode", "u1"), ("angle_delta", "i1"), ("tx_type", "u1"), ("flags", "u1"), ("bits", "<f4")])
BEST_DTYPE = np.dtype([
    ("combo", "<i4"), ("cost", "<f4"), ("distortion", "<f4"), ("bits", "<f4"), ("satd", "<u4"), ("eob", "<i4"),
    ("reserved", "<u4", (2,)),
])
assert BLOCK8_DTYPE.itemsize == 60 and COMBO_DTYPE.itemsize == 8 and BEST_DTYPE.itemsize == 32

CANDIDATE_DTYPE = np.dtype([
    ("px", "<u2"), ("py", "<u2"), ("mode", "u1"), ("angle_delta", "i1"), ("tx_type", "u1"),
    ("flags", "u1"), ("dcs_ctx", "u1"), ("skip_ctx", "u1"), ("reserved", "<u2"), ("mode_bits", "<f4"),
    ("extra_bits", "<f4"),
])
RESULT_DTYPE = np.dtype([
    ("distortion", "<f4"), ("bits", "<f4"), ("cost", "<f4"), ("satd", "<u4"), ("eob", "<i4"),
    ("reserved", "<u4", (3,)),
])
assert CANDIDATE_DTYPE.itemsize == 20 and RESULT_DTYPE.itemsize == 32

_P = C.c_void_p


class RdLambdas(C.Structure):
    _fields_ = [("mode_lambda", C.c_float), ("lambda_d", C.c_float), ("trellis_lambda0", C.c_float),
                ("satd_scale", C.c_float), ("satd_bridge", C.c_float)]


class SequenceHeaderParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("profile", C.c_uint32), ("bit_depth", C.c_uint32),
                ("monochrome", C.c_int32), ("color_present", C.c_int32), ("primaries", C.c_uint32),
                ("transfer", C.c_uint32), ("matrix", C.c_uint32), ("full_range", C.c_int32),
                ("chroma_sample_position", C.c_uint32), ("ss_x", C.c_uint32), ("ss_y", C.c_uint32),
                ("enable_filter_intra", C.c_int32), ("enable_intra_edge_filter", C.c_int32)]


class FrameHeaderParams(C.Structure):
    _fields_ = [("w8", C.c_int32), ("h8", C.c_int32), ("tile_cols_log2", C.c_int32), ("tile_rows_log2", C.c_int32),
                ("base_q_idx", C.c_uint32), ("qm_y", C.c_uint32), ("qm_u", C.c_uint32), ("qm_v", C.c_uint32),
                ("uac_delta", C.c_int32), ("udc_delta", C.c_int32), ("monochrome", C.c_int32), ("aq", C.c_int32),
                ("delta_q_res_log2", C.c_uint32), ("allow_intrabc", C.c_int32), ("updating_cdf", C.c_int32),
                ("lf_y", C.c_int32), ("lf_u", C.c_int32), ("lf_v", C.c_int32), ("lf_sharpness", C.c_int32),
                ("cdef_bits", C.c_int32), ("cdef_damping", C.c_int32), ("cdef_strengths", (C.c_uint8 * 4) * 8),
                ("lr_luma_wiener", C.c_int32)]


class AvifItemParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("bit_depth", C.c_uint8), ("channels", C.c_uint8),
                ("seq_profile", C.c_uint8), ("seq_level_idx", C.c_uint8), ("monochrome", C.c_int32),
                ("chroma_sub_x", C.c_int32), ("chroma_sub_y", C.c_int32), ("color_present", C.c_int32),
                ("primaries", C.c_uint16), ("transfer", C.c_uint16), ("matrix", C.c_uint16),
                ("full_range", C.c_int32), ("icc", C.c_void_p), ("icc_len", C.c_size_t), ("exif", C.c_void_p),
                ("exif_len", C.c_size_t), ("irot_steps", C.c_uint8), ("imir_axis", C.c_int32),
                ("clli_present", C.c_int32), ("max_content_light_level", C.c_uint16),
                ("max_pic_average_light_level", C.c_uint16)]


class EncodeConfig(C.Structure):
    _fields_ = [("quality", C.c_int32), ("chroma", C.c_int32), ("color_present", C.c_int32),
                ("primaries", C.c_uint32), ("transfer", C.c_uint32), ("matrix", C.c_uint32),
                ("full_range", C.c_int32), ("chroma_sample_position", C.c_uint32), ("icc", C.c_void_p),
                ("icc_len", C.c_size_t), ("orientation", C.c_int32), ("clli_present", C.c_int32),
                ("max_content_light_level", C.c_uint16), ("max_pic_average_light_level", C.c_uint16),
                ("exif", C.c_void_p), ("exif_len", C.c_size_t), ("threads", C.c_int32), ("speed", C.c_int32),
                ("updating_cdf", C.c_int32), ("adaptive_quant", C.c_int32), ("variance_boost", C.c_int32),
                ("dark_aq", C.c_int32), ("cdef", C.c_int32), ("wiener", C.c_int32),
                ("quantization_matrices", C.c_int32), ("screen_content", C.c_int32), ("intrabc", C.c_int32),
                ("qmatrix_level", C.c_int32), ("alpha_quality", C.c_int32)]


class EncodePlan(C.Structure):
    _fields_ = [("base_q_idx", C.c_uint8), ("qm_y", C.c_uint8), ("qm_u", C.c_uint8), ("qm_v", C.c_uint8),
                ("sub", C.c_int32), ("cdef", C.c_int32), ("aq", C.c_int32), ("variance_boost", C.c_int32),
                ("dark_aq", C.c_int32)]


class EncodeStats(C.Structure):
    """mt_encode_stats: what one encode call did."""
    _fields_ = [("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("kernel_launches", C.c_uint32),
                ("tokens", C.c_uint32), ("blocks", C.c_uint32), ("levels", C.c_uint32), ("blocks_ms", C.c_float),
                ("call_ms", C.c_float)]


COEF_BLOCK_DTYPE = np.dtype([("cf_offset", "<u4"), ("log2n", "u1"), ("plane", "u1"), ("skip_ctx", "u1"),
                              ("dcs_ctx", "u1"), ("y_mode", "u1"), ("txtp", "u1"), ("code_txtp", "u1"),
                              ("tx_class", "u1")])
assert COEF_BLOCK_DTYPE.itemsize == 12


class CdfSlotLayout(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("skip", "intrabc", "part_bl8", "part_split", "kf_y", "uv_mode",
                                          "angle_delta", "filter_intra", "filter_intra_mode", "palette_y_mode",
                                          "palette_y_size", "palette_uv_mode", "cfl_sign", "cfl_alpha", "txsz",
                                          "txtp8", "txtp4", "txtp16")] + [
        ("txb_skip", C.c_int32 * 5), ("base_tok", (C.c_int32 * 2) * 5), ("br_tok", (C.c_int32 * 2) * 4),
        ("eob_base", (C.c_int32 * 2) * 5), ("eob_hi", (C.c_int32 * 2) * 5), ("dc_sign", C.c_int32 * 2),
        ("eob_bin", C.c_int32), ("delta_q", C.c_int32), ("wiener_restore", C.c_int32), ("nslots", C.c_int32)]


def _bind(lib):
    sig = {
        "mt_version": (C.c_char_p, []),
        "mt_quant_init": (C.c_int, [C.c_uint8, C.c_uint8, C.c_uint8, C.POINTER(Quant)]),
        "mt_quant_init_chroma": (C.c_int, [C.c_uint8, C.c_int32, C.c_int32, C.c_uint8, C.c_uint8, C.POINTER(Quant)]),
        "mt_qm_row": (_P, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "mt_default_scan": (_P, [C.c_int32]),
        "mt_coef_costs_build": (C.c_int, [C.POINTER(CoefCdfs), C.POINTER(CoefCosts)]),
        "mt_qcat": (C.c_int, [C.c_int32]),
        "mt_range_encoder_new": (_P, [C.c_int32]),
        "mt_range_encoder_free": (None, [_P]),
        "mt_range_encode_bool": (C.c_int, [_P, C.c_int32, C.c_uint16]),
        "mt_range_encode_symbol": (C.c_int, [_P, C.c_int32, _P, C.c_int32, C.c_int32]),
        "mt_range_encode_literal": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
        "mt_range_encode_signed_subexp_with_ref": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_uint32,
                                                             C.c_int32]),
        "mt_range_encoder_done": (C.c_int, [_P, C.POINTER(_P), C.POINTER(C.c_size_t)]),
        "mt_cdf_slot_count": (C.c_int32, []),
        "mt_cdfs_default": (C.c_int, [C.c_int32, _P, C.c_size_t, _P, _P, C.c_int32, C.POINTER(C.c_size_t),
                                      C.POINTER(C.c_int32)]),
        "mt_pack_tile": (C.c_int, [C.c_uint8, C.c_int32, _P, _P, _P, C.c_int32, C.POINTER(_P),
                                   C.POINTER(C.c_size_t), C.POINTER(_P)]),
        "mt_pack_tile_filtered": (C.c_int, [C.c_uint8, C.c_int32, _P, _P, _P, C.c_int32, _P, C.c_int32,
                                            C.POINTER(_P), C.POINTER(C.c_size_t)]),
        "mt_tile_trace_free": (None, [_P]),
        "mt_replay_tile_with_filters": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32,
                                                  C.c_int32, C.c_int32, C.c_int32, C.POINTER(_P),
                                                  C.POINTER(C.c_size_t)]),
        "mt_free": (None, [_P]),
        "mt_cdf_layout": (C.c_int, [C.POINTER(CdfSlotLayout)]),
        "mt_encode_rgb8": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(EncodeConfig), C.POINTER(_P),
                                     C.POINTER(C.c_size_t)]),
        "mt_encode_rgb8_ex": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(EncodeConfig), C.POINTER(_P),
                                        C.POINTER(C.c_size_t), _P, C.POINTER(EncodeStats)]),
        "mt_encode_rgb8_device": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(EncodeConfig), C.POINTER(_P),
                                            C.POINTER(C.c_size_t), C.POINTER(EncodeStats)]),
        "mt_encode_release_buffers": (None, []),
        "mt_encode_rgb8_batch": (C.c_int, [C.c_int32, _P, _P, _P, C.POINTER(EncodeConfig), _P, _P, _P,
                                           C.POINTER(EncodeStats)]),
        "mt_encode_yuv8": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_uint32, C.POINTER(EncodeConfig), C.POINTER(_P),
                                     C.POINTER(C.c_size_t), _P]),
        "mt_emit_coeffs_device": (C.c_int, [_P, _P, C.c_int32, _P, _P, _P, _P, _P]),
        "mt_emit_coeffs": (C.c_int, [_P, C.c_size_t, _P, C.c_int32, C.POINTER(_P), _P, _P]),
        "mt_encode_config_default": (C.c_int, [C.POINTER(EncodeConfig)]),
        "mt_encode_config_validate": (C.c_int, [C.POINTER(EncodeConfig)]),
        "mt_validate_rgb8_input": (C.c_int, [C.c_uint32, C.c_uint32, C.c_size_t]),
        "mt_encode_config_effective": (C.c_int, [C.POINTER(EncodeConfig), C.POINTER(EncodePlan)]),
        "mt_leb128": (C.c_int, [C.c_uint64, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
        "mt_wrap_obu": (C.c_int, [C.c_int32, _P, C.c_size_t, C.POINTER(_P), C.POINTER(C.c_size_t)]),
        "mt_tiling_increments": (C.c_int, [C.c_int32] * 4 + [_P, C.POINTER(C.c_int32), _P, C.POINTER(C.c_int32)]),
        "mt_sequence_header": (C.c_int, [C.POINTER(SequenceHeaderParams), C.POINTER(_P), C.POINTER(C.c_size_t)]),
        "mt_frame_header": (C.c_int, [C.POINTER(FrameHeaderParams), C.c_int32, C.POINTER(_P),
                                      C.POINTER(C.c_size_t)]),
        "mt_assemble_frame_obus": (C.c_int, [C.POINTER(FrameHeaderParams), _P, _P, C.c_int32, C.POINTER(_P),
                                             C.POINTER(C.c_size_t)]),
        "mt_av1_stream": (C.c_int, [C.POINTER(SequenceHeaderParams), C.POINTER(FrameHeaderParams), _P, _P,
                                    C.c_int32, C.POINTER(_P), C.POINTER(C.c_size_t)]),
        "mt_av1_level_for": (C.c_uint8, [C.c_uint32, C.c_uint32]),
        "mt_wrap_av1_image": (C.c_int, [_P, C.c_size_t, C.POINTER(AvifItemParams), C.POINTER(_P),
                                        C.POINTER(C.c_size_t)]),
        "mt_quality_to_q": (C.c_uint8, [C.c_uint8]),
        "mt_qm_levels": (C.c_int, [C.c_uint8, C.c_int32, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
        "mt_rd_lambdas_init": (C.c_int, [C.c_uint8, C.c_int32, C.c_int32, C.c_uint8, C.POINTER(RdLambdas)]),
        "mt_coef_cdfs_default": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(CoefCdfs)]),
        "mt_candidate_chain": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, C.POINTER(CoefCosts),
                                         _P, C.c_int32, _P, _P, _P]),
        "mt_candidate_chain_device": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, _P, _P,
                                                C.c_int32, _P, _P, _P, _P, _P]),
        "mt_candidate_chain_scratch_bytes": (C.c_size_t, [C.c_int32]),
        "mt_rdo_level8": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                    C.c_int32, _P, C.c_int32, _P, _P]),
        "mt_rdo_level8_device": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, _P, _P, C.c_int32,
                                           _P, C.c_int32, _P, _P, _P, _P]),
        "mt_rdo_level8_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
        "mt_rdo_level4": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                    C.c_int32, _P, C.c_int32, _P, _P]),
        "mt_rdo_level16": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                     C.c_int32, _P, C.c_int32, _P, _P]),
        "mt_rdo_level4_device": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, _P, _P, C.c_int32,
                                           _P, C.c_int32, _P, _P, _P, _P]),
        "mt_rdo_level16_device": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, _P, _P, C.c_int32,
                                            _P, C.c_int32, _P, _P, _P, _P]),
        "mt_rdo_level4_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
        "mt_rdo_level16_scratch_bytes": (C.c_size_t, [C.c_int32, C.c_int32]),
        "mt_rdo_level8_device_noalloc": (C.c_int, [_P, _P, C.POINTER(ChainParams), C.POINTER(Quant), _P, _P, _P,
                                                   C.c_int32, _P, C.c_int32, _P, _P]),
        "mt_padded_plane_dims": (C.c_int, [C.c_int32, C.c_int32, C.c_int32] + [C.POINTER(C.c_int32)] * 4),
        "mt_csc_rgb8": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P]),
        "mt_csc_rgb8_device": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P]),
        "mt_deblock_plane": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "mt_deblock_plane_device": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P,
                                              C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]),
        "mt_loop_filter_levels": (C.c_int, [C.c_int32] * 3 + [C.POINTER(C.c_int32)] * 3),
        "mt_deblock_frame_scratch_bytes": (C.c_size_t, [C.POINTER(DeblockFrameParams)]),
        "mt_deblock_frame_device": (C.c_int, [_P] * 9 + [C.POINTER(DeblockFrameParams)] + [C.c_int32] * 3 + [_P, _P]),
        "mt_deblock_frame_device_to": (C.c_int, [_P] * 12 + [C.POINTER(DeblockFrameParams)] + [C.c_int32] * 3 +
                                       [_P, _P]),
        "mt_deblock_frame": (C.c_int, [_P] * 9 + [C.POINTER(DeblockFrameParams)] + [C.c_int32] * 3),
        "mt_cdef_tables_device": (C.c_int, [_P] * 7 + [C.POINTER(CdefParams)] + [_P] * 6),
        "mt_cdef_scratch_bytes": (C.c_size_t, [C.POINTER(CdefParams)]),
        "mt_cdef_frame_device": (C.c_int, [_P] * 7 + [C.POINTER(CdefParams), _P, C.POINTER(CdefDecision), _P, _P]),
        "mt_cdef_frame": (C.c_int, [_P] * 7 + [C.POINTER(CdefParams), C.POINTER(CdefDecision), _P]),
        "mt_tiling_spec_min": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
        "mt_aq_grid_scratch_bytes": (C.c_size_t, [C.POINTER(AqParams)]),
        "mt_aq_grid_device": (C.c_int, [_P, C.POINTER(AqParams), _P, _P, _P, _P]),
        "mt_aq_grid": (C.c_int, [_P, C.POINTER(AqParams), _P, _P]),
        "mt_dark_pow_device": (C.c_int, [_P, _P, C.c_int64, _P]),
        "mt_mode_beam_device": (C.c_int, [_P, _P, C.POINTER(ChainParams), _P, C.c_int32, _P, _P, _P]),
        "mt_sse_recon_device": (C.c_int, [_P] + [C.c_int32] * 4 + [_P, _P, _P] + [C.c_int32] * 3 + [C.c_float, _P, _P]),
        "mt_sse_recon": (C.c_int, [_P] + [C.c_int32] * 5 + [_P, _P, _P] + [C.c_int32] * 3 + [C.c_float, _P]),
        "mt_mode_beam": (C.c_int, [_P, _P, C.POINTER(ChainParams), _P, C.c_int32, _P, _P]),
        "mt_trellis_optimize_ctx_device": (C.c_int, [_P, _P, _P, C.c_int32, C.POINTER(Quant), _P, _P, C.c_float,
                                                     C.c_float, _P]),
        "mt_split16_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                             C.c_int32, _P, _P, _P, _P]),
        "mt_split16_depth2_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                               C.c_int32, _P, _P, _P, _P]),
        "mt_split16_depth2": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P,
                                        C.POINTER(CoefCosts), _P, C.c_int32, _P, _P, _P]),
        "mt_filter_intra_beam_device": (C.c_int, [_P, _P] + [C.c_int32] * 8 + [_P, C.c_int32, _P, _P, _P, _P]),
        "mt_filter_intra_beam": (C.c_int, [_P, _P] + [C.c_int32] * 8 + [_P, C.c_int32, _P, _P, _P]),
        "mt_cfl_alpha_device": (C.c_int, [_P, C.c_int32, _P, _P] + [C.c_int32] * 8 + [_P, C.c_int32, _P, _P, _P]),
        "mt_cfl_alpha": (C.c_int, [_P, C.c_int32, C.c_int32, _P, _P] + [C.c_int32] * 9 + [_P, C.c_int32, _P, _P]),
        "mt_split4tx_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                         C.c_int32, _P, _P, _P, _P]),
        "mt_split4tx": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                  C.c_int32, _P, _P, _P]),
        "mt_leaf8_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                           C.c_int32, _P, _P, _P, _P]),
        "mt_leaf8_tx_refine_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                                C.c_int32, _P, _P, _P, _P]),
        "mt_leaf16_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                            C.c_int32, _P, _P, _P, _P]),
        "mt_luma_palette_device": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                             _P, C.c_int32, C.POINTER(PaletteOpts), _P, _P, _P]),
        "mt_luma_palette": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P,
                                      C.c_int32, C.POINTER(PaletteOpts), _P, _P]),
        "mt_uv_palette_device": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32,
                                           C.POINTER(PaletteOpts), _P, _P, _P]),
        "mt_uv_palette": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32,
                                    C.POINTER(PaletteOpts), _P, _P]),
        "mt_leaf16_tx_refine_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                                 C.c_int32, _P, _P, _P, _P]),
        "mt_leaf16": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                C.c_int32, C.c_int32, _P, _P, _P]),
        "mt_leaf32_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                            C.c_int32, _P, _P, _P, _P]),
        "mt_leaf32": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                                C.c_int32, _P, _P, _P]),
        "mt_quad32_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                            C.c_int32, _P, _P]),
        "mt_quad32_luma": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts),
                                     _P, C.c_int32, _P]),
        "mt_uv_mode_cdfs_default": (C.c_int, [C.POINTER(UvModeCdfs)]),
        "mt_uv_mode_costs_build": (C.c_int, [C.POINTER(UvModeCdfs), C.POINTER(UvModeCosts)]),
        "mt_uv_mode_bits": (C.c_float, [C.POINTER(UvModeCosts), C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                        C.c_int32]),
        "mt_pick_uv16_420_device": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                              C.POINTER(Quant), _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P]),
        "mt_pick_uv16_420": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                       C.POINTER(Quant), _P, C.POINTER(CoefCosts), C.POINTER(UvModeCosts), _P,
                                       C.c_int32, _P, _P, _P]),
        "mt_pick_uv16_444": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                       C.POINTER(Quant), _P, C.POINTER(CoefCosts), C.POINTER(UvModeCosts), _P,
                                       C.c_int32, _P, _P, _P]),
        "mt_pick_uv32_444": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                       C.POINTER(Quant), _P, C.POINTER(CoefCosts), C.POINTER(UvModeCosts), _P,
                                       C.c_int32, _P, _P, _P]),
        "mt_pick_uv32_444_device": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                              C.POINTER(Quant), _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P]),
        "mt_pick_uv32_420": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                       C.POINTER(Quant), _P, C.POINTER(CoefCosts), C.POINTER(UvModeCosts), _P,
                                       C.c_int32, _P, _P, _P]),
        "mt_pick_uv32_420_device": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                              C.POINTER(Quant), _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P]),
        "mt_pick_uv16_444_device": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(Split16Params), C.POINTER(Uv16Params),
                                              C.POINTER(Quant), _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P]),
        "mt_grid16_luma_device": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, _P, _P,
                                            C.c_int32, _P, _P, _P]),
        "mt_grid16_luma": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts),
                                     _P, C.c_int32, _P, _P]),
        "mt_leaf8": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts), _P,
                               C.c_int32, C.c_int32, _P, _P, _P]),
        "mt_split16_luma": (C.c_int, [_P, _P, C.POINTER(Split16Params), C.POINTER(Quant), _P, C.POINTER(CoefCosts),
                                      _P, C.c_int32, _P, _P, _P]),
        "mt_screen_gate_scratch_bytes": (C.c_size_t, [C.POINTER(ScreenGateParams)]),
        "mt_screen_gate_device": (C.c_int, [_P, C.POINTER(ScreenGateParams), _P, C.POINTER(ScreenGateResult), _P]),
        "mt_screen_gate": (C.c_int, [_P, C.POINTER(ScreenGateParams), C.POINTER(ScreenGateResult)]),
        "mt_fwd_txfm_quant_device": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.POINTER(Quant), _P, _P, _P, _P]),
        "mt_inv_txfm_dequant_device": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.POINTER(Quant), _P, _P, _P]),
        "mt_trellis_optimize_device": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float, _P]),
        "mt_intra_predict_device": (C.c_int, [_P, C.POINTER(ChainParams), _P, C.c_int32, _P, _P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def load():
    """Load the CUDA library (raises OSError when it is missing or broken)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"maroontree_b200: CUDA library not built ({LIB_PATH}); run python -m maroontree_b200.build")
        _lib = _bind(C.CDLL(LIB_PATH))
    return _lib


EXPORTED_SYMBOLS = (
    "mt_version", "mt_quant_init", "mt_quant_init_chroma", "mt_qm_row", "mt_default_scan",
    "mt_coef_costs_build", "mt_qcat", "mt_coef_cdfs_default", "mt_range_encoder_new", "mt_range_encoder_free",
    "mt_range_encode_bool", "mt_range_encode_symbol", "mt_range_encode_literal",
    "mt_range_encode_signed_subexp_with_ref", "mt_range_encoder_done", "mt_cdf_slot_count", "mt_cdfs_default", "mt_cdf_layout",
    "mt_emit_coeffs_device", "mt_emit_coeffs", "mt_encode_rgb8", "mt_encode_rgb8_ex", "mt_encode_rgb8_device", "mt_encode_release_buffers", "mt_encode_rgb8_batch", "mt_encode_yuv8",
    "mt_pack_tile", "mt_pack_tile_filtered", "mt_tile_trace_free", "mt_replay_tile_with_filters", "mt_free",
    "mt_leb128", "mt_wrap_obu", "mt_tiling_increments", "mt_sequence_header", "mt_frame_header",
    "mt_assemble_frame_obus", "mt_av1_stream", "mt_av1_level_for", "mt_wrap_av1_image",
    "mt_encode_config_default", "mt_encode_config_validate", "mt_validate_rgb8_input", "mt_encode_config_effective", "mt_quality_to_q", "mt_qm_levels",
    "mt_rd_lambdas_init", "mt_candidate_chain", "mt_candidate_chain_device", "mt_candidate_chain_scratch_bytes",
    "mt_rdo_level8", "mt_rdo_level8_device", "mt_rdo_level8_scratch_bytes", "mt_rdo_level8_device_noalloc",
    "mt_rdo_level4", "mt_rdo_level4_device", "mt_rdo_level4_scratch_bytes", "mt_fwd_txfm_quant_device",
    "mt_rdo_level16", "mt_rdo_level16_device", "mt_rdo_level16_scratch_bytes",
    "mt_padded_plane_dims", "mt_csc_rgb8", "mt_csc_rgb8_device", "mt_deblock_plane", "mt_deblock_plane_device",
    "mt_loop_filter_levels", "mt_deblock_frame_scratch_bytes", "mt_deblock_frame_device", "mt_deblock_frame_device_to", "mt_deblock_frame",
    "mt_cdef_tables_device", "mt_cdef_scratch_bytes", "mt_cdef_frame_device", "mt_cdef_frame",
    "mt_inv_txfm_dequant_device", "mt_trellis_optimize_device", "mt_intra_predict_device",
    "mt_tiling_spec_min", "mt_aq_grid_scratch_bytes", "mt_aq_grid_device", "mt_aq_grid", "mt_dark_pow_device",
    "mt_screen_gate_scratch_bytes", "mt_screen_gate_device", "mt_screen_gate", "mt_mode_beam_device", "mt_mode_beam",
    "mt_sse_recon_device", "mt_sse_recon", "mt_trellis_optimize_ctx_device", "mt_split16_luma_device",
    "mt_split16_luma", "mt_split16_depth2_device", "mt_split16_depth2", "mt_cfl_alpha_device", "mt_cfl_alpha",
    "mt_filter_intra_beam_device", "mt_filter_intra_beam", "mt_split4tx_device", "mt_split4tx",
    "mt_leaf8_luma_device", "mt_leaf8_tx_refine_device", "mt_leaf8", "mt_leaf16_luma_device", "mt_leaf16_tx_refine_device", "mt_luma_palette_device", "mt_luma_palette", "mt_uv_palette_device", "mt_uv_palette",
    "mt_leaf16", "mt_leaf32_luma_device", "mt_leaf32", "mt_quad32_luma_device", "mt_quad32_luma",
    "mt_grid16_luma_device", "mt_grid16_luma", "mt_uv_mode_cdfs_default", "mt_uv_mode_costs_build",
    "mt_uv_mode_bits", "mt_pick_uv16_420_device", "mt_pick_uv16_420",
    "mt_pick_uv16_444_device", "mt_pick_uv16_444", "mt_pick_uv32_420_device", "mt_pick_uv32_420",
    "mt_pick_uv32_444_device", "mt_pick_uv32_444",
)


def ptr(a):
    """Address of a numpy array, torch tensor, ctypes object or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    if isinstance(a, int):
        return a
    return C.addressof(a)
