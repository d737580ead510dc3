"""ctypes bindings of the oracle library (test infrastructure: the CPU checker
of the CUDA path; see oracle.h).  Only tests, ``__graft_entry__.smoke`` and the
bench's CPU-baseline leg load this."""
import ctypes as C
import os

import numpy as np

from maroontree_b200 import abi

from . import build as _build

_lib = None
_P = C.c_void_p


def load():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        lib = C.CDLL(path)
        sig = {
            "or_quant_init": (C.c_int, [C.c_uint8, C.c_uint8, C.c_uint8, C.POINTER(abi.Quant)]),
            "or_quant_init_chroma": (C.c_int, [C.c_uint8, C.c_int32, C.c_int32, C.c_uint8, C.c_uint8,
                                               C.POINTER(abi.Quant)]),
            "or_qm_row": (_P, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "or_default_scan": (_P, [C.c_int32]),
            "or_fwd_txfm_quant": (None, [_P, C.c_int32, C.c_int32, C.POINTER(abi.Quant), _P, _P, _P]),
            "or_inv_txfm_dequant": (None, [_P, C.c_int32, C.c_int32, C.POINTER(abi.Quant), _P, _P]),
            "or_trellis_optimize": (None, [_P, _P, C.c_float, C.c_float, _P, C.c_int32, C.c_float]),
            "or_intra_predict": (None, [_P] + [C.c_int32] * 13 + [_P]),
            "or_dc_pred": (C.c_int32, [_P] + [C.c_int32] * 6),
            "or_luma_satd": (C.c_uint64, [_P] + [C.c_int32] * 6 + [_P, _P]),
            "or_cdf_cost": (C.c_float, [_P, C.c_int32]),
            "or_real_block_bits": (C.c_float, [_P, _P, C.c_int32, C.c_int32, C.POINTER(abi.CoefCdfs), C.c_int32,
                                               C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P]),
            "or_edge_filter_strength": (C.c_int, [C.c_int] * 4),
            "or_use_edge_upsample": (C.c_int, [C.c_int] * 4),
            "or_csc_rgb8": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P]),
            "or_cdef_frame": (C.c_int, [_P] * 7 + [C.POINTER(abi.CdefParams), C.POINTER(abi.CdefDecision)] + [_P] * 6),
            "or_weighted_sse": (C.c_float, [_P, C.c_int32, C.c_int32]),
            "or_cdef_frame_lambda": (C.c_float, [C.c_int32] * 4),
            "or_loop_filter_levels": (None, [C.c_int32, C.c_int32] + [C.POINTER(C.c_int32)] * 3),
            "or_deblock_frame": (C.c_int, [_P] * 9 + [C.POINTER(abi.DeblockFrameParams)] + [C.c_int32] * 3),
            "or_real_block_bits_wh": (C.c_float, [_P, _P, C.c_int32, C.c_int32, C.POINTER(abi.CoefCdfs)] +
                                      [C.c_int32] * 5 + [_P]),
            "or_deblock_plane": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P, _P, _P,
                                           C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
            "or_coef_costs_build": (None, [C.POINTER(abi.CoefCdfs), C.POINTER(abi.CoefCosts)]),
            "or_fast_round": (C.c_float, [C.c_float]),
            "or_dct1d": (None, [_P, C.c_int32]),
            "or_sse_recon": (C.c_int, [_P] + [C.c_int32] * 4 + [_P, _P, _P] + [C.c_int32] * 3 + [C.c_float, _P]),
            "or_mode_beam": (C.c_int, [_P, _P, C.POINTER(abi.ChainParams), _P, C.c_int32, _P, _P]),
            "or_dirty_log1pf": (C.c_float, [C.c_float]),
            "or_dark_pow": (None, [_P, _P, C.c_int64]),
            "or_dark_protection": (C.c_int32, [C.c_int32, C.c_int32, _P] + [C.c_int32] * 5 + [C.c_float]),
            "or_tiling_spec_min": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
            "or_aq_grid": (C.c_int, [_P, C.POINTER(abi.AqParams), _P, _P]),
            "or_screen_gate": (C.c_int, [_P, C.POINTER(abi.ScreenGateParams), C.POINTER(abi.ScreenGateResult)]),
            "or_hash8": (C.c_uint32, [_P, C.c_int32, C.c_int32, C.c_int32]),
            "or_candidate_chain": (C.c_int, [_P, _P, C.POINTER(abi.ChainParams), C.POINTER(abi.Quant), _P,
                                             C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P, _P, C.c_int32]),
            "or_real_block_bits_bounded": (C.c_float, [_P, _P, C.c_int32, C.c_int32, C.POINTER(abi.CoefCdfs)] +
                                           [C.c_int32] * 5 + [_P, C.c_float]),
            "or_trellis_optimize_ctx": (None, [_P, _P, C.c_float, C.c_float, _P, C.c_int32, C.c_float,
                                               C.POINTER(abi.CoefCdfs), C.c_int32, _P, C.c_int32, C.c_float]),
            "or_luma_bits_1d": (C.c_float, [_P, C.c_int32, C.c_int32, C.POINTER(abi.CoefCdfs), C.c_int32, C.c_int32]),
            "or_coef_res_ctx": (C.c_uint8, [_P, _P, C.c_int32]),
            "or_split16_depth2": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                            C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P, _P, C.c_int32]),
            "or_filter_intra_predict": (None, [_P] + [C.c_int32] * 7 + [_P]),
            "or_filter_intra_beam": (C.c_int, [_P, _P] + [C.c_int32] * 8 + [_P, C.c_int32, _P, _P, _P]),
            "or_cfl_alpha": (C.c_int, [_P, C.c_int32, _P, _P] + [C.c_int32] * 8 + [_P, C.c_int32, _P, _P]),
            "or_split4tx": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                      C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_luma_palette": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P,
                                          C.c_int32, C.POINTER(abi.PaletteOpts), _P, _P]),
            "or_uv_palette": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, _P, C.c_int32,
                                        C.POINTER(abi.PaletteOpts), _P, _P]),
            "or_block_color_histogram": (None, [_P] + [C.c_int32] * 5 + [_P, _P, _P]),
            "or_dp_palette_center_sets": (None, [_P, _P, C.c_int32, C.c_int32, _P, _P]),
            "or_luma_nearest_indices": (None, [_P] + [C.c_int32] * 5 + [_P, C.c_int32, _P]),
            "or_palette_color_ctx_nb": (None, [C.c_int32] * 4 + [_P, _P]),
            "or_palette_color_ctx": (None, [_P] + [C.c_int32] * 3 + [_P, _P]),
            "or_dirty_log2f": (C.c_float, [C.c_float]),
            "or_leaf16": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                    C.POINTER(abi.CoefCdfs), _P, C.c_int32, C.c_int32, _P, _P, _P]),
            "or_dct1d_32": (None, [_P]),
            "or_quad32_luma": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                         C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P]),
            "or_uv_mode_bits": (C.c_float, [C.POINTER(abi.UvModeCdfs), C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            C.c_int32]),
            "or_pick_uv16_420": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Uv16Params),
                                           C.POINTER(abi.Quant), _P, C.POINTER(abi.CoefCdfs),
                                           C.POINTER(abi.UvModeCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_pick_uv32_444": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Uv16Params),
                                           C.POINTER(abi.Quant), _P, C.POINTER(abi.CoefCdfs),
                                           C.POINTER(abi.UvModeCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_pick_uv32_420": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Uv16Params),
                                           C.POINTER(abi.Quant), _P, C.POINTER(abi.CoefCdfs),
                                           C.POINTER(abi.UvModeCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_pick_uv16_444": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Uv16Params),
                                           C.POINTER(abi.Quant), _P, C.POINTER(abi.CoefCdfs),
                                           C.POINTER(abi.UvModeCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_grid16_luma": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                         C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P]),
            "or_leaf32": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                    C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P, _P]),
            "or_leaf8": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                   C.POINTER(abi.CoefCdfs), _P, C.c_int32, C.c_int32, _P, _P, _P]),
            "or_split16_luma": (C.c_int, [_P, _P, C.POINTER(abi.Split16Params), C.POINTER(abi.Quant), _P,
                                          C.POINTER(abi.CoefCdfs), _P, C.c_int32, _P, _P, _P, C.c_int32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def p(a):
    return None if a is None else a.ctypes.data


def quant_new(qidx, bd=8, qm_level=15):
    q = abi.Quant()
    assert load().or_quant_init(qidx, bd, qm_level, C.byref(q)) == 0
    return q


def quant_new_chroma(qidx, dc_delta, ac_delta, bd=8, qm_level=15):
    q = abi.Quant()
    assert load().or_quant_init_chroma(qidx, dc_delta, ac_delta, bd, qm_level, C.byref(q)) == 0
    return q


def qm_row(level, chroma, n):
    a = load().or_qm_row(level, chroma, n, n)
    if not a:
        return None
    return np.ctypeslib.as_array((C.c_uint8 * (n * n)).from_address(a)).copy()


def default_scan(n):
    a = load().or_default_scan(n)
    return np.ctypeslib.as_array((C.c_uint16 * (n * n)).from_address(a)).copy()


def fwd_txfm_quant(resid, tx_type, q, qm):
    resid = np.ascontiguousarray(resid, np.int32).reshape(-1)
    n = int(round(len(resid) ** 0.5))
    cf = np.zeros(n * n, np.int32)
    tf = np.zeros(n * n, np.float32)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    load().or_fwd_txfm_quant(p(resid), tx_type, n, C.byref(q), p(qm), p(cf), p(tf))
    return cf, tf


def inv_txfm_dequant(levels, tx_type, q, qm):
    levels = np.ascontiguousarray(levels, np.int32).reshape(-1)
    n = int(round(len(levels) ** 0.5))
    out = np.zeros(n * n, np.int32)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    load().or_inv_txfm_dequant(p(levels), tx_type, n, C.byref(q), p(qm), p(out))
    return out


def trellis_optimize(cf, tf, dc_q, ac_q, scan, lambda0):
    cf = np.ascontiguousarray(cf, np.int32).copy()
    tf = np.ascontiguousarray(tf, np.float32)
    scan = np.ascontiguousarray(scan, np.uint16)
    load().or_trellis_optimize(p(cf), p(tf), dc_q, ac_q, p(scan), len(scan), lambda0)
    return cf


def intra_predict(recon, ox, oy, bw, bh, mode, delta=0, have_tr=False, have_bl=False, filter_type=False, bd=8,
                  fw=None, fh=None):
    recon = np.ascontiguousarray(recon, np.uint16)
    h, w = recon.shape
    out = np.zeros(bw * bh, np.int32)
    load().or_intra_predict(p(recon), w, ox, oy, bw, bh, mode, delta, int(have_tr), int(have_bl),
                            fw if fw is not None else w, fh if fh is not None else h, int(filter_type), bd, p(out))
    return out.reshape(bh, bw)


def cdf_cost(cdf, s):
    cdf = np.ascontiguousarray(cdf, np.uint16)
    return load().or_cdf_cost(p(cdf), s)


def coef_costs(cdfs):
    out = abi.CoefCosts()
    load().or_coef_costs_build(C.byref(cdfs), C.byref(out))
    return out


def candidate_chain(src, recon, prm, q, qm, cdfs, cands, want_levels=False, want_recon=False, threads=1):
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    cands = np.ascontiguousarray(cands, abi.CANDIDATE_DTYPE)
    n = len(cands)
    N = prm.tx_size * prm.tx_size
    res = np.zeros(n, abi.RESULT_DTYPE)
    lv = np.zeros((n, N), np.int32) if want_levels else None
    ro = np.zeros((n, N), np.int32) if want_recon else None
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    rc = load().or_candidate_chain(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(cands), n,
                                   p(res), p(lv), p(ro), threads)
    assert rc == 0, rc
    return res, lv, ro


def csc_rgb8(rgb, sub):
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w = rgb.shape[:2]
    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    pcw, pch = (pw >> 1, ph >> 1) if sub == 2 else (pw, ph)
    y = np.zeros((ph, pw), np.uint16)
    cb = np.zeros((pch, pcw), np.uint16)
    cr = np.zeros((pch, pcw), np.uint16)
    assert load().or_csc_rgb8(p(rgb), w, h, sub, p(y), p(cb), p(cr)) == 0
    return y, cb, cr


def deblock_plane(px, vis_w, vis_h, bw4, bh4, level, sharp, is_luma, vedge4=None, hedge4=None, sb_rows4=16, bd=8):
    out = np.array(px, dtype=np.uint16, copy=True, order="C")
    h, w = out.shape
    bw4 = np.ascontiguousarray(bw4, np.uint8)
    bh4 = np.ascontiguousarray(bh4, np.uint8)
    nc4 = bw4.shape[1]
    ve = None if vedge4 is None else np.ascontiguousarray(vedge4, np.uint8)
    he = None if hedge4 is None else np.ascontiguousarray(hedge4, np.uint8)
    assert load().or_deblock_plane(p(out), w, h, vis_w, vis_h, p(bw4), p(bh4), p(ve), p(he), nc4, level, sharp,
                                   int(bool(is_luma)), sb_rows4, bd) == 0
    return out


def weighted_sse(err):
    err = np.ascontiguousarray(err, np.int32)
    h, w = err.shape
    return load().or_weighted_sse(p(err), w, h)


def cdef_frame(recon, src, skip8, prm):
    """Returns (filtered planes, decision dict, tables dict)."""
    mono = bool(prm.mono)
    out = [np.array(x, dtype=np.uint16, copy=True, order="C") for x in recon]
    src = [np.ascontiguousarray(x, np.uint16) for x in src]
    skip8 = np.ascontiguousarray(skip8, np.uint8)
    uc, ur = (prm.w8 + 63) // 64, (prm.h8 + 63) // 64
    nb = (prm.w8 // 8) * (prm.h8 // 8)
    grid = np.zeros(uc * ur, np.uint8)
    tabs = [np.zeros((ur * uc, 12), np.int64) for _ in range(3)]
    dirs = np.zeros(nb, np.uint8)
    vars_ = np.zeros(nb, np.int32)
    d = abi.CdefDecision()
    ch = (lambda a, i: None) if mono else (lambda a, i: p(a[i]))
    assert load().or_cdef_frame(p(out[0]), ch(out, 1), ch(out, 2), p(src[0]), ch(src, 1), ch(src, 2), p(skip8),
                                C.byref(prm), C.byref(d), p(grid), p(tabs[0]), p(tabs[1]), p(tabs[2]), p(dirs),
                                p(vars_)) == 0
    dec = {"bits": d.bits, "damping": d.damping, "unit_cols": d.unit_cols, "unit_rows": d.unit_rows,
           "strengths": [tuple(d.strengths[e]) for e in range(d.n_strengths)], "grid": grid}
    return out, dec, {"luma": tabs[0], "u": tabs[1], "v": tabs[2], "dirs": dirs, "vars": vars_}


def loop_filter_levels(base_q_idx, sub):
    a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
    load().or_loop_filter_levels(base_q_idx, sub, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def deblock_frame(planes, disp_w, disp_h, sub_x, sub_y, tx_maps, pred_maps, lvl_y, lvl_u, lvl_v, mono=False):
    out = [np.array(x, dtype=np.uint16, copy=True, order="C") for x in planes]
    g = abi.DeblockFrameParams()
    g.w8, g.h8 = out[0].shape[1], out[0].shape[0]
    g.disp_w, g.disp_h, g.sub_x, g.sub_y, g.mono, g.bd = disp_w, disp_h, sub_x, sub_y, int(mono), 8
    tm = [np.ascontiguousarray(m, np.uint8) for m in tx_maps]
    pm = [np.ascontiguousarray(m, np.uint8) for m in pred_maps]
    ch = (lambda i: None) if mono else (lambda i: p(out[i]))
    assert load().or_deblock_frame(p(out[0]), ch(1), ch(2), *[p(m) for m in tm], *[p(m) for m in pm], C.byref(g),
                                   lvl_y, lvl_u, lvl_v) == 0
    return out


def real_block_bits_wh(cf, scan, w, h, cdfs, skip_ctx, dcs_ctx, txtp_mode=-1, txtp=0, skip_bits=None):
    cf = np.ascontiguousarray(cf, np.int32)
    scan = np.ascontiguousarray(scan, np.uint16)
    sb = None if skip_bits is None else np.ascontiguousarray(skip_bits, np.float32)
    return load().or_real_block_bits_wh(p(cf), p(scan), w, h, C.byref(cdfs), skip_ctx, dcs_ctx, txtp_mode, txtp,
                                        int(sb is not None), None if sb is None else p(sb))


def dark_protection(plane, base_q, bd=8, enabled=True, sb_x=0, sb_y=0):
    """dark_protection over the SB at (sb_x, sb_y) of a u16 plane (src/aq_common.rs:312-345)."""
    plane = np.ascontiguousarray(plane, np.uint16)
    h, w = plane.shape
    scale = np.float32(1.0) / np.float32(1 << (bd - 8))
    return load().or_dark_protection(int(enabled), base_q, p(plane), w, sb_y, sb_x, w, h, float(scale))


def dark_pow(x):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    load().or_dark_pow(p(x), p(out), x.size)
    return out


def tiling_spec_min(w8, h8):
    a, b = C.c_int32(), C.c_int32()
    assert load().or_tiling_spec_min(w8, h8, C.byref(a), C.byref(b)) == 0
    return a.value, b.value


def aq_grid(luma, prm):
    """Returns (cells (sb_rows, sb_cols) AQ_CELL_DTYPE, tile refs (ntiles, 2) f32)."""
    luma = np.ascontiguousarray(luma, np.uint16)
    sbr, sbc = (prm.h8 + 63) // 64, (prm.w8 + 63) // 64
    cells = np.zeros((sbr, sbc), abi.AQ_CELL_DTYPE)
    tc = -(-sbc // -(-sbc // (1 << prm.tile_cols_log2)))
    tr = -(-sbr // -(-sbr // (1 << prm.tile_rows_log2)))
    refs = np.zeros((tc * tr, 2), np.float32)
    assert load().or_aq_grid(p(luma), C.byref(prm), p(cells), p(refs)) == 0
    return cells, refs


def screen_gate(luma, sub_x, sub_y, base_q_idx, bd=8):
    luma = np.ascontiguousarray(luma, np.uint16)
    prm = abi.ScreenGateParams()
    prm.h8, prm.w8 = luma.shape
    prm.sub_x, prm.sub_y, prm.bd, prm.base_q_idx = sub_x, sub_y, bd, base_q_idx
    r = abi.ScreenGateResult()
    assert load().or_screen_gate(p(luma), C.byref(prm), C.byref(r)) == 0
    return r.as_dict()


def hash8(luma, x, y):
    luma = np.ascontiguousarray(luma, np.uint16)
    return load().or_hash8(p(luma), luma.shape[1], x, y)


def dct1d(buf):
    b = np.ascontiguousarray(buf, np.int32).copy()
    load().or_dct1d(p(b), len(b))
    return b


def mode_beam(src, recon, prm, blocks):
    """(scores, modes): nblocks x 11 each, ascending (score, mode)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.BLOCK8_DTYPE)
    scores = np.zeros((len(blocks), 11), np.uint64)
    modes = np.zeros((len(blocks), 11), np.uint8)
    assert load().or_mode_beam(p(src), p(recon), C.byref(prm), p(blocks), len(blocks), p(scores), p(modes)) == 0
    return scores, modes


def sse_recon(src, vis_w, vis_h, pos, pred, resid, w, h, scale=0.0, bd=8):
    src = np.ascontiguousarray(src, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    pred = np.ascontiguousarray(pred, np.int32)
    resid = None if resid is None else np.ascontiguousarray(resid, np.int32)
    out = np.zeros(len(pos), np.int64)
    assert load().or_sse_recon(p(src), src.shape[1], vis_w, vis_h, bd, p(pos), p(pred), p(resid), len(pos), w, h,
                               scale, p(out)) == 0
    return out


def real_block_bits_bounded(cf, scan, w, h, cdfs, skip_ctx, dcs_ctx, txtp_mode, txtp, bound, skip_bits=None):
    cf = np.ascontiguousarray(cf, np.int32)
    scan = np.ascontiguousarray(scan, np.uint16)
    sb = None if skip_bits is None else np.ascontiguousarray(skip_bits, np.float32)
    return load().or_real_block_bits_bounded(p(cf), p(scan), w, h, C.byref(cdfs), skip_ctx, dcs_ctx, txtp_mode,
                                             txtp, int(sb is not None), None if sb is None else p(sb), bound)


def trellis_optimize_ctx(cf, tf, q, qm, cdfs, dcs_ctx, lambda0, band_tilt=0.0, n=8):
    """trellis_optimize_ctx of one n x n luma block; returns the new levels."""
    cf = np.array(cf, np.int32, copy=True)
    tf = np.ascontiguousarray(tf, np.float32)
    scan = default_scan(n)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    load().or_trellis_optimize_ctx(p(cf), p(tf), float(q.dc_q), float(q.ac_q), p(scan), n, lambda0, C.byref(cdfs),
                                   dcs_ctx, p(qm), q.qm_level, band_tilt)
    return cf


def luma_bits_1d(cf, n, vertical, cdfs, dcs, y_mode):
    cf = np.ascontiguousarray(cf, np.int32)
    return load().or_luma_bits_1d(p(cf), n, int(vertical), C.byref(cdfs), dcs, y_mode)


def coef_res_ctx(cf, n=8):
    cf = np.ascontiguousarray(cf, np.int32)
    scan = default_scan(n)
    return load().or_coef_res_ctx(p(cf), p(scan), n * n)


def split16_luma(src, recon, prm, q, qm, cdfs, jobs, threads=1):
    """split16_luma_try of a batch of jobs: (results, cf n x 256, rec n x 16 x 16)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32)
    rec = np.zeros((n, 16, 16), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    assert load().or_split16_luma(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs), n,
                                  p(res), p(cf), p(rec), threads) == 0
    return res, cf, rec


def split16_depth2(src, recon, prm, q, qm, cdfs, jobs, threads=1):
    """split16_depth2_try of a batch of jobs: (results, cf n x 256, rec n x 16 x 16)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_D2_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32)
    rec = np.zeros((n, 16, 16), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)
    assert load().or_split16_depth2(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs), n,
                                    p(res), p(cf), p(rec), threads) == 0
    return res, cf, rec


def cfl_alpha(luma, src_u, src_v, sub_x, sub_y, cw, ch, blocks, vis=(0, 0), bd=8):
    """cfl_ac + cfl_best_alpha of n chroma blocks: (alpha n x 2, ac n x ch x cw)."""
    luma = np.ascontiguousarray(luma, np.uint16)
    src_u = np.ascontiguousarray(src_u, np.uint16)
    src_v = np.ascontiguousarray(src_v, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.CFL_BLOCK_DTYPE)
    n = len(blocks)
    alpha = np.zeros((n, 2), np.int8)
    ac = np.zeros((n, ch, cw), np.int32)
    assert load().or_cfl_alpha(p(luma), luma.shape[1], p(src_u), p(src_v), src_u.shape[1], sub_x, sub_y, cw, ch,
                               vis[0], vis[1], bd, p(blocks), n, p(alpha), p(ac)) == 0
    return alpha, ac


def filter_intra_predict(recon, ox, oy, w, h, mode, bd=8):
    recon = np.ascontiguousarray(recon, np.uint16)
    out = np.zeros((h, w), np.int32)
    load().or_filter_intra_predict(p(recon), recon.shape[1], ox, oy, w, h, mode, bd, p(out))
    return out


def filter_intra_beam(src, recon, w, h, pos, vis=(0, 0), bd=8):
    """rank_filter_intra_modes of n blocks: (scores n x 5, modes n x 5, preds n x 5 x h x w)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    scores = np.zeros((n, 5), np.uint64)
    modes = np.zeros((n, 5), np.uint8)
    preds = np.zeros((n, 5, h, w), np.int16)
    assert load().or_filter_intra_beam(p(src), p(recon), src.shape[1], src.shape[1], src.shape[0], vis[0], vis[1], bd,
                                       w, h, p(pos), n, p(scores), p(modes), p(preds)) == 0
    return scores, modes, preds


def _chunked(n, threads, run):
    """Runs run(lo, hi) over [0, n) in `threads` contiguous chunks on host
    threads (each chunk is one foreign call; ctypes releases the GIL)."""
    threads = max(1, min(int(threads), n)) if n else 1
    if threads == 1:
        run(0, n)
        return
    import concurrent.futures as cf

    bounds = [(n * k // threads, n * (k + 1) // threads) for k in range(threads)]
    with cf.ThreadPoolExecutor(threads) as ex:
        for f in [ex.submit(run, lo, hi) for lo, hi in bounds if hi > lo]:
            f.result()


def split4tx(src, recon, prm, q, qm, cdfs, jobs, threads=1):
    """split4tx_try of a batch of 8x8 jobs: (results, cf n x 64, rec n x 8 x 8)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_RESULT_DTYPE)
    cf = np.zeros((n, 64), np.int32)
    rec = np.zeros((n, 8, 8), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_split4tx(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs[lo:hi]),
                                  hi - lo, p(res[lo:hi]), p(cf[lo:hi]), p(rec[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf, rec


def leaf8(src, recon, prm, q, qm, cdfs, jobs, refine=False, threads=1):
    """pick_block8's luma candidates / refinement of n 8x8 jobs: (results, cf n x 64, rec n x 8 x 8)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 64), np.int32)
    rec = np.zeros((n, 8, 8), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_leaf8(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs[lo:hi]),
                           hi - lo, int(bool(refine)), p(res[lo:hi]), p(cf[lo:hi]), p(rec[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf, rec


def leaf16(src, recon, prm, q, qm, cdfs, jobs, refine=False, threads=1):
    """pick_luma16's mode-loop candidates / refinement of n 16x16 jobs: (results, cf n x 256, rec n x 16 x 16)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32)
    rec = np.zeros((n, 16, 16), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_leaf16(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs[lo:hi]),
                           hi - lo, int(bool(refine)), p(res[lo:hi]), p(cf[lo:hi]), p(rec[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf, rec


def dct1d_32(buf):
    """dct1d_32_i32 of 32 integers."""
    b = np.ascontiguousarray(buf, np.int32).copy()
    load().or_dct1d_32(p(b))
    return b


def leaf32(src, recon, prm, q, qm, cdfs, jobs, threads=1):
    """pick_luma32's mode-loop candidates of n 32x32 jobs: (results, cf n x 1024, rec n x 32 x 32)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 1024), np.int32)
    rec = np.zeros((n, 32, 32), np.uint16)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_leaf32(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs), p(jobs[lo:hi]),
                                hi - lo, p(res[lo:hi]), p(cf[lo:hi]), p(rec[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf, rec


def quad32_luma(src, recon, prm, q, qm, cdfs, jobs, threads=1):
    """rd_pick_luma64's four-TX_32X32 leg of n (64x64 block, mode, delta) jobs: the results."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.QUAD32_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.QUAD32_RESULT_DTYPE)
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_quad32_luma(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs),
                                     p(jobs[lo:hi]), hi - lo, p(res[lo:hi])) == 0

    _chunked(n, threads, run)
    return res


def luma_palette(src, w, h, pos, opts, bd=8):
    """Lossy luma palette candidates of n w x h blocks: (candidates n x 14, maps n x 14 x h x w)."""
    src = np.ascontiguousarray(src, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    cands = np.zeros((n, abi.PALETTE_SLOTS), abi.PALETTE_CAND_DTYPE)
    maps = np.zeros((n, abi.PALETTE_SLOTS, h, w), np.uint8)
    assert load().or_luma_palette(p(src), src.shape[1], src.shape[1], src.shape[0], bd, w, h, p(pos), n,
                                  C.byref(opts), p(cands), p(maps)) == 0
    return cands, maps


def uv_palette(src_u, src_v, w, h, pos, opts):
    """UV palette candidates of n w x h chroma blocks: (candidates n x 4, maps n x 4 x h x w)."""
    src_u = np.ascontiguousarray(src_u, np.uint16)
    src_v = np.ascontiguousarray(src_v, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    cands = np.zeros((n, abi.UV_PALETTE_SLOTS), abi.UV_PALETTE_CAND_DTYPE)
    maps = np.zeros((n, abi.UV_PALETTE_SLOTS, h, w), np.uint8)
    assert load().or_uv_palette(p(src_u), p(src_v), src_u.shape[1], w, h, p(pos), n, C.byref(opts), p(cands),
                                p(maps)) == 0
    return cands, maps


def block_color_histogram(src, px, py, w, h):
    """(values, counts) ascending, or None when the block has < 2 or > 64 distinct values."""
    src = np.ascontiguousarray(src, np.uint16)
    vals = np.zeros(64, np.int32)
    cnts = np.zeros(64, np.uint32)
    nn = C.c_int32()
    load().or_block_color_histogram(p(src), src.shape[1], px, py, w, h, p(vals), p(cnts), C.byref(nn))
    return None if nn.value == 0 else (vals[:nn.value].copy(), cnts[:nn.value].copy())


def dp_palette_center_sets(hist, kmax=8):
    """Optimal centre sets for sizes 2..kmax of a [(value, count)] histogram: list of 7 lists."""
    vals = np.ascontiguousarray([v for v, _ in hist], np.int32)
    cnts = np.ascontiguousarray([c for _, c in hist], np.uint32)
    sets = np.zeros((7, 8), np.int32)
    lens = np.zeros(7, np.int32)
    load().or_dp_palette_center_sets(p(vals), p(cnts), len(hist), kmax, p(sets), p(lens))
    return [sets[k, :lens[k]].tolist() for k in range(7)]


def luma_nearest_indices(src, px, py, w, h, centers):
    src = np.ascontiguousarray(src, np.uint16)
    c = np.ascontiguousarray(centers, np.int32)
    out = np.zeros(w * h, np.uint8)
    load().or_luma_nearest_indices(p(src), src.shape[1], px, py, w, h, p(c), len(c), p(out))
    return out


def palette_color_ctx_nb(l, u, ul, cur):
    a, b = C.c_int32(), C.c_int32()
    load().or_palette_color_ctx_nb(-1 if l is None else l, -1 if u is None else u, ul, cur, C.byref(a), C.byref(b))
    return a.value, b.value


def palette_color_ctx(map_, stride, y, x):
    m = np.ascontiguousarray(map_, np.uint8)
    a, b = C.c_int32(), C.c_int32()
    load().or_palette_color_ctx(p(m), stride, y, x, C.byref(a), C.byref(b))
    return a.value, b.value


def dirty_log2f(d):
    return load().or_dirty_log2f(d)


# ---------------------------------------------------------------------------
# The default decision snapshot and the frame laws, restated for the checker.

GOLDEN_CDFS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                           "cdfs_default.json")
_GOLDEN = None


def _golden_cdfs():
    global _GOLDEN
    if _GOLDEN is None:
        import json

        _GOLDEN = json.load(open(GOLDEN_CDFS))
    return _GOLDEN


def _icdf(vals, width):
    """src/tables.rs:31-35 icdf: 32768 - v per entry, then the terminal 0."""
    out = np.zeros(width, np.uint16)
    out[:len(vals)] = [32768 - v for v in vals]
    return out


def default_cdfs(qctx, w, h=None, plane=0):
    """One (class, plane) coefficient slice of Cdfs::new(qctx)
    (src/coder/cdfs.rs:401-629) from the reference's arrays
    (tests/golden/cdfs_default.json): class by the AV1 txSzCtx of w x h, eob_pt
    CDF by coefficient count (capped at 1024), the 1-D eob_pt CDF for luma
    16 / 64 / 128, the tx-type CDFs for luma without a 32-point side (INTRA1
    at square sizes 4 / 8, INTRA2 at 16)."""
    h = w if h is None else h
    g = _golden_cdfs()
    lg = {4: 0, 8: 1, 16: 2, 32: 3, 64: 4}
    sqr, up = min(lg[w], lg[h]), max(lg[w], lg[h])
    n = (4, 8, 16, 32, 64)[(sqr + up + 1) >> 1]
    pl = "CHROMA" if plane else "LUMA"
    c = abi.CoefCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    arr("txb_skip")[...] = np.stack([_icdf([v], 2) for v in g[f"SKIP_TX{n}"][qctx]])
    bt = arr("base_tok")
    for k, row in enumerate(g[f"BASE_TOK_TX{n}_{pl}_Q"][qctx]):
        bt[k] = _icdf(row, 4)
    br = arr("br_tok")
    for k, row in enumerate(g[f"BR_TOK_TX{min(n, 32)}_{pl}_Q"][qctx]):
        br[k] = _icdf(row, 4)
    arr("eob_base")[...] = np.stack([_icdf(r, 3) for r in g[f"EOB_BASE_TX{n}_{pl}_Q"][qctx]])
    arr("eob_hi")[...] = np.stack([_icdf([v], 2) for v in g[f"EOB_HI_TX{n}_{pl}"][qctx]])
    arr("dc_sign")[...] = np.stack([_icdf([v], 2) for v in g["DC_SIGN_Q"][qctx][plane]])
    area = min(w * h, 1024)
    arr("eob_bin")[...] = _icdf(g[f"EOB_BIN_{area}_{pl}"][qctx], 11)
    if plane == 0 and area in (16, 64, 128):
        arr("eob_bin_1d")[...] = _icdf(g[f"EOB_BIN_{area}_LUMA_1D"][qctx], 11)
    if plane == 0 and up <= 2:
        tab = g[("TXTP_INTRA1_TX4", "TXTP_INTRA1_TX8", "TXTP_INTRA2_TX16")[sqr]]
        tx = arr("txtp")
        for m, row in enumerate(tab):
            tx[m] = _icdf(row, 16)
    return c


def qcat(q):
    """src/coef_q.rs:31-41."""
    return 0 if q <= 20 else 1 if q <= 60 else 2 if q <= 120 else 3


def quality_to_q(quality):
    """src/avif.rs:637-666 quality_to_q."""
    anchors = [(1, 215), (30, 140), (40, 116), (50, 91), (60, 70), (70, 53), (80, 35), (85, 28), (90, 17),
               (93, 12), (96, 7), (98, 5), (99, 3), (100, 1)]
    q = min(max(quality, 1), 100)
    prev = anchors[0]
    for l1, q1 in anchors[1:]:
        if q <= l1:
            l0, q0 = prev
            t = q - l0
            v = q0 + int((q1 - q0) * t / max(l1 - l0, 1))  # Rust i32 division truncates toward zero
            return min(max(v, 1), 255)
        prev = (l1, q1)
    return 1


_f32 = np.float32


def _fast_round(v):
    """src/util.rs:36-59 fast_round (x86-64)."""
    b = np.array([v], _f32).view(np.uint32) + np.uint32(1)
    u = b.view(_f32)[0]
    magic = _f32((1 << 23) + (1 << 22))
    return _f32(_f32(u + magic) - magic)


def qm_level_law(q, sub):
    """src/quant.rs:138-153."""
    f = _f32
    qi = f(q)
    top = f(8.0) if sub else f(15.0)
    if qi <= 20:
        return 8 if sub else 15
    if qi <= 48:
        return int(_fast_round(f(top + f(f((f(8.0) - top) * f(qi - f(20.0))) / f(28.0)))))
    if qi >= 128:
        return 0
    return int(_fast_round(f(f(f(8.0) * f(f(128.0) - qi)) / f(80.0))))


def qm_chroma_level_law(q, sub):
    """src/quant.rs:155-167 (top_ease 1, qm_hq knee 12 width 5)."""
    f = _f32
    if sub:
        return qm_level_law(q, sub)
    pinned = min(2, qm_level_law(q, sub))
    t = f(np.clip(f(f(f(12.0) - f(q)) / f(5.0)), 0, 1))
    if t > 0:
        v = f(f(pinned) + f(f(f(15.0) - f(pinned)) * t))
        return int(np.floor(v + 0.5))
    return pinned


def rd_lambdas(q, dc_q, sub):
    """The frame's decision lambdas as abi.RdLambdas (8-bit): src/cost.rs:122-148
    (aom_ssimulacra2_rdmult_weight, mode_lambda_weight), :286-292 (mode_lambda_q),
    src/partition_rd.rs:30-71 (luma_satd_scale, k_satd),
    src/coder/lossy_state.rs:1769-1789, :2396-2408, with the shipped tuning."""
    f = _f32
    scale = {2: f(0.8), 1: f(0.65), 0: f(0.6)}[sub]
    w = f(f(min(max(((255 - q) * 3) // 4, 0), 72) + 128) * f(1.0 / 128.0))
    if sub == 1:
        weight = f(w * scale)
    else:
        r = f(np.clip(f(f(f(q) - f(0.0)) / f(72.0)), 0, 1))
        weight = f(f(f(3.0) + f(f(w - f(3.0)) * r)) * scale)
    dc = f(dc_q)
    mult = f(f(3.3) + f(f(0.0015) * dc))
    mlq = f(f(f(f(f(0.009005174719460433) * f(1.0)) * dc) * dc) * mult)
    out = abi.RdLambdas()
    out.mode_lambda = f(mlq * weight)
    out.lambda_d = f(f(out.mode_lambda) / f(2.775))
    out.trellis_lambda0 = f(0.05)
    qi = f(q)
    if sub:
        out.satd_scale = f(1.25)
    elif qi <= 20:
        out.satd_scale = f(2.921556)
    elif qi >= 48:
        out.satd_scale = f(1.25)
    else:
        out.satd_scale = f(f(2.921556) + f(f(f(f(1.25) - f(2.921556)) * f(qi - f(20.0))) / f(28.0)))
    k = [f(24.5), f(21.3), f(18.2)] if sub else [f(35.0), f(21.2), f(18.1)]
    if qi <= 28:
        ks = k[0]
    elif qi >= 140:
        ks = k[2]
    elif qi <= 81:
        ks = f(k[0] + f(f(f(k[1] - k[0]) * f(qi - f(28.0))) / f(53.0)))
    else:
        ks = f(k[1] + f(f(f(k[2] - k[1]) * f(qi - f(81.0))) / f(59.0)))
    out.satd_bridge = f(f(f(2.775) / ks) * f(7.130643))
    return out


# ---------------------------------------------------------------------------
# Entropy path checker: the range decoder (oracle_entropy.cpp) and Cdfs::new
# assembled in semantic-slot order from the reference's arrays.

class RangeDecoder:
    """OdEcDecoder (src/odec.rs:615-760) over a byte string."""

    def __init__(self, data):
        self._buf = C.create_string_buffer(bytes(data), max(1, len(data)))
        lib = load()
        lib.or_dec_new.restype = C.c_void_p
        lib.or_dec_new.argtypes = [C.c_void_p, C.c_size_t]
        lib.or_dec_free.argtypes = [C.c_void_p]
        lib.or_dec_bool.argtypes = [C.c_void_p, C.c_uint16]
        lib.or_dec_literal.restype = C.c_uint32
        lib.or_dec_literal.argtypes = [C.c_void_p, C.c_uint32]
        lib.or_dec_symbol.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        lib.or_dec_signed_subexp_with_ref.restype = C.c_int32
        lib.or_dec_signed_subexp_with_ref.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_uint32, C.c_int32]
        self._d = lib.or_dec_new(C.addressof(self._buf), len(data))

    def bool(self, f):
        return bool(load().or_dec_bool(self._d, f))

    def literal(self, bits):
        return load().or_dec_literal(self._d, bits)

    def symbol(self, cdf, adapt=True):
        assert cdf.dtype == np.uint16 and cdf.flags.c_contiguous
        return load().or_dec_symbol(self._d, cdf.ctypes.data, len(cdf), int(bool(adapt)))

    def signed_subexp_with_ref(self, low, high, k, r):
        return load().or_dec_signed_subexp_with_ref(self._d, low, high, k, r)

    def __del__(self):
        if getattr(self, "_d", None):
            load().or_dec_free(self._d)
            self._d = None


def cdfs_new_slots(qctx, sections=None):
    """Cdfs::new(qctx) (src/coder/cdfs.rs:401-629) as a list of np.uint16 inverse
    CDFs (counter last) in Cdfs::semantic_slots order (src/coder/cdfs.rs:193-355),
    from the reference's arrays (tests/golden/cdfs_default.json); the values
    Cdfs::new writes inline are listed with their source lines."""
    g = _golden_cdfs()
    out = []

    def one(vals):
        out.append(np.array([32768 - v for v in vals] + [0], np.uint16))

    def rows(t):
        for r in t:
            one(r)

    def singles(t):
        for v in t:
            one([v])

    def flat(t):
        while isinstance(t[0], list):
            t = [x for row in t for x in row]
        return t

    sec = sections if sections is not None else {}
    sec["skip"] = len(out)
    singles(g["SKIP_CDF"])
    one([30531])  # intrabc (cdfs.rs:508)
    singles([28581, 23846, 20847, 24315, 18196, 12133, 18791, 10887, 11005, 27179, 20004, 11281, 26549, 19308,
             14224, 28015, 21546, 14400, 28165, 22401, 16088])  # TXPART_CDF (cdfs.rs:71-79)
    one([770, 2421, 5225, 12907, 15819, 18927, 21561, 24089, 26595, 28526, 30529])  # txtp_inter2 (:513-515)
    singles([16384, 4167, 1998, 748])  # txtp_inter3 (:516-519)
    one([4096, 11264, 19328])  # mv_joint
    for _ in range(2):
        one([16384])  # mv_sign
    for _ in range(2):
        one([28672, 30976, 31858, 32320, 32551, 32656, 32740, 32757, 32762, 32767])  # mv_classes
    for _ in range(2):
        one([27648])  # mv_class0
    for _ in range(2):
        singles([17408, 17920, 18944, 20480, 22528, 24576, 28672, 29952, 29952, 30720])  # mv_class_n
    sec["part_bl8"] = len(out)
    rows(g["PART_BL8_CDF"])
    sec["part_split"] = len(out)
    for lvl in g["PART_SPLIT_CDF"]:
        rows(lvl)
    sec["kf_y"] = len(out)
    for a in g["KF_Y_MODE_CDF"]:
        rows(a)
    sec["uv_mode"] = len(out)
    rows(g["UV_MODE_NOCFL_CDF"])
    rows(g["UV_MODE_CFL_CDF"])
    sec["angle_delta"] = len(out)
    rows(g["ANGLE_DELTA_CDF"])
    sec["filter_intra"] = len(out)
    singles(g["FILTER_INTRA_CDF"])
    one(g["FILTER_INTRA_MODE_CDF"])
    sec["palette_y_mode"] = len(out)
    singles(flat(g["PALETTE_Y_MODE"]))
    ys = g["PALETTE_Y_SIZE"]
    rows([ys[k * 6:(k + 1) * 6] for k in range(7)])
    sec["palette_uv_mode"] = len(out)
    singles([32461, 21488])  # palette_uv_mode (cdfs.rs:573)
    for n in range(2, 9):
        for ctx in range(5):
            one(g["PALETTE_Y_COLOR"][f"{n},{ctx}"])
    us = g["PALETTE_UV_SIZE"]
    rows([us[k * 6:(k + 1) * 6] for k in range(7)])
    for n in range(2, 9):
        t = g["PALETTE_UV_COLOR"][str(n)]
        rows([t[c * (n - 1):(c + 1) * (n - 1)] for c in range(5)])
    one(g["CFL_SIGN_CDF"])
    rows(g["CFL_ALPHA_CDF"])
    sec["txsz"] = len(out)
    for k in range(4):
        rows(g[f"TXSZ_CAT{k}_CDF"])
    sec["txtp8"] = len(out)
    rows(g["TXTP_INTRA1_TX8"])
    sec["txtp4"] = len(out)
    rows(g["TXTP_INTRA1_TX4"])
    sec["txtp16"] = len(out)
    rows(g["TXTP_INTRA2_TX16"])
    for k, n in enumerate((4, 8, 16, 32, 64)):
        sec[f"txb_skip{k}"] = len(out)
        singles(g[f"SKIP_TX{n}"][qctx])
    for k, n in enumerate((4, 8, 16, 32)):
        for pi, p in enumerate(("LUMA", "CHROMA")):
            sec[f"base_tok{k}{pi}"] = len(out)
            rows(g[f"BASE_TOK_TX{n}_{p}_Q"][qctx])
    sec["base_tok40"] = len(out)
    rows(g["BASE_TOK_TX64_LUMA_Q"][qctx])
    for k, n in enumerate((4, 8, 16, 32)):
        for pi, p in enumerate(("LUMA", "CHROMA")):
            sec[f"br_tok{k}{pi}"] = len(out)
            rows(g[f"BR_TOK_TX{n}_{p}_Q"][qctx])
    for k, n in enumerate((4, 8, 16, 32)):
        for pi, p in enumerate(("LUMA", "CHROMA")):
            sec[f"eob_base{k}{pi}"] = len(out)
            rows(g[f"EOB_BASE_TX{n}_{p}_Q"][qctx])
    sec["eob_base40"] = len(out)
    rows(g["EOB_BASE_TX64_LUMA_Q"][qctx])
    for k, n in enumerate((4, 8, 16, 32)):
        for pi, p in enumerate(("LUMA", "CHROMA")):
            sec[f"eob_hi{k}{pi}"] = len(out)
            singles(g[f"EOB_HI_TX{n}_{p}"][qctx])
    sec["eob_hi40"] = len(out)
    singles(g["EOB_HI_TX64_LUMA"][qctx])
    for p in range(2):
        sec[f"dc_sign{p}"] = len(out)
        singles(g["DC_SIGN_Q"][qctx][p])
    sec["eob_bin"] = len(out)
    for name in ("16_CHROMA", "16_LUMA", "32_CHROMA", "32_LUMA", "64_LUMA", "16_LUMA_1D", "64_LUMA_1D",
                 "128_LUMA_1D", "64_CHROMA", "256_LUMA", "256_CHROMA", "128_CHROMA", "128_LUMA", "1024_LUMA",
                 "1024_CHROMA", "512_CHROMA", "512_LUMA"):
        one(g[f"EOB_BIN_{name}"][qctx])
    one([28160, 32120, 32677])  # delta_q (cdfs.rs:621)
    one([11570])  # wiener_restore (tile_encode.rs:34-36)
    return out


def gather_split_prob(cdf, top):
    """gather_split_prob_icdf (src/coeffs.rs:2927-2935)."""
    v = [int(x) for x in cdf]
    out = (v[1] - v[4]) + v[5] + (v[8] - v[7]) if top else (v[0] - v[1]) + (v[2] - v[6]) + (v[7] - v[8])
    return min(max(out, 1), 32767)


class EmitSlots(C.Structure):
    """The CDF groups the coefficient coders touch, as slot numbers."""
    _fields_ = [("txb_skip", C.c_int32 * 4), ("base_tok", (C.c_int32 * 2) * 4), ("br_tok", (C.c_int32 * 2) * 4),
                ("eob_base", (C.c_int32 * 2) * 4), ("eob_hi", (C.c_int32 * 2) * 4), ("dc_sign", C.c_int32 * 2),
                ("eob_bin", C.c_int32), ("txtp4", C.c_int32), ("txtp8", C.c_int32), ("txtp16", C.c_int32)]


def emit_slots(qctx=0):
    sec = {}
    cdfs_new_slots(qctx, sec)
    e = EmitSlots()
    for k in range(4):
        e.txb_skip[k] = sec[f"txb_skip{k}"]
        for p in range(2):
            e.base_tok[k][p] = sec[f"base_tok{k}{p}"]
            e.br_tok[k][p] = sec[f"br_tok{k}{p}"]
            e.eob_base[k][p] = sec[f"eob_base{k}{p}"]
            e.eob_hi[k][p] = sec[f"eob_hi{k}{p}"]
    e.dc_sign[0], e.dc_sign[1] = sec["dc_sign0"], sec["dc_sign1"]
    e.eob_bin, e.txtp4, e.txtp8, e.txtp16 = sec["eob_bin"], sec["txtp4"], sec["txtp8"], sec["txtp16"]
    return e, sec


def emit_coeffs(levels, blocks):
    """The oracle's coefficient coders over a block list: (tokens, offsets, res_ctx)."""
    levels = np.ascontiguousarray(levels, np.int32).ravel()
    blocks = np.ascontiguousarray(blocks, abi.COEF_BLOCK_DTYPE)
    n = len(blocks)
    e, _ = emit_slots()
    cap = int(sum(8 + 40 * (1 << (2 * int(b))) for b in blocks["log2n"])) + 1
    toks = np.zeros(cap, np.uint32)
    offsets = np.zeros(n + 1, np.uint32)
    res = np.zeros(max(n, 1), np.uint8)
    lib = load()
    lib.or_emit_coeffs.restype = C.c_int
    lib.or_emit_coeffs.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                   C.c_void_p]
    assert lib.or_emit_coeffs(p(levels), p(blocks), n, C.addressof(e), p(toks), cap, p(offsets), p(res)) == 0
    return toks[:offsets[n]].copy(), offsets, res[:n]


def grid16_luma(src, recon, prm, q, qm, cdfs, jobs, threads=1, want_cf=False):
    """rd_pick_luma64's sixteen-TX_16X16 leg of n (64x64 block, mode, delta) jobs:
    (results, levels or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.GRID16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.GRID16_RESULT_DTYPE)
    cf = np.zeros((n, 4096), np.int32) if want_cf else None
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert load().or_grid16_luma(p(src), p(recon), C.byref(prm), C.byref(q), p(qm), C.byref(cdfs),
                                     p(jobs[lo:hi]), hi - lo, p(res[lo:hi]),
                                     None if cf is None else p(cf[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf


def uv_mode_cdfs():
    """The mode CDFs uv_mode_bits reads, from the reference's default arrays
    (tests/golden/cdfs_default.json): uv_mode with CfL allowed per y mode,
    angle_delta per directional mode, cfl_sign, cfl_alpha."""
    g = _golden_cdfs()
    c = abi.UvModeCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    um = np.asarray(g["UV_MODE_CFL_CDF"]).reshape(13, 13)
    arr("uv_mode")[...] = np.stack([_icdf(r, 14) for r in um])
    ad = np.asarray(g["ANGLE_DELTA_CDF"]).reshape(8, 6)
    arr("angle_delta")[...] = np.stack([_icdf(r, 7) for r in ad])
    arr("cfl_sign")[...] = _icdf(np.asarray(g["CFL_SIGN_CDF"]).reshape(-1), 8)
    ca = np.asarray(g["CFL_ALPHA_CDF"]).reshape(6, 15)
    arr("cfl_alpha")[...] = np.stack([_icdf(r, 16) for r in ca])
    return c


def uv_mode_bits(cdfs, y_mode, uv_mode, cfl=None):
    au, av = cfl if cfl is not None else (0, 0)
    return load().or_uv_mode_bits(C.byref(cdfs), y_mode, uv_mode, int(cfl is not None), au, av)


def _pick_uv16(entry, dtype, per_job, src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm, cdfs, mode_cdfs, jobs,
               threads, want_cf, want_rec):
    planes = [np.ascontiguousarray(a, np.uint16) for a in (src_u, src_v, rec_u, rec_v, luma)]
    jobs = np.ascontiguousarray(jobs, dtype)
    n = len(jobs)
    res = np.zeros(n, abi.UV16_RESULT_DTYPE)
    cf = np.zeros((n, per_job), np.int32) if want_cf else None
    rec = np.zeros((n, per_job), np.uint16) if want_rec else None
    qm = None if qm is None else np.ascontiguousarray(qm, np.uint8)

    def run(lo, hi):
        assert getattr(load(), entry)(*[p(a) for a in planes], C.byref(prm), C.byref(uvp), C.byref(q), p(qm),
                                      C.byref(cdfs), C.byref(mode_cdfs), p(jobs[lo:hi]), hi - lo, p(res[lo:hi]),
                                      None if cf is None else p(cf[lo:hi]),
                                      None if rec is None else p(rec[lo:hi])) == 0

    _chunked(n, threads, run)
    return res, cf, rec


def pick_uv16_420(src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm, cdfs, mode_cdfs, jobs, threads=1,
                  want_cf=False, want_rec=False):
    """pick_uv16_420 of n 16x16 leaves: (results, levels or None, reconstruction or None)."""
    return _pick_uv16("or_pick_uv16_420", abi.UV16_JOB_DTYPE, 128, src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm,
                      cdfs, mode_cdfs, jobs, threads, want_cf, want_rec)


def pick_uv16_444(src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm, cdfs, mode_cdfs, jobs, threads=1,
                  want_cf=False, want_rec=False):
    """pick_uv16_444 of n 16x16 leaves: (results, levels or None, reconstruction or None)."""
    return _pick_uv16("or_pick_uv16_444", abi.UV16_444_JOB_DTYPE, 512, src_u, src_v, rec_u, rec_v, luma, prm, uvp, q,
                      qm, cdfs, mode_cdfs, jobs, threads, want_cf, want_rec)


def pick_uv32_420(src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm, cdfs, mode_cdfs, jobs, threads=1,
                  want_cf=False, want_rec=False):
    """pick_uv32_420 of n 32x32 leaves: (results, levels or None, reconstruction or None)."""
    return _pick_uv16("or_pick_uv32_420", abi.UV16_444_JOB_DTYPE, 512, src_u, src_v, rec_u, rec_v, luma, prm, uvp, q,
                      qm, cdfs, mode_cdfs, jobs, threads, want_cf, want_rec)


def pick_uv32_444(src_u, src_v, rec_u, rec_v, luma, prm, uvp, q, qm, cdfs, mode_cdfs, jobs, threads=1,
                  want_cf=False, want_rec=False):
    """pick_uv32_444 of n 32x32 leaves: (results, levels or None, reconstruction or None)."""
    return _pick_uv16("or_pick_uv32_444", abi.UV32_444_JOB_DTYPE, 2048, src_u, src_v, rec_u, rec_v, luma, prm, uvp, q,
                      qm, cdfs, mode_cdfs, jobs, threads, want_cf, want_rec)

