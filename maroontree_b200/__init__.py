"""maroontree_b200: B200-native intra rate-distortion core of the maroontree AVIF
encoder, behind a C ABI (``include/maroontree_b200.h``).

Python here is a thin host mirror over that ABI (ctypes); the arithmetic runs
in the sm_100a kernels of ``csrc/``.  There is no CPU fallback: the calls raise
when the library or a CUDA device is missing.
"""
import ctypes as C

import numpy as np

from . import abi
from .abi import (CANDIDATE_DTYPE, RESULT_DTYPE, ChainParams, CoefCdfs, CoefCosts, Quant, load, ptr)

__all__ = [
    "abi", "load", "Quant", "CoefCdfs", "CoefCosts", "ChainParams", "CANDIDATE_DTYPE", "RESULT_DTYPE",
    "quant_new", "quant_new_chroma", "qm_row", "default_scan", "qcat", "coef_cdfs_default", "quality_to_q", "qm_levels", "rd_lambdas", "coef_costs", "chain_params", "candidate_chain",
    "candidate_chain_device", "chain_scratch_bytes", "rdo_level8", "rdo_level8_device", "rdo_level8_scratch_bytes", "rdo_level4", "padded_plane_dims", "csc_rgb8", "deblock_plane", "loop_filter_levels", "deblock_frame", "cdef_params", "cdef_frame", "MtError",
]


class MtError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"{what} failed with code {code}")
        self.code = code


def _check(rc, what):
    if rc != abi.MT_OK:
        raise MtError(rc, what)


def quant_new(base_q_idx, bd=8, qm_level=15):
    """``Quant::new_with_qm`` (src/quant.rs:351-373)."""
    q = Quant()
    _check(load().mt_quant_init(base_q_idx, bd, qm_level, C.byref(q)), "mt_quant_init")
    return q


def quant_new_chroma(base_q_idx, dc_delta, ac_delta, bd=8, qm_level=15):
    """``Quant::new_chroma_with_delta_qm`` (src/quant.rs:393-418)."""
    q = Quant()
    _check(load().mt_quant_init_chroma(base_q_idx, dc_delta, ac_delta, bd, qm_level, C.byref(q)),
           "mt_quant_init_chroma")
    return q


def qm_row(level, chroma, n):
    """Inverse QM weights of an n x n transform as a numpy array, or None when flat."""
    p = load().mt_qm_row(level, chroma, n, n)
    if not p:
        return None
    return np.ctypeslib.as_array((C.c_uint8 * (n * n)).from_address(p)).copy()


def default_scan(n):
    p = load().mt_default_scan(n)
    return np.ctypeslib.as_array((C.c_uint16 * (n * n)).from_address(p)).copy()


def quality_to_q(quality):
    """``quality_to_q`` (src/avif.rs:637-666)."""
    return load().mt_quality_to_q(quality)


def qm_levels(base_q_idx, sub):
    """(luma, chroma) quantisation-matrix levels of the QM level laws (src/quant.rs:138-167)."""
    y, uv = C.c_uint8(), C.c_uint8()
    _check(load().mt_qm_levels(base_q_idx, sub, C.byref(y), C.byref(uv)), "mt_qm_levels")
    return y.value, uv.value


def rd_lambdas(base_q_idx, dc_q, sub, bd=8):
    """The frame's decision lambdas (``abi.RdLambdas``): mlam, lambda_d, trellis
    lambda0, the SATD scale and bridge of the luma proxy."""
    out = abi.RdLambdas()
    _check(load().mt_rd_lambdas_init(base_q_idx, dc_q, sub, bd, C.byref(out)), "mt_rd_lambdas_init")
    return out


def qcat(base_q_idx):
    """Coefficient CDF q context of a base qindex (``qcat``, src/coef_q.rs:31-41)."""
    return load().mt_qcat(base_q_idx)


def coef_cdfs_default(qctx, tx_w, tx_h=None, plane=0):
    """The (class, plane) coefficient slice of the default decision snapshot
    ``Cdfs::new(qctx)`` (src/coder/cdfs.rs:401-629) for a tx_w x tx_h transform."""
    c = CoefCdfs()
    _check(load().mt_coef_cdfs_default(qctx, tx_w, tx_w if tx_h is None else tx_h, plane, C.byref(c)),
           "mt_coef_cdfs_default")
    return c


def coef_costs(cdfs):
    out = CoefCosts()
    _check(load().mt_coef_costs_build(C.byref(cdfs), C.byref(out)), "mt_coef_costs_build")
    return out


def chain_params(frame_w, frame_h, stride=None, tx_size=8, trellis_lambda0=0.05, mode_lambda=1.0,
                 satd_scale=1.25, satd_bridge=0.0, skip_bits=None, vis=None):
    p = ChainParams()
    p.tx_size, p.bd, p.frame_w, p.frame_h = tx_size, 8, frame_w, frame_h
    if vis is not None:
        p.vis_w, p.vis_h = vis
    p.stride = stride if stride is not None else frame_w
    p.trellis_lambda0, p.mode_lambda, p.satd_scale, p.satd_bridge = trellis_lambda0, mode_lambda, satd_scale, satd_bridge
    if skip_bits is not None:
        p.use_skip_bits = 1
        p.skip_bits[0], p.skip_bits[1] = skip_bits
    return p


def candidate_chain(src, recon, prm, quant, qmrow, costs, cands, want_levels=False, want_recon=False):
    """Evaluate the candidate chain with host buffers (copies in and out)."""
    lib = load()
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    cands = np.ascontiguousarray(cands, CANDIDATE_DTYPE)
    n = len(cands)
    N = prm.tx_size * prm.tx_size
    res = np.zeros(n, RESULT_DTYPE)
    lv = np.zeros((n, N), np.int32) if want_levels else None
    ro = np.zeros((n, N), np.int32) if want_recon else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(lib.mt_candidate_chain(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                                  ptr(cands), n, ptr(res), ptr(lv), ptr(ro)), "mt_candidate_chain")
    return res, lv, ro


def candidate_chain_device(d_src, d_recon, prm, quant, d_qm, d_costs, d_cands, n, d_res, d_lv=None, d_ro=None,
                           d_scratch=None, stream=0):
    """Device-pointer form: arguments are torch CUDA tensors (or raw addresses)."""
    _check(load().mt_candidate_chain_device(ptr(d_src), ptr(d_recon), C.byref(prm), C.byref(quant), ptr(d_qm),
                                            ptr(d_costs), ptr(d_cands), n, ptr(d_res), ptr(d_lv), ptr(d_ro),
                                            ptr(d_scratch), stream or None), "mt_candidate_chain_device")


def chain_scratch_bytes(n):
    return load().mt_candidate_chain_scratch_bytes(n)


def rdo_level8(src, recon, prm, quant, qmrow, costs, blocks, combos, want_results=False):
    """One batched RDO level with host buffers: per-block best (and optionally
    every candidate result, combo-major)."""
    lib = load()
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.BLOCK8_DTYPE)
    combos = np.ascontiguousarray(combos, abi.COMBO_DTYPE)
    best = np.zeros(len(blocks), abi.BEST_DTYPE)
    res = np.zeros(len(blocks) * len(combos), RESULT_DTYPE) if want_results else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(lib.mt_rdo_level8(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                             ptr(blocks), len(blocks), ptr(combos), len(combos), ptr(best), ptr(res)),
           "mt_rdo_level8")
    return best, res


def rdo_level4(src, recon, prm, quant, qmrow, costs, blocks, combos, want_results=False):
    """The batched 4x4 level (``mt_rdo_level4``): blocks on the 4-sample grid,
    prm.tx_size = 4, the 16-entry 4x4 QM row and the TX_4X4 cost slice."""
    lib = load()
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.BLOCK8_DTYPE)
    combos = np.ascontiguousarray(combos, abi.COMBO_DTYPE)
    best = np.zeros(len(blocks), abi.BEST_DTYPE)
    res = np.zeros(len(blocks) * len(combos), RESULT_DTYPE) if want_results else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(lib.mt_rdo_level4(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                             ptr(blocks), len(blocks), ptr(combos), len(combos), ptr(best), ptr(res)),
           "mt_rdo_level4")
    return best, res


def rdo_level16(src, recon, prm, quant, qmrow, costs, blocks, combos, want_results=False):
    """The batched 16x16 level (``mt_rdo_level16``): blocks on the 16-sample
    grid, prm.tx_size = 16, the 256-entry 16x16 QM row and the TX_16X16 cost
    slice."""
    lib = load()
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.BLOCK8_DTYPE)
    combos = np.ascontiguousarray(combos, abi.COMBO_DTYPE)
    best = np.zeros(len(blocks), abi.BEST_DTYPE)
    res = np.zeros(len(blocks) * len(combos), RESULT_DTYPE) if want_results else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(lib.mt_rdo_level16(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                              ptr(blocks), len(blocks), ptr(combos), len(combos), ptr(best), ptr(res)),
           "mt_rdo_level16")
    return best, res


def mode_beam(src, recon, prm, blocks):
    """``proxy_mode_beam``'s ranking (``mt_mode_beam``): (scores, modes), each
    nblocks x 11 in ascending (score, mode) order; prm.tx_size is the block size."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.BLOCK8_DTYPE)
    scores = np.zeros((len(blocks), abi_beam_modes()), np.uint64)
    modes = np.zeros((len(blocks), abi_beam_modes()), np.uint8)
    _check(load().mt_mode_beam(ptr(src), ptr(recon), C.byref(prm), ptr(blocks), len(blocks), ptr(scores), ptr(modes)),
           "mt_mode_beam")
    return scores, modes


def sse_recon(src, vis_w, vis_h, pos, pred, resid, w, h, wsse_scale=0.0, bd=8):
    """``sse_recon`` decision distortion of n blocks (``mt_sse_recon``): plain SSE,
    or with wsse_scale > 0 the scaled weighted SSE; returns int64[n]."""
    src = np.ascontiguousarray(src, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    pred = np.ascontiguousarray(pred, np.int32)
    resid = None if resid is None else np.ascontiguousarray(resid, np.int32)
    out = np.zeros(len(pos), np.int64)
    _check(load().mt_sse_recon(ptr(src), src.shape[1], src.shape[0], vis_w, vis_h, bd, ptr(pos), ptr(pred),
                               ptr(resid), len(pos), w, h, wsse_scale, ptr(out)), "mt_sse_recon")
    return out


def uv_mode_cdfs_default():
    """The mode CDFs uv_mode_bits reads, from the default decision snapshot."""
    c = abi.UvModeCdfs()
    _check(load().mt_uv_mode_cdfs_default(C.byref(c)), "mt_uv_mode_cdfs_default")
    return c


def uv_mode_costs(cdfs):
    out = abi.UvModeCosts()
    _check(load().mt_uv_mode_costs_build(C.byref(cdfs), C.byref(out)), "mt_uv_mode_costs_build")
    return out


def uv_mode_bits(costs, y_mode, uv_mode, cfl=None):
    """uv_mode_bits(y_mode, uv_mode, cfl) on the host; cfl: (alpha_u, alpha_v) or None."""
    au, av = cfl if cfl is not None else (0, 0)
    return load().mt_uv_mode_bits(C.byref(costs), y_mode, uv_mode, int(cfl is not None), au, av)


def uv16_params(luma_stride, joint_k=4, angle_deltas=True, dir_lambda=0.0):
    """``mt_uv16_params``: dir_lambda is the 4:4:4 search's directional-stage lambda."""
    u = abi.Uv16Params()
    u.luma_stride, u.joint_k, u.angle_deltas, u.dir_lambda = luma_stride, joint_k, int(bool(angle_deltas)), dir_lambda
    return u


def _pick_uv16(entry, dtype, per_job, src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant, qmrow, costs, mode_costs,
               jobs, want_cf, want_rec):
    planes = [np.ascontiguousarray(a, np.uint16) for a in (src_u, src_v, rec_u, rec_v, luma)]
    jobs = np.ascontiguousarray(jobs, dtype)
    n = len(jobs)
    res = np.zeros(n, abi.UV16_RESULT_DTYPE)
    cf = np.zeros((n, per_job), np.int32) if want_cf else None
    rec = np.zeros((n, per_job), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(getattr(load(), entry)(*[ptr(a) for a in planes], C.byref(prm), C.byref(uvp), C.byref(quant), ptr(qm),
                                  C.byref(costs), C.byref(mode_costs), ptr(jobs), n, ptr(res), ptr(cf), ptr(rec)),
           entry)
    return res, cf, rec


def pick_uv16_420(src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant, qmrow, costs, mode_costs, jobs, want_cf=False,
                  want_rec=False):
    """pick_uv16_420 over (16x16 leaf) jobs (``mt_pick_uv16_420``): (results,
    levels n x 128 or None, reconstruction n x 128 or None), U then V."""
    return _pick_uv16("mt_pick_uv16_420", abi.UV16_JOB_DTYPE, 128, src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant,
                      qmrow, costs, mode_costs, jobs, want_cf, want_rec)


def pick_uv32_420(src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant, qmrow, costs, mode_costs, jobs, want_cf=False,
                  want_rec=False):
    """pick_uv32_420 over (32x32 leaf) jobs (``mt_pick_uv32_420``, mt_uv16_444_job layout): (results,
    levels n x 512 or None, reconstruction n x 512 or None), U then V."""
    return _pick_uv16("mt_pick_uv32_420", abi.UV16_444_JOB_DTYPE, 512, src_u, src_v, rec_u, rec_v, luma, prm, uvp,
                      quant, qmrow, costs, mode_costs, jobs, want_cf, want_rec)


def pick_uv32_444(src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant, qmrow, costs, mode_costs, jobs, want_cf=False,
                  want_rec=False):
    """pick_uv32_444 over (32x32 leaf) jobs (``mt_pick_uv32_444``): (results,
    levels n x 2048 or None, reconstruction n x 2048 or None), U then V."""
    return _pick_uv16("mt_pick_uv32_444", abi.UV32_444_JOB_DTYPE, 2048, src_u, src_v, rec_u, rec_v, luma, prm, uvp,
                      quant, qmrow, costs, mode_costs, jobs, want_cf, want_rec)


def pick_uv16_444(src_u, src_v, rec_u, rec_v, luma, prm, uvp, quant, qmrow, costs, mode_costs, jobs, want_cf=False,
                  want_rec=False):
    """pick_uv16_444 over (16x16 leaf) jobs (``mt_pick_uv16_444``): (results,
    levels n x 512 or None, reconstruction n x 512 or None), U then V."""
    return _pick_uv16("mt_pick_uv16_444", abi.UV16_444_JOB_DTYPE, 512, src_u, src_v, rec_u, rec_v, luma, prm, uvp,
                      quant, qmrow, costs, mode_costs, jobs, want_cf, want_rec)


def split16_params(frame_w, frame_h, stride=None, trellis_lambda0=0.05, rd_lambda=1.0, band_tilt=0.0,
                   wsse_scale=0.0, tx_search=False, tx_guard_shift=4, skip_bits=None, vis=None, bd=8):
    """``mt_split16_params``: skip_bits, when given, is 13 (all_zero = 1, all_zero = 0)
    pairs of the TX_8X8 class (the reference's skip_price rows)."""
    p = abi.Split16Params()
    p.frame_w, p.frame_h, p.bd = frame_w, frame_h, bd
    p.stride = stride if stride is not None else frame_w
    if vis is not None:
        p.vis_w, p.vis_h = vis
    p.trellis_lambda0, p.rd_lambda, p.band_tilt, p.wsse_scale = trellis_lambda0, rd_lambda, band_tilt, wsse_scale
    p.tx_search, p.tx_guard_shift = int(bool(tx_search)), tx_guard_shift
    if skip_bits is not None:
        p.use_skip_bits = 1
        for k, (one, zero) in enumerate(skip_bits):
            p.skip_bits[k][0], p.skip_bits[k][1] = one, zero
    return p


def split16_luma(src, recon, prm, quant, qmrow, costs, jobs, want_cf=False, want_rec=False):
    """``split16_luma_try`` of a batch of (16x16 block, mode) jobs (``mt_split16_luma``):
    returns (results, cf n x 256 or None, rec n x 16 x 16 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32) if want_cf else None
    rec = np.zeros((n, 16, 16), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_split16_luma(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                                  ptr(jobs), n, ptr(res), ptr(cf), ptr(rec)), "mt_split16_luma")
    return res, cf, rec


def split16_depth2(src, recon, prm, quant, qmrow, costs, jobs, want_cf=False, want_rec=False):
    """``split16_depth2_try`` of a batch of jobs (``mt_split16_depth2``): sixteen TX_4X4
    per job; qmrow / costs are the 4x4 row and the TX_4X4 slice.  Returns (results,
    cf n x 256 or None, rec n x 16 x 16 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_D2_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32) if want_cf else None
    rec = np.zeros((n, 16, 16), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_split16_depth2(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                                    ptr(jobs), n, ptr(res), ptr(cf), ptr(rec)), "mt_split16_depth2")
    return res, cf, rec


def filter_intra_beam(src, recon, w, h, pos, vis=(0, 0), bd=8, want_preds=False):
    """The filter-intra shortlist ranking (``mt_filter_intra_beam``): (scores, modes),
    each n x 5 ascending, and the five predictions n x 5 x h x w or None."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    scores = np.zeros((n, 5), np.uint64)
    modes = np.zeros((n, 5), np.uint8)
    preds = np.zeros((n, 5, h, w), np.int16) if want_preds else None
    _check(load().mt_filter_intra_beam(ptr(src), ptr(recon), src.shape[1], src.shape[1], src.shape[0], vis[0], vis[1],
                                       bd, w, h, ptr(pos), n, ptr(scores), ptr(modes), ptr(preds)),
           "mt_filter_intra_beam")
    return scores, modes, preds


def cfl_alpha(luma, src_u, src_v, sub_x, sub_y, cw, ch, blocks, vis=(0, 0), bd=8, want_ac=False):
    """Chroma-from-luma alpha of n chroma blocks (``mt_cfl_alpha``): returns
    (alpha n x 2 int8 for U and V, the AC n x ch x cw or None)."""
    luma = np.ascontiguousarray(luma, np.uint16)
    src_u = np.ascontiguousarray(src_u, np.uint16)
    src_v = np.ascontiguousarray(src_v, np.uint16)
    blocks = np.ascontiguousarray(blocks, abi.CFL_BLOCK_DTYPE)
    n = len(blocks)
    alpha = np.zeros((n, 2), np.int8)
    ac = np.zeros((n, ch, cw), np.int32) if want_ac else None
    _check(load().mt_cfl_alpha(ptr(luma), luma.shape[1], luma.shape[0], ptr(src_u), ptr(src_v), src_u.shape[1],
                               src_u.shape[0], sub_x, sub_y, cw, ch, vis[0], vis[1], bd, ptr(blocks), n, ptr(alpha),
                               ptr(ac)), "mt_cfl_alpha")
    return alpha, ac


def palette_opts(smooth_t=0, smooth_guard=True, viterbi_lambda=0.0, color_costs=None):
    """``mt_palette_opts``: palette_smooth tolerance, its guard, the Viterbi lambda
    (0 = nearest + smoothing) and the palette_y_color bits [size - 2][ctx][symbol]."""
    o = abi.PaletteOpts()
    o.smooth_t, o.smooth_guard, o.viterbi_lambda = int(smooth_t), int(bool(smooth_guard)), float(viterbi_lambda)
    if color_costs is not None:
        cc = np.ascontiguousarray(color_costs, np.float32).reshape(7, 5, 8)
        C.memmove(C.addressof(o.color_costs), cc.ctypes.data, cc.nbytes)
    return o


def luma_palette(src, w, h, pos, opts, bd=8, want_maps=False):
    """The lossy luma palette candidates of n w x h blocks (``mt_luma_palette``):
    returns (candidates n x 14, maps n x 14 x h x w or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    cands = np.zeros((n, abi.PALETTE_SLOTS), abi.PALETTE_CAND_DTYPE)
    maps = np.zeros((n, abi.PALETTE_SLOTS, h, w), np.uint8) if want_maps else None
    _check(load().mt_luma_palette(ptr(src), src.shape[1], src.shape[1], src.shape[0], bd, w, h, ptr(pos), n,
                                  C.byref(opts), ptr(cands), ptr(maps)), "mt_luma_palette")
    return cands, maps


def uv_palette(src_u, src_v, w, h, pos, opts, want_maps=False):
    """The UV palette candidates of n w x h chroma blocks (``mt_uv_palette``):
    exact_uv_palette in slot 0, or the four lossy_uv_palette_from_hist
    candidates (8 / 4 colours by k-means, 8 / 4 dominant pairs); ``opts`` carries
    the Viterbi lambda and the palette_uv_color bits.  Returns (candidates n x 4,
    maps n x 4 x h x w or None)."""
    src_u = np.ascontiguousarray(src_u, np.uint16)
    src_v = np.ascontiguousarray(src_v, np.uint16)
    if src_u.shape != src_v.shape:
        raise ValueError("U and V planes differ in shape")
    pos = np.ascontiguousarray(pos, np.uint16).reshape(-1, 2)
    n = len(pos)
    cands = np.zeros((n, abi.UV_PALETTE_SLOTS), abi.UV_PALETTE_CAND_DTYPE)
    maps = np.zeros((n, abi.UV_PALETTE_SLOTS, h, w), np.uint8) if want_maps else None
    _check(load().mt_uv_palette(ptr(src_u), ptr(src_v), src_u.shape[1], src_u.shape[0], w, h, ptr(pos), n,
                                C.byref(opts), ptr(cands), ptr(maps)), "mt_uv_palette")
    return cands, maps


def split4tx(src, recon, prm, quant, qmrow, costs, jobs, want_cf=False, want_rec=False):
    """The 8x8 leaf's ``split4tx_try`` (``mt_split4tx``): four TX_4X4 per 8x8 job;
    returns (results, cf n x 64 or None, rec n x 8 x 8 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.SPLIT16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.SPLIT16_RESULT_DTYPE)
    cf = np.zeros((n, 64), np.int32) if want_cf else None
    rec = np.zeros((n, 8, 8), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_split4tx(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs), ptr(jobs),
                              n, ptr(res), ptr(cf), ptr(rec)), "mt_split4tx")
    return res, cf, rec


def leaf8(src, recon, prm, quant, qmrow, costs, jobs, refine=False, want_cf=False, want_rec=False):
    """The 8x8 leaf's luma search (``mt_leaf8``): the mode loop's candidates, or with
    refine the winners' transform-type refinement.  Returns (results, cf n x 64 or
    None, rec n x 8 x 8 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 64), np.int32) if want_cf else None
    rec = np.zeros((n, 8, 8), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_leaf8(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs), ptr(jobs), n,
                           int(bool(refine)), ptr(res), ptr(cf), ptr(rec)), "mt_leaf8")
    return res, cf, rec


def leaf16(src, recon, prm, quant, qmrow, costs, jobs, refine=False, want_cf=False, want_rec=False):
    """The 16x16 leaf's mode-loop candidates, or with refine the winners' transform-type
    refinement (``mt_leaf16``); qmrow / costs are the 16x16 row and the TX_16X16
    slice.  Returns (results, cf n x 256 or None, rec n x 16 x 16 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 256), np.int32) if want_cf else None
    rec = np.zeros((n, 16, 16), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_leaf16(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs), ptr(jobs),
                            n, int(bool(refine)), ptr(res), ptr(cf), ptr(rec)), "mt_leaf16")
    return res, cf, rec


def leaf32(src, recon, prm, quant, qmrow, costs, jobs, want_cf=False, want_rec=False):
    """The 32x32 leaf's mode-loop candidates (``mt_leaf32``); qmrow / costs are the
    32x32 row and the TX_32X32 slice.  Returns (results, cf n x 1024 or None,
    rec n x 32 x 32 or None)."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.LEAF8_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.LEAF8_RESULT_DTYPE)
    cf = np.zeros((n, 1024), np.int32) if want_cf else None
    rec = np.zeros((n, 32, 32), np.uint16) if want_rec else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_leaf32(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs), ptr(jobs),
                            n, ptr(res), ptr(cf), ptr(rec)), "mt_leaf32")
    return res, cf, rec


def quad32_luma(src, recon, prm, quant, qmrow, costs, jobs):
    """The 64x64 leaf's four-TX_32X32 leg (``mt_quad32_luma``); qmrow / costs are
    the 32x32 row and the TX_32X32 slice.  Returns the results."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.QUAD32_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.QUAD32_RESULT_DTYPE)
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_quad32_luma(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                                 ptr(jobs), n, ptr(res)), "mt_quad32_luma")
    return res


def grid16_luma(src, recon, prm, quant, qmrow, costs, jobs, want_cf=False):
    """The 64x64 leaf's sixteen-TX_16X16 leg (``mt_grid16_luma``); qmrow / costs
    are the 16x16 row and the TX_16X16 slice.  Returns (results, levels or None),
    levels n x 4096 with transform t at t * 256."""
    src = np.ascontiguousarray(src, np.uint16)
    recon = np.ascontiguousarray(recon, np.uint16)
    jobs = np.ascontiguousarray(jobs, abi.GRID16_JOB_DTYPE)
    n = len(jobs)
    res = np.zeros(n, abi.GRID16_RESULT_DTYPE)
    cf = np.zeros((n, 4096), np.int32) if want_cf else None
    qm = None if qmrow is None else np.ascontiguousarray(qmrow, np.uint8)
    _check(load().mt_grid16_luma(ptr(src), ptr(recon), C.byref(prm), C.byref(quant), ptr(qm), C.byref(costs),
                                 ptr(jobs), n, ptr(res), ptr(cf)), "mt_grid16_luma")
    return res, cf


def split16_luma_device(d_src, d_recon, prm, quant, d_qm, d_costs, d_jobs, n, d_results, d_cf=None, d_rec=None,
                        stream=0):
    _check(load().mt_split16_luma_device(ptr(d_src), ptr(d_recon), C.byref(prm), C.byref(quant), ptr(d_qm),
                                         ptr(d_costs), ptr(d_jobs), n, ptr(d_results), ptr(d_cf), ptr(d_rec),
                                         stream), "mt_split16_luma_device")


def trellis_optimize_ctx_device(d_levels, d_targets, d_dcs, n, quant, d_qm, d_costs, lambda0, band_tilt=0.0, stream=0):
    """``trellis_optimize_ctx`` of n TX_8X8 luma blocks in place (``mt_trellis_optimize_ctx_device``)."""
    _check(load().mt_trellis_optimize_ctx_device(ptr(d_levels), ptr(d_targets), ptr(d_dcs), n, C.byref(quant),
                                                 ptr(d_qm), ptr(d_costs), lambda0, band_tilt, stream),
           "mt_trellis_optimize_ctx_device")


def abi_beam_modes():
    return 11


def rdo_level8_scratch_bytes(nblocks, ncombos):
    """Device working storage ``mt_rdo_level8_device`` needs."""
    return load().mt_rdo_level8_scratch_bytes(nblocks, ncombos)


def rdo_level8_device(d_src, d_recon, prm, quant, d_qm, d_costs, d_blocks, nblocks, d_combos, ncombos, d_best,
                      d_results, d_scratch, stream=0):
    _check(load().mt_rdo_level8_device(ptr(d_src), ptr(d_recon), C.byref(prm), C.byref(quant), ptr(d_qm),
                                       ptr(d_costs), ptr(d_blocks), nblocks, ptr(d_combos), ncombos, ptr(d_best),
                                       ptr(d_results), ptr(d_scratch), stream or None), "mt_rdo_level8_device")


def padded_plane_dims(w, h, sub):
    v = [C.c_int32() for _ in range(4)]
    _check(load().mt_padded_plane_dims(w, h, sub, *[C.byref(x) for x in v]), "mt_padded_plane_dims")
    return tuple(x.value for x in v)


def csc_rgb8(rgb, sub):
    """Interleaved u8 RGB (h, w, 3) -> padded (Y, Cb, Cr) u16 planes; sub 0 = 4:4:4, 2 = 4:2:0."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w = rgb.shape[:2]
    pw, ph, pcw, pch = padded_plane_dims(w, h, sub)
    y = np.zeros((ph, pw), np.uint16)
    cb = np.zeros((pch, pcw), np.uint16)
    cr = np.zeros((pch, pcw), np.uint16)
    _check(load().mt_csc_rgb8(ptr(rgb), w, h, sub, ptr(y), ptr(cb), ptr(cr)), "mt_csc_rgb8")
    return y, cb, cr


def _u8_map(m, nr4, nc4):
    if m is None:
        return None
    m = np.asarray(m)
    if m.ndim != 2 or m.shape[0] < nr4 or m.shape[1] != nc4:
        raise ValueError(f"block map shape {m.shape}: need at least {nr4} rows of {nc4} cells")
    return np.ascontiguousarray(m[:nr4], np.uint8)


def deblock_plane(px, vis_w, vis_h, bw4, bh4, level, sharp, is_luma, vedge4=None, hedge4=None, bd=8):
    """``filter_plane`` (src/loopfilter.rs:482-648) on a copy of ``px``.

    px: (h, w) u16 padded plane; bw4 / bh4: (>= ceil(vis_h/4), nc4) u8 block
    width / height maps in 4-sample units; vedge4 / hedge4: optional block
    start flags (None = alignment rule).  Returns the filtered plane."""
    out = np.array(px, dtype=np.uint16, copy=True, order="C")
    h, w = out.shape
    nr4 = (vis_h + 3) // 4
    nc4 = np.asarray(bw4).shape[-1]
    bw4 = _u8_map(bw4, nr4, nc4)
    bh4 = _u8_map(bh4, nr4, nc4)
    ve = _u8_map(vedge4, nr4, nc4)
    he = _u8_map(hedge4, nr4, nc4)
    _check(load().mt_deblock_plane(ptr(out), w, h, vis_w, vis_h, ptr(bw4), ptr(bh4), ptr(ve), ptr(he), nc4, level,
                                   sharp, int(bool(is_luma)), bd), "mt_deblock_plane")
    return out


def cdef_params(disp_w, disp_h, sub_x, sub_y, base_q_idx, mono=False, slow=True, bd=8):
    """``mt_cdef_params`` of a frame whose padded planes are align8(disp)."""
    p = abi.CdefParams()
    p.w8, p.h8 = (disp_w + 7) & ~7, (disp_h + 7) & ~7
    p.disp_w, p.disp_h, p.sub_x, p.sub_y = disp_w, disp_h, sub_x, sub_y
    p.mono, p.base_q_idx, p.bd, p.slow = int(mono), base_q_idx, bd, int(slow)
    return p


def _decision_dict(d, grid):
    n = d.n_strengths
    return {"bits": d.bits, "damping": d.damping, "unit_cols": d.unit_cols, "unit_rows": d.unit_rows,
            "strengths": [tuple(d.strengths[e]) for e in range(n)], "grid": grid}


def cdef_frame(recon, src, skip8, prm):
    """``frame_cdef`` (src/coder/frame_cdef.rs:49-520) on copies of the recon
    planes.  recon / src: [Y] or [Y, U, V] u16 planes; skip8: (h8/8, w8/8) u8.
    Returns (filtered planes, decision dict)."""
    mono = bool(prm.mono)
    out = [np.array(p, dtype=np.uint16, copy=True, order="C") for p in recon]
    src = [np.ascontiguousarray(p, np.uint16) for p in src]
    skip8 = np.ascontiguousarray(skip8, np.uint8)
    nu = ((prm.w8 + 63) // 64) * ((prm.h8 + 63) // 64)
    grid = np.zeros(nu, np.uint8)
    d = abi.CdefDecision()
    ch = (lambda a, i: None) if mono else (lambda a, i: ptr(a[i]))
    _check(load().mt_cdef_frame(ptr(out[0]), ch(out, 1), ch(out, 2), ptr(src[0]), ch(src, 1), ch(src, 2), ptr(skip8),
                                C.byref(prm), C.byref(d), ptr(grid)), "mt_cdef_frame")
    return out, _decision_dict(d, grid)


def tiling_spec_min(w8, h8):
    """``plan_tiling(sb_cols, sb_rows, 1)`` (src/coder/tiling.rs:92-136): (cols_log2, rows_log2)."""
    a, b = C.c_int32(), C.c_int32()
    _check(load().mt_tiling_spec_min(w8, h8, C.byref(a), C.byref(b)), "mt_tiling_spec_min")
    return a.value, b.value


def aq_params(w8, h8, base_q_idx, bd=8, variance_boost=True, dark_aq=True, octile=6, boost_only=False,
              strength=1.0, tiling=None):
    """``mt_aq_params`` with the reference's defaults (adaptive quant, Variance
    Boost and dark protection on); tiling defaults to the spec minimum."""
    p = abi.AqParams()
    p.w8, p.h8 = w8, h8
    p.tile_cols_log2, p.tile_rows_log2 = tiling if tiling is not None else tiling_spec_min(w8, h8)
    p.base_q_idx, p.bd, p.variance_boost, p.dark_aq = base_q_idx, bd, int(variance_boost), int(dark_aq)
    p.octile, p.boost_only, p.strength = octile, int(boost_only), strength
    return p


def aq_grid(luma, prm):
    """``precompute_aq_grid`` of every tile (src/coder/lossy_state.rs:3937-3963).

    luma: (h8, w8) u16 padded source.  Returns (cells, tile_refs): cells an
    (sb_rows, sb_cols) array of ``AQ_CELL_DTYPE``, tile_refs (ntiles, 2) f32."""
    luma = np.ascontiguousarray(luma, np.uint16)
    assert luma.shape == (prm.h8, prm.w8)
    sbr, sbc = (prm.h8 + 63) // 64, (prm.w8 + 63) // 64
    cells = np.zeros((sbr, sbc), abi.AQ_CELL_DTYPE)
    tc = -(-sbc // -(-sbc // (1 << prm.tile_cols_log2)))
    tr = -(-sbr // -(-sbr // (1 << prm.tile_rows_log2)))
    refs = np.zeros((tc * tr, 2), np.float32)
    _check(load().mt_aq_grid(ptr(luma), C.byref(prm), ptr(cells), ptr(refs)), "mt_aq_grid")
    return cells, refs


def aq_grid_device(d_luma, prm, d_cells, d_tile_refs, d_scratch, stream=0):
    """Device form: torch tensors (or raw pointers) on the current device."""
    _check(load().mt_aq_grid_device(ptr(d_luma), C.byref(prm), ptr(d_cells), ptr(d_tile_refs), ptr(d_scratch),
                                    stream or None), "mt_aq_grid_device")


def aq_grid_scratch_bytes(prm):
    return load().mt_aq_grid_scratch_bytes(C.byref(prm))


def dark_pow_device(d_x, d_out, n, stream=0):
    """The dark-protection weight's power (``powf(x, 1.2f)`` of the C library on (1, 4.5])."""
    _check(load().mt_dark_pow_device(ptr(d_x), ptr(d_out), n, stream or None), "mt_dark_pow_device")


def screen_gate_params(w8, h8, sub_x, sub_y, base_q_idx, bd=8):
    p = abi.ScreenGateParams()
    p.w8, p.h8, p.sub_x, p.sub_y, p.bd, p.base_q_idx = w8, h8, sub_x, sub_y, bd, base_q_idx
    return p


def screen_gate(luma, sub_x, sub_y, base_q_idx, bd=8):
    """``screen_frame_gate`` (src/coder/screen_gate.rs:64-273) of a padded luma
    plane; returns the ``mt_screen_gate_result`` fields as a dict."""
    luma = np.ascontiguousarray(luma, np.uint16)
    prm = screen_gate_params(luma.shape[1], luma.shape[0], sub_x, sub_y, base_q_idx, bd)
    r = abi.ScreenGateResult()
    _check(load().mt_screen_gate(ptr(luma), C.byref(prm), C.byref(r)), "mt_screen_gate")
    return r.as_dict()


def loop_filter_levels(base_q_idx, sub_x, sub_y):
    """``loop_filter_levels`` / ``loop_filter_sharpness`` (src/obu.rs:306-334): (lvl_y, lvl_uv, sharp)."""
    a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
    _check(load().mt_loop_filter_levels(base_q_idx, sub_x, sub_y, C.byref(a), C.byref(b), C.byref(c)),
           "mt_loop_filter_levels")
    return a.value, b.value, c.value


def deblock_frame(planes, disp_w, disp_h, sub_x, sub_y, tx_maps, pred_maps, lvl_y, lvl_u, lvl_v, mono=False):
    """``frame_deblock`` (src/coder/frame_deblock.rs:206-224) on copies of the planes.

    tx_maps: (blk4, blk4h, blk4v, blk4t) luma transform-block maps with block
    start flags; pred_maps: (pblk4, pblk4h) luma prediction-block sizes; all
    (h8/4, w8/4) u8."""
    out = [np.array(p, dtype=np.uint16, copy=True, order="C") for p in planes]
    g = abi.DeblockFrameParams()
    g.w8, g.h8 = out[0].shape[1], out[0].shape[0]
    g.disp_w, g.disp_h, g.sub_x, g.sub_y, g.mono, g.bd = disp_w, disp_h, sub_x, sub_y, int(mono), 8
    tm = [np.ascontiguousarray(m, np.uint8) for m in tx_maps]
    pm = [np.ascontiguousarray(m, np.uint8) for m in pred_maps]
    ch = (lambda i: None) if mono else (lambda i: ptr(out[i]))
    _check(load().mt_deblock_frame(ptr(out[0]), ch(1), ch(2), *[ptr(m) for m in tm], *[ptr(m) for m in pm],
                                   C.byref(g), lvl_y, lvl_u, lvl_v), "mt_deblock_frame")
    return out
