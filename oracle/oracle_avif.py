"""Oracle encode (test infrastructure only): mt_encode_rgb8's decision rule
and everything after it, on the CPU and without the product library -- the
checker of the device encoder's bytes and the timed CPU baseline of the
encode.

  * decisions, reconstruction and levels: oracle_encode.cpp or_encode_decide
    (the candidate chain of the oracle over the 8x8 blocks, superblocks in the
    wavefront on host threads);
  * deblocking with the shipped levels and the CDEF decision: the oracle's
    frame filters;
  * block syntax, coefficient tokens and each tile's range coding with the
    cdef_idx literals: or_encode_pack;
  * headers and the AVIF container, restated here from src/bitwriter.rs,
    src/obu.rs and src/isobmff.rs for the subset the encoder writes (the
    spec-minimum uniform tiling, reduced still-picture header, lossy frame header without segmentation,
    delta-q, IntraBC or restoration; a colour item with ispe, pixi, av1C and
    an nclx colr).
"""
import ctypes as C
import os

import numpy as np

from maroontree_b200 import abi

from . import pyoracle as po

_P = C.c_void_p
_bound = False


def _lib():
    global _bound
    lib = po.load()
    if not _bound:
        lib.or_encode_decide.restype = C.c_int
        lib.or_encode_decide.argtypes = [C.c_int32] * 5 + [C.POINTER(abi.ChainParams)] * 2 + \
            [C.POINTER(abi.Quant)] * 2 + [_P, _P] + [C.POINTER(abi.CoefCdfs)] * 2 + [_P] * 11 + [C.c_int32]
        lib.or_encode_pack.restype = C.c_int
        lib.or_encode_pack.argtypes = [C.c_int32] * 5 + [_P] * 5 + [_P, C.POINTER(po.EmitSlots), _P, _P, _P,
                                                                   C.c_int32, C.c_size_t, _P, C.c_int32,
                                                                   C.c_int32, _P, C.c_size_t, _P, C.c_int32,
                                                                   C.POINTER(C.c_int32), C.POINTER(C.c_size_t)]
        _bound = True
    return lib


# ---------------------------------------------------------------------------
# Headers and container.

class _Bits:
    """BitWriter (src/bitwriter.rs:31-100): f(n) most significant bit first."""

    def __init__(self):
        self.out, self.cur, self.n = bytearray(), 0, 0

    def f(self, v, n):
        for i in range(n - 1, -1, -1):
            self.cur = (self.cur << 1) | ((v >> i) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.cur)
                self.cur, self.n = 0, 0

    def flag(self, b):
        self.f(1 if b else 0, 1)

    def trailing(self):
        self.f(1, 1)
        self.align()

    def align(self):
        if self.n:
            self.out.append((self.cur << (8 - self.n)) & 0xFF)
            self.cur, self.n = 0, 0

    def bytes(self):
        self.align()
        return bytes(self.out)


def leb128(v):
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        out.append(b | (0x80 if v else 0))
        if not v:
            return bytes(out)


def obu(obu_type, payload):
    """wrap_obu (src/obu.rs:46-58): header with obu_has_size_field, leb128 size."""
    return bytes([(obu_type & 0xF) << 3 | 0x02]) + leb128(len(payload)) + payload


def _bits_for(v):
    """src/obu.rs:64-70."""
    b = 1
    while (1 << b) <= max(v - 1, 0):
        b += 1
    return b


def sequence_header(w, h, profile, ss, cicp):
    """seq_header_ss (src/obu.rs:630-727) for 8-bit colour: reduced still
    picture, CDEF and restoration enabled, filter intra and intra edge filter
    enabled.  cicp = (primaries, transfer, matrix, full_range, csp)."""
    b = _Bits()
    b.f(profile, 3)
    b.flag(True)
    b.flag(True)
    b.f(0, 5)
    wb, hb = _bits_for(w), _bits_for(h)
    b.f(wb - 1, 4)
    b.f(hb - 1, 4)
    b.f(w - 1, wb)
    b.f(h - 1, hb)
    for v in (False, True, True, False, True, True):  # 128x128 SB, filter intra, edge filter, superres, cdef, lr
        b.flag(v)
    b.flag(False)  # high_bitdepth
    if profile != 1:
        b.flag(False)  # mono_chrome
    prim, tran, mat, full, csp = cicp
    b.flag(True)
    b.f(prim, 8)
    b.f(tran, 8)
    b.f(mat, 8)
    if mat != 0:  # MC_IDENTITY codes neither range nor subsampling
        b.flag(bool(full))
        if ss:
            b.f(csp, 2)
    b.flag(False)  # separate_uv_delta_q
    b.flag(False)  # film_grain_params_present
    b.trailing()
    return obu(1, b.bytes())


def _tile_log2(blk, target):
    k = 0
    while (blk << k) < target:
        k += 1
    return k


def _increments(lo, hi, target):
    """increment_bits (src/coder/tiling.rs:78-95)."""
    v, cur = [], lo
    while cur < hi:
        if cur < target:
            v.append(True)
            cur += 1
        else:
            v.append(False)
            break
    return v


def tiling(w8, h8):
    """plan_tiling(sb_cols, sb_rows, 1) (src/coder/tiling.rs:92-136): the
    spec-minimum (TileColsLog2, TileRowsLog2) with the increment bits that
    signal them, and the uniform tile size in superblocks
    (tile_starts_sb, :140-152)."""
    sbc, sbr = (w8 + 63) // 64, (h8 + 63) // 64
    min_c, max_c = _tile_log2(64, sbc), _tile_log2(1, min(sbc, 64))
    max_r = _tile_log2(1, min(sbr, 64))
    min_t = max(min_c, _tile_log2(2304, sbr * sbc))
    tcl = min(min_c, max_c)
    trl = min(max(min_t - tcl, 0), max_r)
    incr = _increments(min_c, max_c, tcl) + _increments(max(min_t - tcl, 0), max_r, trl)
    return tcl, trl, incr, -(-sbc // (1 << tcl)), -(-sbr // (1 << trl))


def frame_header(w8, h8, q, qm, lf, sharp, cdef, updating_cdf=True):
    """frame_header_lossy_impl (src/obu.rs:396-527) in the spec-minimum tiling,
    no delta-q or IntraBC, the luma DC delta of -8 (src/quant.rs:350-352), no
    chroma deltas; cdef = (damping, bits, strengths) or None (the no-op
    parameters); restoration off.  For one tile: byte aligned without trailing
    bits (the header of an OBU_FRAME); for several: with trailing bits (an
    OBU_FRAME_HEADER)."""
    b = _Bits()
    b.flag(not updating_cdf)
    b.flag(True)   # allow_screen_content_tools
    b.flag(True)   # force_integer_mv
    b.flag(False)  # render_and_frame_size_different
    b.flag(False)  # allow_intrabc
    b.flag(True)   # uniform_tile_spacing_flag
    tcl, trl, incr, _, _ = tiling(w8, h8)
    for v in incr:
        b.flag(v)
    if tcl + trl > 0:
        b.f(0, tcl + trl)  # context_update_tile_id
        b.f(3, 2)          # tile_size_bytes_minus_1: TileSizeBytes 4
    b.f(q, 8)
    b.flag(True)
    b.f(-8 & 0x7F, 7)  # DeltaQYDc
    b.flag(False)      # DeltaQUDc
    b.flag(False)      # DeltaQUAc
    qy, quv = qm
    use_qm = qy < 15 or quv < 15
    b.flag(use_qm)
    if use_qm:
        b.f(qy, 4)
        b.f(quv, 4)
    b.flag(False)  # segmentation_enabled
    b.flag(False)  # delta_q_present
    ly, luv = lf
    b.f(ly, 6)
    b.f(ly, 6)
    if ly:
        b.f(luv, 6)
        b.f(luv, 6)
    b.f(sharp, 3)
    b.flag(False)  # loop_filter_delta_enabled
    damping, bits, strengths = cdef if cdef is not None else (3, 0, [(0, 0, 0, 0)])
    b.f(damping - 3, 2)  # write_cdef_params (src/obu.rs:343-365)
    b.f(bits, 2)
    for i in range(1 << bits):
        yp, ys, up, us = strengths[i] if i < len(strengths) else (0, 0, 0, 0)
        b.f(yp, 4)
        b.f(3 if ys == 4 else ys, 2)
        b.f(up, 4)
        b.f(3 if us == 4 else us, 2)
    for _ in range(3):  # write_lr_params (src/obu.rs:373-394): RESTORE_NONE on every plane
        b.f(0, 2)
    b.flag(True)   # tx_mode_select
    b.flag(False)  # reduced_tx_set
    if tcl + trl > 0:
        b.trailing()
    return b.bytes()


def frame_obus(fh, tiles):
    """assemble_frame_obus (src/coder/frame_encode.rs:444-525): one tile as an
    OBU_FRAME; several as an OBU_FRAME_HEADER and an OBU_TILE_GROUP whose
    tiles but the last carry their size less one in 4 little-endian bytes
    (src/obu.rs:296-300).  fh is frame_header()'s output for the tiling."""
    if len(tiles) == 1:
        return obu(6, fh + tiles[0])
    tg = b"\0" + b"".join((len(t) - 1).to_bytes(4, "little") + t for t in tiles[:-1]) + tiles[-1]
    return obu(3, fh) + obu(4, tg)


def level_for(w, h):
    """src/isobmff.rs:162-176."""
    px = w * h
    for lim, lvl in ((147456, 0), (278784, 1), (737280, 4), (2228224, 8), (8912896, 12), (35651584, 16)):
        if px <= lim:
            return lvl
    return 19


def _box(kind, payload):
    return (8 + len(payload)).to_bytes(4, "big") + kind + payload


def _fullbox(kind, ver, flags, payload):
    return _box(kind, bytes([ver]) + flags.to_bytes(3, "big") + payload)


def wrap_av1_image(av1, w, h, profile, ss, cicp):
    """wrap_av1_image (src/isobmff.rs:210-494) for a 3-channel 8-bit item with an
    nclx colr and no ICC, EXIF, rotation, mirror or light level; av1C without
    configOBUs (src/avif.rs:698-706)."""
    u32 = lambda v: v.to_bytes(4, "big")
    u16 = lambda v: v.to_bytes(2, "big")
    ftyp = _box(b"ftyp", b"avif" + u32(0) + b"avif" + b"mif1" + b"miaf")
    hdlr = _fullbox(b"hdlr", 0, 0, u32(0) + b"pict" + u32(0) * 3 + b"\0")
    pitm = _fullbox(b"pitm", 0, 0, u16(1))

    def iloc(off):
        return _fullbox(b"iloc", 0, 0, bytes([0x44, 0x00]) + u16(1) + u16(1) + u16(0) + u16(1) + u32(off) +
                        u32(len(av1)))

    iinf = _fullbox(b"iinf", 0, 0, u16(1) + _fullbox(b"infe", 2, 0, u16(1) + u16(0) + b"av01" + b"\0"))
    prim, tran, mat, full, _ = cicp
    av1c = bytes([0x81, ((profile & 7) << 5) | (level_for(w, h) & 0x1F), 0x0C if ss else 0x00, 0])
    colr = b"nclx" + u16(prim) + u16(tran) + u16(mat) + bytes([0x80 if full else 0])
    ipco = _box(b"ipco", _fullbox(b"ispe", 0, 0, u32(w) + u32(h)) + _fullbox(b"pixi", 0, 0, bytes([3, 8, 8, 8])) +
                _box(b"av1C", av1c) + _box(b"colr", colr))
    ipma = _fullbox(b"ipma", 0, 0, u32(1) + u16(1) + bytes([4, 1, 2, 0x80 | 3, 4]))
    iprp = _box(b"iprp", ipco + ipma)

    def meta(off):
        return _fullbox(b"meta", 0, 0, hdlr + pitm + iloc(off) + iinf + iprp)

    off = len(ftyp) + len(meta(0)) + 8  # the item's first byte inside mdat
    return ftyp + meta(off) + _box(b"mdat", av1)


# ---------------------------------------------------------------------------
# The encode.

SRGB_YCBCR = (1, 13, 6, 1, 0)  # Cicp::srgb_ycbcr (src/color.rs:251-259): BT.709, sRGB, BT.601, full range


def _planes_from(y, u, v):
    return [np.ascontiguousarray(x, np.uint16) for x in (y, u, v)]


def encode(planes, w, h, sub, quality, threads=None, cicp=SRGB_YCBCR, want_recon=False):
    """The encode of padded 8-bit planes (luma pw x ph; chroma halved in 4:2:0)
    displayed at w x h.  Returns the AVIF bytes (and the decoder's output
    planes: deblocked and CDEF-filtered)."""
    lib = _lib()
    threads = threads or os.cpu_count() or 1
    src = _planes_from(*planes)
    ph, pw = src[0].shape
    pch, pcw = src[1].shape
    sx = 1 if sub else 0
    q = po.quality_to_q(quality)
    qm_y, qm_uv = po.qm_level_law(q, sub), po.qm_chroma_level_law(q, sub)
    nc = 4 if sub else 8
    qy, qc = po.quant_new(q, 8, qm_y), po.quant_new_chroma(q, 0, 0, 8, qm_uv)
    qmy, qmc = po.qm_row(qm_y, 0, 8), po.qm_row(qm_uv, 1, nc)
    lam = po.rd_lambdas(q, qy.dc_q, sub)
    qctx = po.qcat(q)
    cdy, cdc = po.default_cdfs(qctx, 8, 8, 0), po.default_cdfs(qctx, nc, nc, 1)
    py = abi.ChainParams()
    py.tx_size, py.bd, py.frame_w, py.frame_h, py.stride = 8, 8, pw, ph, pw
    py.trellis_lambda0, py.mode_lambda = lam.trellis_lambda0, lam.mode_lambda
    py.satd_scale, py.satd_bridge = lam.satd_scale, lam.satd_bridge
    pc = abi.ChainParams.from_buffer_copy(py)
    pc.tx_size, pc.frame_w, pc.frame_h, pc.stride = nc, pcw, pch, pcw
    nbx, nby = pw // 8, ph // 8
    nb = nbx * nby
    rec = [np.zeros_like(s) for s in src]
    mode, tx = np.zeros(nb, np.uint8), np.zeros(nb, np.uint8)
    lv = [np.zeros(nb * 64, np.int32), np.zeros(nb * nc * nc, np.int32), np.zeros(nb * nc * nc, np.int32)]
    p = po.p
    _, _, _, tsw, tsh = tiling(pw, ph)
    rc = lib.or_encode_decide(pw, ph, sub, tsw, tsh, C.byref(py), C.byref(pc), C.byref(qy), C.byref(qc), p(qmy), p(qmc),
                              C.byref(cdy), C.byref(cdc), *[p(x) for x in src], *[p(x) for x in rec], p(mode),
                              p(tx), *[p(x) for x in lv], threads)
    assert rc == 0, rc
    # deblocking over the uniform 8x8 blocks and transforms, then the CDEF decision
    ly, luv, sharp = po.loop_filter_levels(q, 2 * sx)
    n4r, n4c = ph // 4, pw // 4
    col = np.tile((np.arange(n4c) % 2 == 0).astype(np.uint8), (n4r, 1))
    row = np.tile((np.arange(n4r) % 2 == 0).astype(np.uint8)[:, None], (1, n4c))
    two = np.full((n4r, n4c), 2, np.uint8)
    flt = po.deblock_frame(rec, w, h, sx, sx, [two, two, col, row], [two, two], ly, luv, luv)
    prm = abi.CdefParams()
    prm.w8, prm.h8, prm.disp_w, prm.disp_h, prm.sub_x, prm.sub_y = pw, ph, w, h, sx, sx
    prm.mono, prm.base_q_idx, prm.bd, prm.slow = 0, q, 8, 1
    flt, dec, _ = po.cdef_frame(flt, src, np.zeros(nb, np.uint8), prm)
    # the tile
    sec = {}
    slots = po.cdfs_new_slots(qctx, sec)
    lens = np.array([len(s) for s in slots], np.uint16)
    offs = np.zeros(len(slots), np.uint32)
    offs[1:] = np.cumsum(lens[:-1])
    data = np.concatenate(slots).astype(np.uint16)
    order = ("skip", "part_bl8", "part_split", "kf_y", "uv_mode", "angle_delta", "filter_intra", "palette_y_mode",
             "palette_uv_mode", "txsz")
    syn = np.array([sec[k] for k in order], np.int32)
    es, _ = po.emit_slots(qctx)
    bits = dec["bits"] if dec["bits"] > 0 else 0
    grid = np.ascontiguousarray(dec["grid"], np.uint8)
    cap = nb * 1024 + 4096
    out = np.zeros(cap, np.uint8)
    n, nt = C.c_size_t(), C.c_int32()
    tl = np.zeros(4096, np.uint64)
    rc = lib.or_encode_pack(pw, ph, sub, tsw, tsh, p(mode), p(tx), *[p(x) for x in lv], p(syn), C.byref(es), p(data),
                            p(offs), p(lens), len(slots), len(data), p(grid), bits, 1, p(out), cap, p(tl), len(tl),
                            C.byref(nt), C.byref(n))
    assert rc == 0, rc
    tiles, at = [], 0
    for t in range(nt.value):
        tiles.append(out[at:at + int(tl[t])].tobytes())
        at += int(tl[t])
    cdef = (dec["damping"], dec["bits"], dec["strengths"]) if dec["bits"] >= 0 else None
    fh = frame_header(pw, ph, q, (qm_y, qm_uv), (ly, luv), sharp, cdef)
    profile = 0 if sub else 1
    av1 = obu(2, b"") + sequence_header(w, h, profile, bool(sub), cicp) + frame_obus(fh, tiles)
    avif = wrap_av1_image(av1, w, h, profile, bool(sub), cicp)
    return (avif, flt) if want_recon else avif


def encode_rgb8(rgb, quality=80, chroma=2, threads=None, want_recon=False):
    """encode_rgb8 with EncodeConfig's defaults and the given quality and
    chroma format (abi's MT_CHROMA_420 = 0, MT_CHROMA_444 = 2): the Q13 colour
    conversion and padding of the oracle, then encode()."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w = rgb.shape[:2]
    sub = 2 if chroma == 0 else 0
    return encode(po.csc_rgb8(rgb, sub), w, h, sub, quality, threads, SRGB_YCBCR, want_recon)


def encode_yuv8(y, u, v, quality, chroma, cicp, threads=None, want_recon=False):
    """The encode of three 8-bit planes at their displayed sizes (edge samples
    replicated to x8), coded as given."""
    h, w = y.shape
    sub = 2 if chroma == 0 else 0
    pw, ph = (w + 7) & ~7, (h + 7) & ~7

    def pad(x, ww, hh):
        x = np.asarray(x, np.uint16)
        return np.pad(x, ((0, hh - x.shape[0]), (0, ww - x.shape[1])), mode="edge")

    cw, ch = (pw // 2, ph // 2) if sub else (pw, ph)
    return encode([pad(y, pw, ph), pad(u, cw, ch), pad(v, cw, ch)], w, h, sub, quality, threads, cicp, want_recon)
