"""Host entropy path over the C ABI: the range coder (src/odec.rs OdEcEncoder),
the frame-initial CDF set Cdfs::new(qctx) in semantic-slot order, the tile
packer (pack_wavefront_tile) and the filter-syntax replay
(replay_tile_with_filters)."""
import ctypes as C

import numpy as np

from . import abi
from .abi import load, ptr

TOKEN_BOOL = 1 << 30
TOKEN_GATHERED_PARTITION = 2 << 30
TOKEN_NOUPDATE = 3 << 30


def _check(rc, what):
    if rc != abi.MT_OK:
        from . import MtError

        raise MtError(rc, what)


def _take(p, n):
    lib = load()
    try:
        return C.string_at(p, n) if n else b""
    finally:
        lib.mt_free(p)


class RangeEncoder:
    """OdEcEncoder: encode_bool / encode_symbol(_noupdate) / encode_literal /
    encode_signed_subexp_with_ref, then done() -> bytes."""

    def __init__(self, updating_cdf=True):
        self._e = load().mt_range_encoder_new(int(bool(updating_cdf)))
        if not self._e:
            raise MemoryError("mt_range_encoder_new")

    def bool(self, value, f):
        _check(load().mt_range_encode_bool(self._e, int(bool(value)), int(f)), "mt_range_encode_bool")

    def symbol(self, s, cdf, adapt=True):
        """cdf: np.uint16 inverse CDF (counter last), adapted in place."""
        assert cdf.dtype == np.uint16 and cdf.flags.c_contiguous
        _check(load().mt_range_encode_symbol(self._e, int(s), ptr(cdf), len(cdf), int(bool(adapt))),
               "mt_range_encode_symbol")

    def literal(self, value, bits):
        _check(load().mt_range_encode_literal(self._e, int(value), int(bits)), "mt_range_encode_literal")

    def signed_subexp_with_ref(self, v, low, high, k, r):
        _check(load().mt_range_encode_signed_subexp_with_ref(self._e, v, low, high, k, r),
               "mt_range_encode_signed_subexp_with_ref")

    def done(self):
        out, n = C.c_void_p(), C.c_size_t()
        e, self._e = self._e, None
        _check(load().mt_range_encoder_done(e, C.byref(out), C.byref(n)), "mt_range_encoder_done")
        return _take(out, n.value)

    def __del__(self):
        if getattr(self, "_e", None):
            load().mt_range_encoder_free(self._e)
            self._e = None


def cdfs_default(qctx):
    """Cdfs::new(qctx) as (data u16, offsets u32, lens u16) in semantic-slot order."""
    lib = load()
    dl, ns = C.c_size_t(), C.c_int32()
    _check(lib.mt_cdfs_default(qctx, None, 0, None, None, 0, C.byref(dl), C.byref(ns)), "mt_cdfs_default")
    data = np.zeros(dl.value, np.uint16)
    off = np.zeros(ns.value, np.uint32)
    lens = np.zeros(ns.value, np.uint16)
    _check(lib.mt_cdfs_default(qctx, ptr(data), dl.value, ptr(off), ptr(lens), ns.value, None, None),
           "mt_cdfs_default")
    return data, off, lens


class TileTrace:
    def __init__(self, handle):
        self.handle = handle

    def __del__(self):
        if getattr(self, "handle", None):
            load().mt_tile_trace_free(self.handle)
            self.handle = None


def pack_tile(base_q_idx, sb_tokens, cdef_points=None, updating_cdf=True, want_trace=False):
    """pack_wavefront_tile: superblock token streams (lists of u32) -> payload
    bytes (and the TileTrace when want_trace)."""
    starts = np.zeros(len(sb_tokens) + 1, np.uint32)
    starts[1:] = np.cumsum([len(t) for t in sb_tokens])
    ops = np.concatenate([np.asarray(t, np.uint32) for t in sb_tokens]) if sb_tokens else np.zeros(1, np.uint32)
    ops = np.ascontiguousarray(ops, np.uint32)
    cp = None if cdef_points is None else np.ascontiguousarray(cdef_points, np.int32)
    out, n, tr = C.c_void_p(), C.c_size_t(), C.c_void_p()
    _check(load().mt_pack_tile(base_q_idx, int(bool(updating_cdf)), ptr(ops), ptr(starts), ptr(cp), len(sb_tokens),
                               C.byref(out), C.byref(n), C.byref(tr) if want_trace else None), "mt_pack_tile")
    payload = _take(out, n.value)
    return (payload, TileTrace(tr.value)) if want_trace else payload


def pack_tile_filtered(base_q_idx, sb_tokens, cdef_points, sb_cdef_idx=None, cdef_bits=0, updating_cdf=True):
    """pack_tile + replay_tile_with_filters in one pass (``mt_pack_tile_filtered``):
    superblock i's cdef_idx literal coded at its read_cdef() point."""
    starts = np.zeros(len(sb_tokens) + 1, np.uint32)
    starts[1:] = np.cumsum([len(t) for t in sb_tokens])
    ops = np.concatenate([np.asarray(t, np.uint32) for t in sb_tokens]) if sb_tokens else np.zeros(1, np.uint32)
    ops = np.ascontiguousarray(ops, np.uint32)
    cp = np.ascontiguousarray(cdef_points, np.int32)
    idx = None if sb_cdef_idx is None else np.ascontiguousarray(sb_cdef_idx, np.uint8)
    out, n = C.c_void_p(), C.c_size_t()
    _check(load().mt_pack_tile_filtered(base_q_idx, int(bool(updating_cdf)), ptr(ops), ptr(starts), ptr(cp),
                                        len(sb_tokens), ptr(idx), cdef_bits, C.byref(out), C.byref(n)),
           "mt_pack_tile_filtered")
    return _take(out, n.value)


def replay_tile_with_filters(trace, rect, cdef_grid=None, unit_cols=0, cdef_bits=0, updating_cdf=True):
    """replay_tile_with_filters without loop restoration; rect = (x0, y0, w, h)."""
    grid = None if cdef_grid is None else np.ascontiguousarray(cdef_grid, np.uint8).ravel()
    out, n = C.c_void_p(), C.c_size_t()
    _check(load().mt_replay_tile_with_filters(trace.handle, *rect, ptr(grid), unit_cols,
                                              0 if grid is None else len(grid), cdef_bits, int(bool(updating_cdf)),
                                              C.byref(out), C.byref(n)), "mt_replay_tile_with_filters")
    return _take(out, n.value)


def cdf_layout():
    """First slot of every CDF group (``abi.CdfSlotLayout``)."""
    out = abi.CdfSlotLayout()
    _check(load().mt_cdf_layout(C.byref(out)), "mt_cdf_layout")
    return out


def emit_coeffs(levels, blocks):
    """Coefficient tokens of transform blocks (``mt_emit_coeffs``): levels is an
    int32 array, blocks COEF_BLOCK_DTYPE records; returns (tokens u32, offsets
    (n + 1), res_ctx u8)."""
    levels = np.ascontiguousarray(levels, np.int32).ravel()
    blocks = np.ascontiguousarray(blocks, abi.COEF_BLOCK_DTYPE)
    n = len(blocks)
    offsets = np.zeros(n + 1, np.uint32)
    res = np.zeros(max(n, 1), np.uint8)
    tok = C.c_void_p()
    _check(load().mt_emit_coeffs(ptr(levels), len(levels), ptr(blocks), n, C.byref(tok), ptr(offsets), ptr(res)),
           "mt_emit_coeffs")
    total = int(offsets[n])
    try:
        toks = np.frombuffer(C.string_at(tok, total * 4), np.uint32).copy() if total else np.zeros(0, np.uint32)
    finally:
        load().mt_free(tok)
    return toks, offsets, res[:n]
