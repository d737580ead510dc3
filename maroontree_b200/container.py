"""Headers and container over the C ABI: leb128, OBU framing, the sequence
and frame headers, the frame OBU assembly and the AVIF wrapper."""
import ctypes as C

import numpy as np

from . import abi
from .abi import AvifItemParams, FrameHeaderParams, SequenceHeaderParams, load
from .entropy import _check, _take


def _bytes_call(fn, what, *args):
    out, n = C.c_void_p(), C.c_size_t()
    _check(fn(*args, C.byref(out), C.byref(n)), what)
    return _take(out, n.value)


def leb128(value):
    buf = (C.c_uint8 * 16)()
    n = C.c_size_t()
    _check(load().mt_leb128(value, buf, 16, C.byref(n)), "mt_leb128")
    return bytes(buf[:n.value])


def wrap_obu(obu_type, payload):
    p = C.create_string_buffer(bytes(payload), max(1, len(payload)))
    return _bytes_call(load().mt_wrap_obu, "mt_wrap_obu", obu_type, p, len(payload))


def tiling_increments(w8, h8, cols_log2, rows_log2):
    ci, ri = (C.c_uint8 * 8)(), (C.c_uint8 * 8)()
    nc, nr = C.c_int32(), C.c_int32()
    _check(load().mt_tiling_increments(w8, h8, cols_log2, rows_log2, ci, C.byref(nc), ri, C.byref(nr)),
           "mt_tiling_increments")
    return [bool(v) for v in ci[:nc.value]], [bool(v) for v in ri[:nr.value]]


def sequence_header(p):
    return _bytes_call(load().mt_sequence_header, "mt_sequence_header", C.byref(p))


def frame_header(p, trailing=False):
    return _bytes_call(load().mt_frame_header, "mt_frame_header", C.byref(p), int(bool(trailing)))


def _tile_arrays(tiles):
    bufs = [C.create_string_buffer(bytes(t), max(1, len(t))) for t in tiles]
    ptrs = (C.c_void_p * len(tiles))(*[C.addressof(b) for b in bufs])
    lens = (C.c_size_t * len(tiles))(*[len(t) for t in tiles])
    return bufs, ptrs, lens


def assemble_frame_obus(p, tiles):
    bufs, ptrs, lens = _tile_arrays(tiles)
    return _bytes_call(load().mt_assemble_frame_obus, "mt_assemble_frame_obus", C.byref(p), ptrs, lens, len(tiles))


def av1_stream(sp, fp, tiles):
    bufs, ptrs, lens = _tile_arrays(tiles)
    return _bytes_call(load().mt_av1_stream, "mt_av1_stream", C.byref(sp), C.byref(fp), ptrs, lens, len(tiles))


def level_for(w, h):
    return load().mt_av1_level_for(w, h)


def wrap_av1_image(obu, p, icc=None, exif=None):
    keep = []
    if icc is not None:
        b = C.create_string_buffer(bytes(icc), max(1, len(icc)))
        keep.append(b)
        p.icc, p.icc_len = C.addressof(b), len(icc)
    if exif is not None:
        b = C.create_string_buffer(bytes(exif), max(1, len(exif)))
        keep.append(b)
        p.exif, p.exif_len = C.addressof(b), len(exif)
    o = C.create_string_buffer(bytes(obu), max(1, len(obu)))
    return _bytes_call(load().mt_wrap_av1_image, "mt_wrap_av1_image", o, len(obu), C.byref(p))


def srgb_item(width, height, chroma="420", bit_depth=8):
    """AvifItemParams of a colour image with the sRGB-YCbCr CICP (1, 13, 6,
    full range), make_av1c's profile / level / subsampling (src/avif.rs:676-707)."""
    p = AvifItemParams()
    p.width, p.height, p.bit_depth, p.channels = width, height, bit_depth, 3
    p.seq_profile = {"420": 0, "444": 1, "422": 2}[chroma] if bit_depth < 12 else 2
    p.seq_level_idx = level_for(width, height)
    p.chroma_sub_x = int(chroma in ("420", "422"))
    p.chroma_sub_y = int(chroma == "420")
    p.color_present, p.primaries, p.transfer, p.matrix, p.full_range = 1, 1, 13, 6, 1
    p.imir_axis = -1
    return p
