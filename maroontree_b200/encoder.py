"""encode_rgb8 over the C ABI (``mt_encode_rgb8``): an 8-bit RGB image in, AVIF
bytes out, with ``EncodeConfig``'s fields (``abi.EncodeConfig``)."""
import ctypes as C

import numpy as np

from . import abi
from .abi import load, ptr
from .entropy import _check, _take


def config(**kw):
    """EncodeConfig::default() with fields overridden by keyword."""
    c = abi.EncodeConfig()
    _check(load().mt_encode_config_default(C.byref(c)), "mt_encode_config_default")
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _planes_out(w, h, sub):
    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    pcw, pch = (pw >> 1, ph >> 1) if sub else (pw, ph)
    return [np.zeros((ph, pw), np.uint16), np.zeros((pch, pcw), np.uint16), np.zeros((pch, pcw), np.uint16)]


def encode_rgb8(rgb, cfg=None, want_recon=False, stats=None):
    """rgb: (h, w, 3) uint8.  Returns the AVIF bytes (and the decoder's output
    planes, padded, when want_recon); fills ``stats`` (abi.EncodeStats) when
    given."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w = rgb.shape[:2]
    cfg = cfg if cfg is not None else config()
    out, n = C.c_void_p(), C.c_size_t()
    planes = _planes_out(w, h, cfg.chroma == 0) if want_recon else None
    arr = (C.c_void_p * 3)(*[p.ctypes.data for p in planes]) if want_recon else None
    _check(load().mt_encode_rgb8_ex(ptr(rgb), w, h, C.byref(cfg), C.byref(out), C.byref(n), arr,
                                    C.byref(stats) if stats is not None else None), "mt_encode_rgb8")
    data = _take(out, n.value)
    return (data, planes) if want_recon else data


def encode_rgb8_device(d_rgb, w, h, cfg=None, stats=None):
    """The encode of interleaved RGB already in device memory (d_rgb: a device
    pointer as an int, w * h * 3 bytes).  Returns the AVIF bytes."""
    cfg = cfg if cfg is not None else config()
    out, n = C.c_void_p(), C.c_size_t()
    _check(load().mt_encode_rgb8_device(C.c_void_p(d_rgb), w, h, C.byref(cfg), C.byref(out), C.byref(n),
                                        C.byref(stats) if stats is not None else None), "mt_encode_rgb8_device")
    return _take(out, n.value)


def encode_yuv8(y, u, v, cfg, want_recon=False):
    """8-bit planes at their displayed sizes, coded as given (no colour conversion)."""
    y, u, v = [np.ascontiguousarray(p, np.uint8) for p in (y, u, v)]
    h, w = y.shape
    out, n = C.c_void_p(), C.c_size_t()
    planes = _planes_out(w, h, cfg.chroma == 0) if want_recon else None
    arr = (C.c_void_p * 3)(*[p.ctypes.data for p in planes]) if want_recon else None
    _check(load().mt_encode_yuv8(ptr(y), ptr(u), ptr(v), w, h, C.byref(cfg), C.byref(out), C.byref(n), arr),
           "mt_encode_yuv8")
    data = _take(out, n.value)
    return (data, planes) if want_recon else data


def encode_rgb8_batch(images, cfgs=None, stats=None):
    """mt_encode_rgb8_batch: a list of (h, w, 3) uint8 images (and one config
    per image, or one for all) encoded in one call.  Returns the list of AVIF
    bytes; raises on the first failing image.  ``stats``: a list of
    abi.EncodeStats to fill, one per image."""
    n = len(images)
    imgs = [np.ascontiguousarray(im, np.uint8) for im in images]
    if cfgs is None or isinstance(cfgs, abi.EncodeConfig):
        cfgs = [cfgs if cfgs is not None else config()] * n
    carr = (abi.EncodeConfig * n)(*cfgs)
    ptrs = (C.c_void_p * n)(*[im.ctypes.data for im in imgs])
    ws = (C.c_uint32 * n)(*[im.shape[1] for im in imgs])
    hs = (C.c_uint32 * n)(*[im.shape[0] for im in imgs])
    outs = (C.c_void_p * n)()
    lens = (C.c_size_t * n)()
    rcs = (C.c_int32 * n)()
    st = (abi.EncodeStats * n)() if stats is not None else None
    rc = load().mt_encode_rgb8_batch(n, ptrs, ws, hs, carr, outs, lens, rcs, st)
    res = []
    for i in range(n):
        res.append(_take(C.c_void_p(outs[i]), lens[i]) if outs[i] else None)
    if stats is not None:
        for i in range(n):
            C.memmove(C.byref(stats[i]), C.byref(st[i]), C.sizeof(abi.EncodeStats))
    _check(rc, "mt_encode_rgb8_batch")
    return res
