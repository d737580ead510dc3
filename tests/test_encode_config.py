"""The encode boundary's configuration: EncodeConfig::default()
(src/avif.rs:318-344), EncodeConfig::validate and encode_rgb8's input checks
(src/avif.rs:577-635, :915-923) with one error code per EncodeError variant,
and the frame settings a config resolves to (quality_to_q, the QM levels of
EncodeConfig::vb, cdef_enabled).  No device call."""
import ctypes as C

import pytest

from maroontree_b200 import abi


def _cfg(lib, **kw):
    c = abi.EncodeConfig()
    assert lib.mt_encode_config_default(C.byref(c)) == abi.MT_OK
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def test_defaults(mt_lib):
    c = _cfg(mt_lib.load())
    assert (c.quality, c.chroma, c.speed, c.threads) == (80, 0, 1, 0)
    assert (c.color_present, c.primaries, c.transfer, c.matrix, c.full_range) == (1, 1, 13, 6, 1)
    assert (c.updating_cdf, c.adaptive_quant, c.variance_boost, c.dark_aq) == (1, 1, 1, 1)
    assert (c.cdef, c.wiener, c.quantization_matrices, c.screen_content, c.intrabc) == (0, 0, 1, 1, 1)
    assert (c.qmatrix_level, c.alpha_quality) == (-1, -1)


def test_validation_codes(mt_lib):
    lib = mt_lib.load()
    assert lib.mt_encode_config_validate(C.byref(_cfg(lib))) == abi.MT_OK
    assert lib.mt_encode_config_validate(C.byref(_cfg(lib, quality=101))) == abi.MT_ERR_INVALID_QUALITY
    assert lib.mt_encode_config_validate(C.byref(_cfg(lib, alpha_quality=101))) == abi.MT_ERR_INVALID_QUALITY
    assert lib.mt_encode_config_validate(C.byref(_cfg(lib, qmatrix_level=16))) == abi.MT_ERR_INVALID_QUALITY
    assert lib.mt_encode_config_validate(C.byref(_cfg(lib, quality=100, qmatrix_level=15))) == abi.MT_OK


@pytest.mark.parametrize("w,h,n,rc", [(512, 512, 512 * 512 * 3, 0), (0, 5, 0, -20), (16384, 8, 16384 * 24, -20),
                                      (16383, 16383, 16383 * 16383 * 3, 0), (4, 4, 47, -2)])
def test_rgb8_input_checks(mt_lib, w, h, n, rc):
    assert mt_lib.load().mt_validate_rgb8_input(w, h, n) == rc


@pytest.mark.parametrize("quality,chroma,speed,want", [
    (60, 0, 1, (70, 6, 6, 1)), (40, 0, 1, (116, 1, 1, 1)), (80, 0, 1, (35, 8, 8, 1)), (60, 2, 1, (70, 6, 2, 1)),
    (60, 0, 3, (70, 6, 6, 0))])
def test_effective_settings(mt_lib, oracle_lib, quality, chroma, speed, want):
    lib = mt_lib.load()
    plan = abi.EncodePlan()
    assert lib.mt_encode_config_effective(C.byref(_cfg(lib, quality=quality, chroma=chroma, speed=speed)),
                                          C.byref(plan)) == abi.MT_OK
    sub = {0: 2, 1: 1, 2: 0}[chroma]
    q = oracle_lib.quality_to_q(quality)
    assert (plan.base_q_idx, plan.qm_y, plan.qm_u, plan.cdef) == want
    assert plan.qm_y == oracle_lib.qm_level_law(q, sub) and plan.qm_u == oracle_lib.qm_chroma_level_law(q, sub)
    flat = abi.EncodePlan()
    assert lib.mt_encode_config_effective(C.byref(_cfg(lib, quantization_matrices=0)), C.byref(flat)) == 0
    assert (flat.qm_y, flat.qm_u, flat.qm_v) == (15, 15, 15)
