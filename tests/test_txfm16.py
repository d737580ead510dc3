"""The 16x16 transforms of the oracle, pinned to the reference's own checks:
the WC16 weights (src/dct.rs:3833-3844), dct1d_16 on zero / DC / a float model
(src/dct.rs:4052-4089), forward + inverse round trips at high quality
(src/dct.rs:4327-4400, here for every 16x16 type), and the dav1d inverse's
rotation rewrite (rot12) against the reference's literal forms."""
import math

import numpy as np
import pytest

from maroontree_b200 import abi


def _wc(k, n):
    return int(math.floor(65536.0 / (2.0 * math.cos((2 * k + 1) * math.pi / (2 * n))) + 0.5))


def test_wc16_weights():
    # dct.rs:3833-3844: round(65536 / (2 cos((2k+1) pi / 32)))
    assert [_wc(k, 16) for k in range(8)] == [32927, 34242, 37155, 42390, 51653, 69513, 112882, 334309]


def test_dct1d_16_zero_and_dc(oracle_lib):
    assert np.all(oracle_lib.dct1d(np.zeros(16, np.int32)) == 0)
    out = oracle_lib.dct1d(np.full(16, 128, np.int32))
    assert out[0] != 0 and np.all(np.abs(out[1:]) <= 4)


def test_dct1d_16_matches_float_dct(oracle_lib):
    """The integer 16-point DCT against the unnormalised DCT-II with the AC
    bins scaled by sqrt(2) (the reference's float model), within the
    reference's tolerance of 13 on 128-scaled input (dct.rs:4069-4089)."""
    sig = [math.cos(i * 0.4 + 1.0) for i in range(16)]
    fixed = np.array([int(round(v * 128.0)) for v in sig], np.int32)
    got = oracle_lib.dct1d(fixed)
    n = 16
    for k in range(n):
        ref = (math.sqrt(2.0) if k else 1.0) * sum(int(fixed[i]) * math.cos((2 * i + 1) * k * math.pi / (2 * n))
                                                    for i in range(n))
        assert abs(int(got[k]) - round(ref)) <= 13, (k, got[k], ref)


def _patterns():
    ramp = np.zeros((16, 16), np.int32)
    edge = np.zeros((16, 16), np.int32)
    curve = np.zeros((16, 16), np.int32)
    rnd = np.zeros((16, 16), np.int32)
    rng = 777
    for y in range(16):
        for x in range(16):
            ramp[y, x] = x * 3 + y * 2 - 40
            edge[y, x] = -60 if x + y // 2 < 10 else 70
            fx, fy = x / 15.0, y / 15.0
            curve[y, x] = int(90.0 * math.sin(fx * fx - fy * 0.7) - 10.0)
            rng ^= (rng << 13) & 0xFFFFFFFF
            rng ^= rng >> 17
            rng ^= (rng << 5) & 0xFFFFFFFF
            rnd[y, x] = rng % 61 - 30
    return {"ramp": ramp, "edge": edge, "curve": curve, "noise": rnd}


@pytest.mark.parametrize("tx", [abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST, abi.TX_IDTX])
def test_16x16_round_trip_at_high_quality(oracle_lib, tx):
    q = oracle_lib.quant_new(4, 8, 15)
    for name, r in _patterns().items():
        cf, _ = oracle_lib.fwd_txfm_quant(r, tx, q, None)
        rr = oracle_lib.inv_txfm_dequant(cf, tx, q, None).reshape(16, 16)
        en = float(np.sum(r.astype(np.float64) ** 2))
        sse = float(np.sum((r - rr).astype(np.float64) ** 2))
        assert sse / en < 2e-3, (tx, name, sse / en)


def test_16x16_qm_round_trip(oracle_lib):
    """With a quantisation matrix the levels shrink where the weights are large
    and the reconstruction still tracks the residual at high quality."""
    q = oracle_lib.quant_new(4, 8, 6)
    qm = oracle_lib.qm_row(6, 0, 16)
    r = _patterns()["curve"]
    cf, _ = oracle_lib.fwd_txfm_quant(r, abi.TX_DCT_DCT, q, qm)
    rr = oracle_lib.inv_txfm_dequant(cf, abi.TX_DCT_DCT, q, qm).reshape(16, 16)
    assert float(np.sum((r - rr) ** 2.0)) / float(np.sum(r ** 2.0)) < 5e-3


def test_adst16_table_bound():
    """Row sums of |ADST16_FWD_Q12| keep both passes of 8-bit residuals inside
    int32 (the device accumulates in 32 bits)."""
    import re
    import os
    text = open(os.path.join(os.path.dirname(__file__), "..", "maroontree_b200", "csrc", "av1_tables.h")).read()
    body = text.split("MT_ADST16_FWD_Q12[256] = {")[1].split("}")[0]
    a = np.array([int(v) for v in re.findall(r"-?\d+", body)], np.int64).reshape(16, 16)
    s = int(np.abs(a).sum(axis=1).max())
    first = (255 * s + 2048) >> 12
    assert first * s + 2048 < 2 ** 31 and 255 * s < 2 ** 31


def test_rotation_rewrite_is_exact():
    """dav1d writes a rotation x*c1 + y*c2 with one constant minus 4096 and the
    input added back, or with both constants halved and >> 11; the oracle and
    the device use (x*c1 + y*c2 + 2048) >> 12.  Equal for every input in the
    clipped ranges (Python integers: floor shifts, no overflow)."""
    rng = np.random.default_rng(5)
    xs = rng.integers(-(1 << 16), 1 << 16, 20000)
    ys = rng.integers(-(1 << 16), 1 << 16, 20000)
    for x, y in zip(xs.tolist(), ys.tolist()):
        # ((x*401 - y*(4076 - 4096) + 2048) >> 12) - y  ==  rot(x, 401, y, -4076)
        assert ((x * 401 - y * (4076 - 4096) + 2048) >> 12) - y == (x * 401 - y * 4076 + 2048) >> 12
        # (x*1583 - y*1299 + 1024) >> 11  ==  rot(x, 3166, y, -2598)
        assert (x * 1583 - y * 1299 + 1024) >> 11 == (x * 3166 - y * 2598 + 2048) >> 12
        # ((-(x*(3784 - 4096) + y*1567) + 2048) >> 12) - x  ==  rot(x, -3784, y, -1567)
        assert ((-(x * (3784 - 4096) + y * 1567) + 2048) >> 12) - x == (-x * 3784 - y * 1567 + 2048) >> 12
        # ((x*(3920 - 4096) - y*1189 + 2048) >> 12) + x  ==  rot(x, 3920, y, -1189)
        assert ((x * (3920 - 4096) - y * 1189 + 2048) >> 12) + x == (x * 3920 - y * 1189 + 2048) >> 12
