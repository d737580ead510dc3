"""Known-answer and property tests of the oracle, restated from the
reference's own unit tests (file:line of each in its docstring)."""
import math

import numpy as np
import pytest

from maroontree_b200 import abi


def q16(v):
    return int(math.floor(v * 65536.0 + 0.5))


def wc(k, n):
    return q16(1.0 / (2.0 * math.cos((2 * k + 1) * math.pi / (2 * n))))


def test_butterfly_constants_match_formula():
    """dct.rs:3808-3857: WC4/WC8 and SQRT2 are round(65536 / (2 cos((2k+1)pi/2n)))."""
    assert (35468, 85627) == (wc(0, 4), wc(1, 4))
    assert [33410, 39410, 58981, 167963] == [wc(k, 8) for k in range(4)]
    assert 92682 == q16(math.sqrt(2.0))


def test_qm_level0_4x4_weights(oracle_lib):
    """quant.rs:498-509: normative level-0 4x4 weights, rc = x*4 + y."""
    expected = [32, 43, 73, 97, 43, 67, 94, 110, 73, 94, 137, 150, 97, 110, 150, 200]
    row = oracle_lib.qm_row(0, 0, 4)
    for y in range(4):
        for x in range(4):
            assert row[x * 4 + y] == expected[y * 4 + x]


def test_qm_forward_inverse_reciprocal(oracle_lib):
    """quant.rs:511-519: forward weight (1024 + w/2)/w is the reciprocal of the inverse."""
    row = oracle_lib.qm_row(10, 0, 16).astype(np.int64)
    fwd = (1024 + row // 2) // row
    assert np.all(np.abs(fwd * row - 1024) <= row // 2)


def test_flat_level_has_no_row(oracle_lib):
    """quant.rs:485-496: level 15 is flat."""
    assert oracle_lib.qm_row(15, 0, 8) is None


def test_quant_q60(oracle_lib):
    """Quant::new_with_qm at qindex 70 (quality 60): dc index 62 (luma DC delta -8)."""
    q = oracle_lib.quant_new(70, 8, 6)
    assert (q.dc_q, q.ac_q) == (59, 77)
    assert q.q_mult_dc == round(65536 / 59) and q.q_mult_ac == round(65536 / 77)
    assert (q.rmin, q.rmax, q.cf_max) == (-32768, 32767, 32767)


def test_edge_filter_thresholds(oracle_lib):
    """intrapred.rs:2481-2496."""
    s = oracle_lib.load().or_edge_filter_strength
    assert s(4, 4, 0, 55) == 0 and s(4, 4, 0, 56) == 1
    assert s(8, 16, 0, 8) == 1 and s(8, 16, 0, 16) == 2 and s(8, 16, 0, 32) == 3
    u = oracle_lib.load().or_use_edge_upsample
    assert u(8, 8, 0, 23) and not u(8, 8, 0, 40) and not u(8, 8, 1, 23)


def test_satd_zero_for_exact_reconstruction(oracle_lib):
    """partition_rd.rs:147-152."""
    src = (np.arange(64) * 3).astype(np.uint16).reshape(8, 8)
    pred = src.astype(np.int32).ravel()
    lib = oracle_lib.load()
    assert lib.or_luma_satd(src.ctypes.data, 8, 0, 0, 8, 8, 255, pred.ctypes.data, None) == 0


@pytest.mark.parametrize("tx,edge", [(abi.TX_H_DCT, "vert"), (abi.TX_V_DCT, "horz")])
def test_vh_dct_roundtrip(oracle_lib, tx, edge):
    """idct.rs:3293-3335: V/H_DCT 8x8 reconstruct edges within one step^2 MSE."""
    q = oracle_lib.quant_new(40, 8, 15)
    y, x = np.mgrid[0:8, 0:8]
    resid = np.where((x < 4) if edge == "vert" else (y < 4), 60, -60).astype(np.int32)
    cf, _ = oracle_lib.fwd_txfm_quant(resid, tx, q, None)
    assert np.any(cf != 0)
    rr = oracle_lib.inv_txfm_dequant(cf, tx, q, None)
    mse = np.mean((rr - resid.ravel()) ** 2)
    assert mse < q.ac_q ** 2


@pytest.mark.parametrize("tx", list(range(7)))
def test_all_types_roundtrip_8x8(oracle_lib, tx):
    """Every 8x8 forward/inverse pair reconstructs a smooth residual within quantisation error
    (the property idct.rs:3337 asserts for the rect16 seven types)."""
    q = oracle_lib.quant_new(40, 8, 15)
    y, x = np.mgrid[0:8, 0:8]
    resid = (40 * np.cos(np.pi * x / 9) + 25 * np.sin(np.pi * y / 11)).astype(np.int32)
    cf, _ = oracle_lib.fwd_txfm_quant(resid, tx, q, None)
    rr = oracle_lib.inv_txfm_dequant(cf, tx, q, None)
    assert np.mean((rr - resid.ravel()) ** 2) < q.ac_q ** 2


def test_dct_of_constant_is_dc_only(oracle_lib):
    """dct.rs:3993-4001: a flat input leaves only the DC bin (AC within rounding)."""
    q = oracle_lib.quant_new(1, 8, 15)
    cf, tf = oracle_lib.fwd_txfm_quant(np.full(64, 64, np.int32), abi.TX_DCT_DCT, q, None)
    assert cf[0] != 0 and np.all(np.abs(cf[1:]) <= 1)


def test_trellis_output_is_valid(oracle_lib):
    """trellis.rs:1060-1101: only lowers magnitudes, never flips a sign, zeroes past the EOB."""
    rng = np.random.default_rng(0x2545F491)
    scan = oracle_lib.default_scan(8)
    for _ in range(500):
        tf = np.zeros(64, np.float32)
        cf = np.zeros(64, np.int32)
        for _ in range(1 + rng.integers(0, 40)):
            rc = rng.integers(0, 64)
            mag = rng.integers(0, 6) + rng.random()
            sign = 1 if rng.integers(0, 2) == 0 else -1
            tf[rc] = sign * mag
            cf[rc] = int(sign * round(mag))
        opt = oracle_lib.trellis_optimize(cf, tf, 200.0, 220.0, scan, 0.05)
        nz = [i for i in range(64) if opt[scan[i]] != 0]
        if nz:
            assert all(opt[scan[i]] == 0 for i in range(nz[-1] + 1, 64))
        assert np.all(np.abs(opt) <= np.abs(cf))
        assert np.all((opt == 0) | (np.sign(opt) == np.sign(cf)))


def test_cdf_cost_q22(oracle_lib):
    """cost.rs:156-190: cost of an even split is one bit; a certain symbol costs ~0."""
    cdf = np.array([16384, 0], np.uint16)
    assert oracle_lib.cdf_cost(cdf, 0) == pytest.approx(1.0, abs=1e-6)
    cdf = np.array([0, 0], np.uint16)
    assert oracle_lib.cdf_cost(cdf, 0) == 0.0


def test_rate_prefers_clustered_levels(oracle_lib):
    """rate.rs:340-365: clustered low-frequency levels cost fewer bits than scattered ones."""
    from maroontree_b200 import synth

    cdfs = synth.synthetic_cdfs(11)
    scan = oracle_lib.default_scan(8)
    clustered = np.zeros(64, np.int32)
    scattered = np.zeros(64, np.int32)
    for i in (0, 1, 2, 3):
        clustered[scan[i]] = 2
    for i in (0, 12, 24, 36):
        scattered[scan[i]] = 2
    lib = oracle_lib.load()
    f = lambda cf: lib.or_real_block_bits(cf.ctypes.data, scan.ctypes.data, 8, 1, cdfs, 0, 0, 0, 1, 0, None)
    assert f(clustered) < f(scattered)


def test_chain_oracle_is_deterministic_across_threads(oracle_lib):
    """Serial == threaded oracle (the reference's wavefront == serial identity, avif.rs:1983-2005)."""
    import maroontree_b200 as mt
    from maroontree_b200 import synth

    src = synth.rgb_to_luma(synth.generate_rgb(64, 64, 1))
    rec = synth.synthetic_recon(src, 2)
    cands = synth.level_candidates(64, 64, range(13), abi.TX_2D_SCAN_TYPES)
    q = oracle_lib.quant_new(70, 8, 6)
    prm = mt.chain_params(64, 64, mode_lambda=20.0, satd_bridge=0.7)
    cdfs = synth.synthetic_cdfs(5)
    a, la, ra = oracle_lib.candidate_chain(src, rec, prm, q, oracle_lib.qm_row(6, 0, 8), cdfs, cands, True, True, 1)
    b, lb, rb = oracle_lib.candidate_chain(src, rec, prm, q, oracle_lib.qm_row(6, 0, 8), cdfs, cands, True, True, 4)
    assert a.tobytes() == b.tobytes() and np.array_equal(la, lb) and np.array_equal(ra, rb)
