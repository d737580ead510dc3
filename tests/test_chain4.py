"""The 4x4 luma candidate chain (the SPLIT4 pricing of
src/coder/lossy_state.rs:2064-2290 and the 4x4 transform trials of
src/coder/partition_search.rs:4520-4640): oracle pins for the 4x4 transforms
restated from the reference's own tests, and bit-exact GPU parity of the batched
4x4 level (mt_rdo_level4) with the oracle."""
import numpy as np
import pytest

from maroontree_b200 import abi, synth

TYPES = [abi.TX_IDTX, abi.TX_DCT_DCT, abi.TX_V_DCT, abi.TX_H_DCT, abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST]


def test_oracle_adst4_roundtrip_high_quality(oracle_lib):
    """src/idct.rs adst4_roundtrip_highq: forward ADST4 then the dav1d inverse
    tracks the residual at qindex 8 (mean abs error within a quarter of the
    signal, +16)."""
    q = oracle_lib.quant_new_chroma(8, 0, 0)
    residuals = [
        [40, -32, 20, -12, 28, -24, 16, -8, 36, -28, 24, -4, 32, -20, 12, -16],
        [80, 70, -40, 30, -60, 50, 20, -10, 44, -36, 24, -16, 32, -28, 12, -4],
        [-50, 48, -46, 44, 42, -40, 38, -36, 34, 32, -30, 28, 26, -24, 22, -20],
    ]
    for res in residuals:
        res = np.array(res, np.int32)
        levels, _ = oracle_lib.fwd_txfm_quant(res, abi.TX_ADST_ADST, q, None)
        rec = oracle_lib.inv_txfm_dequant(levels, abi.TX_ADST_ADST, q, None)
        err = int(np.abs(rec - res).sum())
        sig = int(np.abs(res).sum())
        assert err * 4 <= sig + 16, (err, sig)


def test_oracle_adst4_dc_only_is_finite(oracle_lib):
    """src/idct.rs adst4_dc_only_is_finite: a lone DC level stays in range."""
    q = oracle_lib.quant_new_chroma(40, 0, 0)
    levels = np.zeros(16, np.int32)
    levels[0] = 12
    rec = oracle_lib.inv_txfm_dequant(levels, abi.TX_ADST_ADST, q, None)
    assert np.all(np.abs(rec) < 4096)


@pytest.mark.parametrize("tx", [t for t in TYPES if t not in (abi.TX_V_DCT, abi.TX_H_DCT)])
def test_oracle_4x4_roundtrip_every_type(oracle_lib, tx):
    """Every 2-D 4x4 type and IDTX reconstructs a random residual at qindex 8
    (flat QM) to within the quantiser's reach.  (The 1-D V/H pair is not
    gain-matched in the reference: its forward x 2 sqrt2 DCT against dav1d's
    identity4 x DCT4 inverse gives a 1/sqrt2 round trip, restated as is.)"""
    rng = np.random.default_rng(tx)
    q = oracle_lib.quant_new(8, 8, 15)
    for _ in range(20):
        res = rng.integers(-80, 81, 16).astype(np.int32)
        levels, _ = oracle_lib.fwd_txfm_quant(res, tx, q, None)
        rec = oracle_lib.inv_txfm_dequant(levels, tx, q, None)
        assert np.abs(rec - res).max() <= 8, (tx, res, rec)


def test_oracle_4x4_qm_changes_only_2d_types(oracle_lib):
    """The quantisation matrix re-rounds the 2-D types only (the identity
    family quantises flat, src/dct.rs:2510-2523)."""
    rng = np.random.default_rng(5)
    res = rng.integers(-120, 121, 16).astype(np.int32)
    q = oracle_lib.quant_new(60, 8, 2)
    qm = oracle_lib.qm_row(2, 0, 4)
    for tx in TYPES:
        a, _ = oracle_lib.fwd_txfm_quant(res, tx, q, None)
        b, _ = oracle_lib.fwd_txfm_quant(res, tx, q, qm)
        if tx in (abi.TX_IDTX, abi.TX_V_DCT, abi.TX_H_DCT):
            assert np.array_equal(a, b)


def _setup4(oracle_lib, w, h, seed, qidx, qm_level, deltas=(0,)):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 7)
    blocks = synth.level_blocks(w, h, n=4, seed=seed)
    # The SPLIT4 trial set: DCT and ADST trellis-optimised, IDTX priced as
    # quantised (plus the asymmetric ADST pairs).
    combos = synth.level_combos(range(13), (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX, abi.TX_ADST_DCT,
                                            abi.TX_DCT_ADST), deltas, no_trellis_types=(abi.TX_IDTX,))
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 4) if qm_level < 15 else None
    cdfs = synth.synthetic_cdfs(seed + 1, n_eob_bins=5)
    prm = mt.chain_params(w, h, tx_size=4, trellis_lambda0=0.05, mode_lambda=0.3 * qidx + 2.0, satd_scale=1.25,
                          satd_bridge=0.8)
    return src, rec, blocks, combos, q, qm, cdfs, prm


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,deltas", [(70, 6, (0,)), (116, 15, (0,)), (30, 2, (-2, 0, 3)), (200, 8, (0,))])
def test_level4_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, deltas):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup4(oracle_lib, 128, 72, qidx, qidx, qm_level, deltas)
    best, res = mt_lib.rdo_level4(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    cands = synth.candidates_of_level(blocks, combos)
    ref, lv, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=8)
    assert (ref["eob"] != abi.MT_EOB_INVALID).all()
    assert res.tobytes() == ref.tobytes()
    win = synth.best_of_level(ref, len(blocks), len(combos))
    assert np.array_equal(best["combo"], win)
    ref_w = ref.reshape(len(combos), len(blocks))[win, np.arange(len(blocks))]
    assert np.array_equal(best["cost"].view(np.uint32), ref_w["cost"].view(np.uint32))


def test_oracle_level4_no_trellis_flag_changes_only_flagged(oracle_lib, mt_lib):
    """MT_CAND_NO_TRELLIS prices the quantised levels: the flagged IDTX
    candidates differ from their trellis-optimised twins somewhere, the others
    not at all."""
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup4(oracle_lib, 64, 32, 4, 60, 15)
    cands = synth.candidates_of_level(blocks, combos)
    a, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands)
    plain = cands.copy()
    plain["flags"] &= ~np.uint8(abi.CAND_NO_TRELLIS)
    b, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, plain)
    flagged = (cands["flags"] & abi.CAND_NO_TRELLIS) != 0
    assert flagged.any() and np.array_equal(a[~flagged], b[~flagged])
    assert not np.array_equal(a[flagged]["cost"], b[flagged]["cost"])


@pytest.mark.gpu
def test_level4_masks_samples_past_the_displayed_frame(mt_lib, oracle_lib, cuda):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup4(oracle_lib, 128, 72, 6, 70, 6)
    prm.vis_w, prm.vis_h = 126, 69
    best, res = mt_lib.rdo_level4(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    ref, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, synth.candidates_of_level(blocks, combos),
                                           threads=8)
    assert res.tobytes() == ref.tobytes()
