"""The batched 16x16 level (mt_rdo_level16): every candidate result bit-exact
against the oracle's 16x16 chain (prediction with the corner filter, the 16x16
transforms with QM, trellis over SCAN_16X16, the TX_16X16 rate walk) and the
per-block winner the first minimum."""
import numpy as np
import pytest

from maroontree_b200 import abi, synth

TYPES16 = (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX, abi.TX_ADST_DCT, abi.TX_DCT_ADST)


def _setup16(oracle_lib, w, h, seed, qidx, qm_level, deltas=(0,)):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 7)
    blocks = synth.level_blocks(w, h, n=16, seed=seed)
    combos = synth.level_combos(range(13), TYPES16, deltas, delta_bits=lambda m, d: 0.5 + 0.0625 * abs(d))
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 16) if qm_level < 15 else None
    cdfs = synth.synthetic_cdfs(seed + 1, n_eob_bins=9)
    prm = mt.chain_params(w, h, tx_size=16, trellis_lambda0=0.05, mode_lambda=0.3 * qidx + 2.0, satd_scale=1.25,
                          satd_bridge=0.8)
    return src, rec, blocks, combos, q, qm, cdfs, prm


def test_oracle_level16_chain_runs(oracle_lib):
    """The oracle prices every 16x16 candidate (no invalid results), levels
    vary with the type, and the trellis only ever lowers magnitudes."""
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup16(oracle_lib, 64, 48, 3, 70, 6, deltas=(-1, 0, 2))
    cands = synth.candidates_of_level(blocks, combos)
    ref, lv, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, want_levels=True, threads=4)
    assert (ref["eob"] != abi.MT_EOB_INVALID).all()
    assert np.isfinite(ref["cost"]).all() and (ref["bits"] > 0).all()
    no_tr = prm.__class__.from_buffer_copy(prm)
    no_tr.trellis_lambda0 = 0.0
    raw, lv0, _ = oracle_lib.candidate_chain(src, rec, no_tr, q, qm, cdfs, cands, want_levels=True, threads=4)
    assert np.all(np.abs(lv) <= np.abs(lv0))
    assert (lv != lv0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,deltas", [(70, 6, (0,)), (116, 15, (-3, 0, 3)), (30, 2, (0,)),
                                                   (200, 8, (-1, 0, 1))])
def test_level16_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, deltas):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup16(oracle_lib, 160, 96, qidx, qidx, qm_level, deltas)
    best, res = mt_lib.rdo_level16(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    cands = synth.candidates_of_level(blocks, combos)
    ref, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=8)
    assert (ref["eob"] != abi.MT_EOB_INVALID).all()
    assert res.tobytes() == ref.tobytes()
    win = synth.best_of_level(ref, len(blocks), len(combos))
    assert np.array_equal(best["combo"], win)
    ref_w = ref.reshape(len(combos), len(blocks))[win, np.arange(len(blocks))]
    assert np.array_equal(best["cost"].view(np.uint32), ref_w["cost"].view(np.uint32))


@pytest.mark.gpu
def test_level16_rejects_v_h_and_out_of_frame(mt_lib, oracle_lib, cuda):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup16(oracle_lib, 64, 64, 4, 70, 6)
    combos = synth.level_combos((abi.DC_PRED, abi.V_PRED), (abi.TX_DCT_DCT, abi.TX_V_DCT))
    blocks = blocks.copy()
    blocks["px"][1] = 56  # crosses the right edge
    best, res = mt_lib.rdo_level16(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    r = res.reshape(len(combos), len(blocks))
    assert np.all(r[1]["eob"] == abi.MT_EOB_INVALID) and np.all(r[3]["eob"] == abi.MT_EOB_INVALID)
    assert np.all(r[:, 1]["eob"] == abi.MT_EOB_INVALID)
    assert best["combo"][1] == -1 and np.all(np.isin(best["combo"][np.arange(len(blocks)) != 1], (0, 2)))


@pytest.mark.gpu
def test_level16_masks_samples_past_the_displayed_frame(mt_lib, oracle_lib, cuda):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup16(oracle_lib, 160, 96, 5, 70, 6)
    prm.vis_w, prm.vis_h = 150, 90
    best, res = mt_lib.rdo_level16(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    ref, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, synth.candidates_of_level(blocks, combos),
                                           threads=8)
    assert res.tobytes() == ref.tobytes()
