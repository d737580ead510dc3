"""Recursive filter-intra prediction and the filter-intra shortlist ranking
(rank_filter_intra_modes).

The oracle's predictor is pinned by the reference's own tests, restated
(src/intrapred.rs:2417-2478): constant edges stay constant for every size,
mode and bit depth; missing edges are filled and outputs stay in range; the
filter is recursive across 4x2 cells (the corner reaches the last rows).  The
GPU tests compare the device kernel's predictions, scores and order with the
oracle bit for bit."""
import numpy as np
import pytest

from maroontree_b200 import synth

SIZES = [(4, 4), (4, 8), (8, 4), (8, 8), (8, 16), (16, 8), (16, 16), (16, 32), (32, 16), (32, 32), (4, 16), (16, 4),
         (8, 32), (32, 8)]


def test_constant_edges_stay_constant(oracle_lib):
    for bd in (8, 10, 12):
        value = 37 << (bd - 8)
        recon = np.full((40, 40), value, np.uint16)
        for w, h in SIZES:
            for mode in range(5):
                out = oracle_lib.filter_intra_predict(recon, 1, 1, w, h, mode, bd)
                assert (out == value).all(), (mode, w, h, bd)


def test_missing_edges_and_clipping(oracle_lib):
    for bd in (8, 10, 12):
        mx = (1 << bd) - 1
        recon = np.full((32, 32), mx, np.uint16)
        for ox, oy in ((0, 0), (1, 0), (0, 1), (1, 1)):
            for mode in range(5):
                out = oracle_lib.filter_intra_predict(recon, ox, oy, 8, 8, mode, bd)
                assert ((out >= 0) & (out <= mx)).all()


def test_recursive_across_cells(oracle_lib):
    recon = np.full((16, 16), 128, np.uint16)
    recon[0, :8] = 16 + 20 * np.arange(8)
    recon[:8, 0] = 240 - 18 * np.arange(8)
    a = oracle_lib.filter_intra_predict(recon, 1, 1, 8, 8, 3)  # D157
    recon[0, 0] ^= 63
    b = oracle_lib.filter_intra_predict(recon, 1, 1, 8, 8, 3)
    assert (a.ravel()[:8] != b.ravel()[:8]).any()
    assert (a.ravel()[32:] != b.ravel()[32:]).any()


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 17)
    return src, rec


def _pos(fw, fh, w, h):
    ys, xs = np.meshgrid(np.arange(0, fh - h + 1, h), np.arange(0, fw - w + 1, w), indexing="ij")
    return np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.uint16)


def test_beam_oracle_orders_by_score_then_mode(oracle_lib):
    src, rec = _frame(64, 48, 2)
    scores, modes, preds = oracle_lib.filter_intra_beam(src, rec, 8, 8, _pos(64, 48, 8, 8))
    assert (np.diff(scores.astype(np.float64), axis=1) >= 0).all()
    for s, m in zip(scores, modes):
        assert sorted(zip(s.tolist(), m.tolist())) == list(zip(s.tolist(), m.tolist()))
    assert len(np.unique(modes[:, 0])) > 1


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(4, 4), (8, 8), (16, 16), (32, 32), (8, 16), (32, 8), (4, 16)])
def test_filter_intra_beam_gpu_matches_oracle(mt_lib, oracle_lib, cuda, w, h):
    src, rec = _frame(128, 96, w * 5 + h)
    pos = _pos(128, 96, w, h)
    vis = (0, 0) if w != 8 else (125, 90)
    scores, modes, preds = mt_lib.filter_intra_beam(src, rec, w, h, pos, vis=vis, want_preds=True)
    ws, wm, wp = oracle_lib.filter_intra_beam(src, rec, w, h, pos, vis=vis)
    assert np.array_equal(preds, wp)
    assert np.array_equal(scores, ws) and np.array_equal(modes, wm)


@pytest.mark.gpu
def test_filter_intra_beam_10bit_and_outside(mt_lib, oracle_lib, cuda):
    src, rec = _frame(64, 64, 4)
    src, rec = src * 4 + 1, rec * 4 + 2
    pos = _pos(64, 64, 16, 16)
    pos[3] = (56, 0)  # crosses the right edge
    scores, modes, _ = mt_lib.filter_intra_beam(src, rec, 16, 16, pos, bd=10)
    ws, wm, _ = oracle_lib.filter_intra_beam(src, rec, 16, 16, pos, bd=10)
    assert np.array_equal(scores, ws) and np.array_equal(modes, wm)
    assert (modes[3] == 255).all()
