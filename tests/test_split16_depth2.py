"""The 16x16 leaf's depth-2 trial (split16_depth2_try): sixteen TX_4X4 per
job with the DCT / ADST / IDTX / V_DCT / H_DCT choice.

The CPU tests pin the oracle's glue (raster order, per-4x4 edge flags, the
patch prediction, the guard and rd gates, the job's own dc_sign contexts)
against a composition of the oracle's primitives, and the 1-D 4x4 walk's
DC-only form term by term, with the default luma TX_4X4 CDFs of the
reference's Cdfs::new(0) (tests/golden/cdfs_luma_tx4_qctx0.json).  The GPU
tests compare the CUDA kernel with the oracle bit for bit."""
import json
import os

import numpy as np
import pytest

from maroontree_b200 import abi, synth

GOLDEN_TX4 = os.path.join(os.path.dirname(__file__), "golden", "cdfs_luma_tx4_qctx0.json")
INF = float("inf")


def _icdf(vals, width):
    """src/tables.rs:31-35 icdf: 32768 - v per entry, then the terminal 0."""
    out = np.zeros(width, np.uint16)
    out[:len(vals)] = [32768 - v for v in vals]
    return out


def luma_tx4_cdfs():
    """Cdfs::new(0)'s (TX_4X4, luma) slice as mt_coef_cdfs."""
    g = json.load(open(GOLDEN_TX4))
    c = abi.CoefCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    arr("txb_skip")[...] = np.stack([_icdf([v], 2) for v in g["skip"]])
    for k, row in enumerate(g["base_tok"]):
        arr("base_tok")[k] = _icdf(row, 4)
    for k, row in enumerate(g["br_tok"]):
        arr("br_tok")[k] = _icdf(row, 4)
    arr("eob_base")[...] = np.stack([_icdf(r, 3) for r in g["eob_base"]])
    arr("eob_hi")[...] = np.stack([_icdf([v], 2) for v in g["eob_hi"]])
    arr("dc_sign")[...] = np.stack([_icdf([v], 2) for v in g["dc_sign"]])
    arr("eob_bin")[...] = _icdf(g["eob_bin"], 11)
    arr("eob_bin_1d")[...] = _icdf(g["eob_bin_1d"], 11)
    for m, row in enumerate(g["txtp"]):
        arr("txtp")[m] = _icdf(row, 16)
    return c


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 13)
    return src, rec


def test_luma_bits_1d_4x4_terms(oracle_lib):
    """luma_bits_1d_4x4 (lossy_state.rs:1010-1143): DC-only blocks cost txb_skip
    0 (context 0), the txtp4 symbol 2 / 3, eob_pt bin 0 of eob_bin_16_l1d,
    eob_base[0] and the DC sign; the eob-coefficient context thresholds are 2
    and 4."""
    c = luma_tx4_cdfs()
    cost = oracle_lib.cdf_cost
    z = np.zeros(16, np.int32)
    assert oracle_lib.luma_bits_1d(z, 4, False, c, 0, 3) == cost(np.array(c.txb_skip[0]), 1)
    for vertical in (True, False):
        cf = z.copy()
        cf[0] = -2
        want = np.float32(cost(np.array(c.txb_skip[0]), 0)) + np.float32(cost(np.array(c.txtp[5]), 2 if vertical else 3))
        want = np.float32(want + np.float32(cost(np.array(c.eob_bin_1d), 0)))
        want = np.float32(want + np.float32(cost(np.array(c.eob_base[0]), 1)))
        want = np.float32(want + np.float32(cost(np.array(c.dc_sign[1]), 1)))
        assert oracle_lib.luma_bits_1d(cf, 4, vertical, c, 1, 5) == want


def _compose(oracle_lib, src, rec, prm, q, qm, c, jb):
    """split16_depth2_try composed from the oracle's primitives."""
    rec = rec.copy()
    px, py = int(jb["px"]), int(jb["py"])
    have_tr, have_bl = bool(jb["flags"] & abi.CAND_HAVE_TR), bool(jb["flags"] & abi.CAND_HAVE_BL)
    ft = bool(jb["flags"] & abi.CAND_FILTER_TYPE)
    mode, delta = int(jb["mode"]), int(jb["angle_delta"])
    scan = oracle_lib.default_scan(4)
    f32 = np.float32
    sse, bits, cf16, types = 0, f32(0), [], []
    rd = lambda d, b: f32(f32(d) + f32(f32(prm.rd_lambda) * f32(b)))
    for j in range(4):
        for i in range(4):
            bx, by = px + 4 * i, py + 4 * j
            tr = (py > 0 and (i < 3 or have_tr)) if j == 0 else i < 3
            bl = (px > 0 and (j < 3 or have_bl)) if i == 0 else False
            pred = oracle_lib.intra_predict(rec, bx, by, 4, 4, mode, delta, tr, bl, ft).ravel()
            resid = src[by:by + 4, bx:bx + 4].astype(np.int32).ravel() - pred
            s = (int(jb["a_coef"][i]) >> 6) - 1 + (int(jb["l_coef"][j]) >> 6) - 1
            ds = int(s != 0) + int(s > 0)

            def trial(t):
                cf, tf = oracle_lib.fwd_txfm_quant(resid, t, q, qm)
                if t in (abi.TX_DCT_DCT, abi.TX_ADST_ADST):
                    cf = oracle_lib.trellis_optimize(cf, tf, float(q.dc_q), float(q.ac_q), scan, prm.trellis_lambda0)
                rr = oracle_lib.inv_txfm_dequant(cf, t, q, qm)
                d = int(oracle_lib.sse_recon(src, prm.frame_w, prm.frame_h, [(bx, by)], pred, rr, 4, 4)[0])
                return cf, rr, d

            cf, rr, d = trial(abi.TX_DCT_DCT)
            dct_sse = d
            b = f32(oracle_lib.real_block_bits_bounded(cf, scan, 4, 4, c, 0, ds, mode, abi.TX_DCT_DCT, INF))
            best = (cf, rr, d, b, abi.TX_DCT_DCT)
            for t in (abi.TX_ADST_ADST, abi.TX_IDTX, abi.TX_V_DCT, abi.TX_H_DCT):
                acf, arr_, asse = trial(t)
                best_rd = rd(best[2], best[3])
                if t in (abi.TX_V_DCT, abi.TX_H_DCT):
                    ab = f32(oracle_lib.luma_bits_1d(acf, 4, t == abi.TX_V_DCT, c, ds, mode))
                else:
                    bound = float(f32(f32(best_rd - f32(asse)) / f32(prm.rd_lambda)))
                    ab = f32(oracle_lib.real_block_bits_bounded(acf, scan, 4, 4, c, 0, ds, mode, t, bound))
                if asse <= dct_sse + (dct_sse >> prm.tx_guard_shift) and rd(asse, ab) < best_rd:
                    best = (acf, arr_, asse, ab, t)
            sse += best[2]
            bits = f32(bits + best[3])
            types.append(best[4])
            cf16.append(best[0])
            rec[by:by + 4, bx:bx + 4] = np.clip(pred.reshape(4, 4) + best[1].reshape(4, 4), 0, 255)
    return sse, bits, np.concatenate(cf16), rec[py:py + 16, px:px + 16], types


def test_depth2_oracle_glue_matches_composition(oracle_lib):
    import maroontree_b200 as mt

    src, rec = _frame(64, 48, 31)
    q = oracle_lib.quant_new(80, 8, 15)
    c = luma_tx4_cdfs()
    prm = mt.split16_params(64, 48, trellis_lambda0=0.05, rd_lambda=22.0, tx_guard_shift=4)
    jobs = synth.split16_jobs(64, 48, (abi.DC_PRED, abi.V_PRED, abi.D157_PRED, abi.SMOOTH_H_PRED, abi.PAETH_PRED),
                              deltas=(0, -3), seed=6)
    res, cf, recs = oracle_lib.split16_depth2(src, rec, prm, q, None, c, jobs)
    seen = set()
    for i, jb in enumerate(jobs):
        sse, bits, cf16, r16, types = _compose(oracle_lib, src, rec, prm, q, None, c, jb)
        assert res["sse"][i] == sse and np.float32(res["bits"][i]) == bits, i
        assert list(res["tx_types"][i]) == types, i
        assert np.array_equal(cf[i], cf16) and np.array_equal(recs[i], r16), i
        seen.update(types)
    assert len(seen) >= 3, seen


def _setup(oracle_lib, w, h, seed, qidx, qm_level, modes=range(13), deltas=(0,)):
    src, rec = _frame(w, h, seed)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 4) if qm_level < 15 else None
    jobs = synth.split16_jobs(w, h, modes, deltas, seed=seed)
    return src, rec, q, qm, jobs


def _check(mt_lib, oracle_lib, src, rec, prm, q, qm, c, jobs):
    res, cf, recs = mt_lib.split16_depth2(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True,
                                         want_rec=True)
    want, wcf, wrec = oracle_lib.split16_depth2(src, rec, prm, q, qm, c, jobs, threads=8)
    bad = (res.view(np.uint8).reshape(len(jobs), -1) != want.view(np.uint8).reshape(len(jobs), -1)).any(axis=1)
    assert not bad.any(), np.nonzero(bad)[0][:5]
    assert np.array_equal(cf, wcf)
    assert np.array_equal(recs, wrec)
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,cdfs", [(70, 6, 0.0, "luma"), (116, 15, 1.0, "luma"),
                                                      (30, 3, 0.75, "synthetic"), (200, 8, 0.0, "synthetic")])
def test_depth2_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, cdfs):
    import maroontree_b200 as mt

    src, rec, q, qm, jobs = _setup(oracle_lib, 160, 96, qidx, qidx, qm_level, deltas=(-2, 0, 3))
    c = luma_tx4_cdfs() if cdfs == "luma" else synth.synthetic_cdfs(qidx + 2, n_eob_bins=5)
    prm = mt.split16_params(160, 96, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, wsse_scale=wsse,
                            tx_guard_shift=4 if qidx != 116 else 5)
    res = _check(mt_lib, oracle_lib, src, rec, prm, q, qm, c, jobs)
    assert len(np.unique(res["tx_types"])) >= 3


@pytest.mark.gpu
def test_depth2_skip_bits_vis_and_rejects(mt_lib, oracle_lib, cuda):
    import maroontree_b200 as mt

    src, rec, q, qm, jobs = _setup(oracle_lib, 96, 64, 12, 90, 6, modes=(0, 2, 4, 10, 12))
    prm = mt.split16_params(96, 64, trellis_lambda0=0.05, rd_lambda=30.0, tx_guard_shift=5, wsse_scale=1.0,
                            skip_bits=[(2.5, 0.25)] + [(0.0, 0.0)] * 12, vis=(90, 61))
    jobs = jobs.copy()
    jobs["py"][2] = 56  # crosses the bottom edge: rejected
    jobs["angle_delta"][4] = -1  # a delta on DC: rejected
    res = _check(mt_lib, oracle_lib, src, rec, prm, q, qm, luma_tx4_cdfs(), jobs)
    assert (res["tx_types"][2] == 255).all() and (res["tx_types"][4] == 255).all()


def _compose4(oracle_lib, src, rec, prm, q, qm, c, jb):
    """split4tx_try (src/coder/block8.rs:157-286) composed from the oracle's primitives."""
    rec = rec.copy()
    px, py = int(jb["px"]), int(jb["py"])
    have_tr, have_bl = bool(jb["flags"] & abi.CAND_HAVE_TR), bool(jb["flags"] & abi.CAND_HAVE_BL)
    ft = bool(jb["flags"] & abi.CAND_FILTER_TYPE)
    mode, delta = int(jb["mode"]), int(jb["angle_delta"])
    scan = oracle_lib.default_scan(4)
    f32 = np.float32
    rd = lambda d, b: f32(f32(d) + f32(f32(prm.rd_lambda) * f32(b)))
    sse, bits, cf4, types = 0, f32(0), [], []
    for qi, (sx, sy) in enumerate(((0, 0), (4, 0), (0, 4), (4, 4))):
        bx, by = px + sx, py + sy
        tr, bl = [(py > 0, px > 0), (have_tr, False), (True, have_bl), (False, False)][qi]
        pred = oracle_lib.intra_predict(rec, bx, by, 4, 4, mode, delta, tr, bl, ft).ravel()
        resid = src[by:by + 4, bx:bx + 4].astype(np.int32).ravel() - pred
        s = (int(jb["a_coef"][sx // 4]) >> 6) - 1 + (int(jb["l_coef"][sy // 4]) >> 6) - 1
        ds = int(s != 0) + int(s > 0)
        best = None
        for t in (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX):
            cf, tf = oracle_lib.fwd_txfm_quant(resid, t, q, qm)
            if t != abi.TX_IDTX:
                cf = oracle_lib.trellis_optimize(cf, tf, float(q.dc_q), float(q.ac_q), scan, prm.trellis_lambda0)
            rr = oracle_lib.inv_txfm_dequant(cf, t, q, qm)
            d = int(oracle_lib.sse_recon(src, prm.frame_w, prm.frame_h, [(bx, by)], pred, rr, 4, 4)[0])
            if best is None:
                dct_sse = d
                b = f32(oracle_lib.real_block_bits_bounded(cf, scan, 4, 4, c, 0, ds, mode, t, INF))
                best = (cf, rr, d, b, t)
                continue
            if d > dct_sse + (dct_sse >> prm.tx_guard_shift):
                continue
            best_rd = rd(best[2], best[3])
            bound = float(f32(f32(best_rd - f32(d)) / f32(prm.rd_lambda)))
            b = f32(oracle_lib.real_block_bits_bounded(cf, scan, 4, 4, c, 0, ds, mode, t, bound))
            if rd(d, b) < best_rd:
                best = (cf, rr, d, b, t)
        sse += best[2]
        bits = f32(bits + best[3])
        types.append(best[4])
        cf4.append(best[0])
        rec[by:by + 4, bx:bx + 4] = np.clip(pred.reshape(4, 4) + best[1].reshape(4, 4), 0, 255)
    return sse, bits, np.concatenate(cf4), rec[py:py + 8, px:px + 8], types


def test_split4tx_oracle_glue_matches_composition(oracle_lib):
    import maroontree_b200 as mt

    src, rec = _frame(48, 32, 41)
    q = oracle_lib.quant_new(80, 8, 15)
    c = luma_tx4_cdfs()
    prm = mt.split16_params(48, 32, trellis_lambda0=0.05, rd_lambda=22.0, tx_guard_shift=4)
    jobs = synth.split16_jobs(48, 32, (abi.DC_PRED, abi.H_PRED, abi.D45_PRED, abi.SMOOTH_PRED), deltas=(0, 2),
                              seed=8, n=8)
    res, cf, recs = oracle_lib.split4tx(src, rec, prm, q, None, c, jobs)
    seen = set()
    for i, jb in enumerate(jobs):
        sse, bits, cf4, r8, types = _compose4(oracle_lib, src, rec, prm, q, None, c, jb)
        assert res["sse"][i] == sse and np.float32(res["bits"][i]) == bits, i
        assert list(res["tx_types"][i]) == types, i
        assert np.array_equal(cf[i], cf4) and np.array_equal(recs[i], r8), i
        seen.update(types)
    assert len(seen) >= 2, seen


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse", [(70, 6, 0.0), (116, 15, 1.0), (30, 3, 0.75)])
def test_split4tx_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    src, rec = _frame(160, 96, qidx + 3)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 4) if qm_level < 15 else None
    jobs = synth.split16_jobs(160, 96, range(13), deltas=(-1, 0, 2), seed=qidx, n=8)
    jobs["px"][5] = 156  # crosses the right edge: rejected
    c = luma_tx4_cdfs()
    prm = mt.split16_params(160, 96, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, wsse_scale=wsse,
                            tx_guard_shift=4, skip_bits=[(1.5, 0.5)] + [(0.0, 0.0)] * 12, vis=(157, 93))
    res, cf, recs = mt_lib.split4tx(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True, want_rec=True)
    want, wcf, wrec = oracle_lib.split4tx(src, rec, prm, q, qm, c, jobs)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)
    assert (res["tx_types"][5] == 255).all() and len(np.unique(res["tx_types"])) >= 3
