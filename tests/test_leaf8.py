"""The 8x8 leaf's luma search (pick_block8) and the 16x16 leaf's (pick_luma16):
the Slow mode loop's candidates and the winner's transform-type refinement.

CPU tests pin the oracle's glue against a composition of its primitives (the
candidate's DCT + trellis_optimize_ctx + sse_recon + luma_bits + syntax bits,
and the refinement's gate sequence), with the default luma TX_8X8 CDFs of the
reference's Cdfs::new(0).  GPU tests compare the CUDA kernels with the oracle
bit for bit."""
import numpy as np
import pytest

from maroontree_b200 import abi, synth
from test_split16 import luma_tx8_cdfs

INF = float("inf")


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 19)
    return src, rec


def _cand(oracle_lib, src, rec, prm, q, qm, c, jb, t, n=8):
    px, py = int(jb["px"]), int(jb["py"])
    fl = int(jb["flags"])
    pred = oracle_lib.intra_predict(rec, px, py, n, n, int(jb["mode"]), int(jb["angle_delta"]), bool(fl & 1),
                                    bool(fl & 2), bool(fl & 4)).ravel()
    resid = src[py:py + n, px:px + n].astype(np.int32).ravel() - pred
    cf, tf = oracle_lib.fwd_txfm_quant(resid, t, q, qm)
    if t in (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST):
        cf = oracle_lib.trellis_optimize_ctx(cf, tf, q, qm, c, int(jb["dcs_ctx"]), prm.trellis_lambda0,
                                             band_tilt=prm.band_tilt, n=n)
    rr = oracle_lib.inv_txfm_dequant(cf, t, q, qm)
    sse = int(oracle_lib.sse_recon(src, prm.frame_w, prm.frame_h, [(px, py)], pred, rr, n, n,
                                   scale=prm.wsse_scale)[0])
    return cf, sse


def test_leaf8_oracle_glue(oracle_lib):
    import maroontree_b200 as mt

    src, rec = _frame(48, 40, 51)
    q = oracle_lib.quant_new(70, 8, 15)
    c = luma_tx8_cdfs()
    prm = mt.split16_params(48, 40, trellis_lambda0=0.05, rd_lambda=18.0, band_tilt=1.9, tx_search=True,
                            tx_guard_shift=5)
    jobs = synth.leaf8_jobs(48, 40, (abi.DC_PRED, abi.V_PRED, abi.D203_PRED, abi.SMOOTH_V_PRED), deltas=(0, 1),
                            seed=3)
    scan = oracle_lib.default_scan(8)
    f32 = np.float32
    rd = lambda d, b: f32(f32(d) + f32(f32(prm.rd_lambda) * f32(b)))
    res, _, _ = oracle_lib.leaf8(src, rec, prm, q, None, c, jobs)
    ref, _, _ = oracle_lib.leaf8(src, rec, prm, q, None, c, jobs, refine=True)
    seen = set()
    for i, jb in enumerate(jobs):
        m, ds = int(jb["mode"]), int(jb["dcs_ctx"])
        cf, sse = _cand(oracle_lib, src, rec, prm, q, None, c, jb, abi.TX_DCT_DCT)
        bits = f32(oracle_lib.real_block_bits_bounded(cf, scan, 8, 8, c, 0, ds, m, abi.TX_DCT_DCT, INF))
        assert res["sse"][i] == sse and f32(res["bits"][i]) == bits
        assert f32(res["cost"][i]) == rd(sse, f32(bits + f32(jb["syntax_bits"])))
        # the refinement's sequence
        dct = (sse, bits)
        best = (sse, bits, abi.TX_DCT_DCT)
        for t in (abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST, abi.TX_IDTX, abi.TX_V_DCT, abi.TX_H_DCT):
            acf, asse = _cand(oracle_lib, src, rec, prm, q, None, c, jb, t)
            base = rd(best[0], best[1])
            if t in (abi.TX_V_DCT, abi.TX_H_DCT):
                ab = f32(oracle_lib.luma_bits_1d(acf, 8, t == abi.TX_V_DCT, c, ds, m))
                gate = asse <= best[0]
            elif t == abi.TX_IDTX:
                ab = f32(oracle_lib.real_block_bits_bounded(acf, scan, 8, 8, c, 0, ds, m, t, INF))
                gate = asse <= best[0] + (best[0] >> prm.tx_guard_shift)
            else:
                bound = float(f32(f32(base - f32(asse)) / f32(prm.rd_lambda)))
                ab = f32(oracle_lib.real_block_bits_bounded(acf, scan, 8, 8, c, 0, ds, m, t, bound))
                gate = asse <= dct[0] + (dct[0] >> prm.tx_guard_shift)
            if gate and rd(asse, ab) < base:
                best = (asse, ab, t)
        assert (ref["sse"][i], f32(ref["bits"][i]), ref["tx_type"][i]) == best, i
        seen.add(best[2])
    assert len(seen) >= 3, seen


@pytest.mark.gpu
@pytest.mark.parametrize("refine", [False, True])
@pytest.mark.parametrize("qidx,qm_level,search,wsse,cdfs", [
    (70, 6, True, 0.0, "luma"), (116, 15, False, 1.0, "luma"), (30, 3, True, 0.75, "synthetic"),
    (200, 8, True, 0.0, "synthetic")])
def test_leaf8_gpu_matches_oracle(mt_lib, oracle_lib, cuda, refine, qidx, qm_level, search, wsse, cdfs):
    import maroontree_b200 as mt

    src, rec = _frame(160, 96, qidx)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8) if qm_level < 15 else None
    c = luma_tx8_cdfs() if cdfs == "luma" else synth.synthetic_cdfs(qidx + 5)
    jobs = synth.leaf8_jobs(160, 96, range(13), deltas=(-2, 0, 3), seed=qidx)
    jobs["px"][7] = 156  # crosses the right edge: rejected
    prm = mt.split16_params(160, 96, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.9,
                            wsse_scale=wsse, tx_search=search, tx_guard_shift=5 if search else 4,
                            skip_bits=[(2.0, 0.3)] + [(0.0, 0.0)] * 12, vis=(157, 94))
    res, cf, recs = mt_lib.leaf8(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, refine=refine, want_cf=True,
                                 want_rec=True)
    want, wcf, wrec = oracle_lib.leaf8(src, rec, prm, q, qm, c, jobs, refine=refine)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)
    assert res["tx_type"][7] == 255
    if refine:
        assert len(np.unique(res["tx_type"])) >= 4


def test_leaf16_oracle_glue(oracle_lib):
    """pick_luma16's candidate (partition_search.rs:4802-4880): DCT_DCT + QM,
    trellis_optimize_ctx at TX_16X16, sse_recon, luma_bits + syntax bits."""
    import maroontree_b200 as mt

    src, rec = _frame(64, 48, 61)
    q = oracle_lib.quant_new(90, 8, 7)
    qm = oracle_lib.qm_row(7, 0, 16)
    c = synth.synthetic_cdfs(12, n_eob_bins=9)
    prm = mt.split16_params(64, 48, trellis_lambda0=0.05, rd_lambda=25.0, band_tilt=2.2)
    jobs = synth.leaf8_jobs(64, 48, (abi.DC_PRED, abi.D113_PRED, abi.SMOOTH_PRED), deltas=(0, -2), seed=9, n=16)
    scan = oracle_lib.default_scan(16)
    f32 = np.float32
    res, cf, recs = oracle_lib.leaf16(src, rec, prm, q, qm, c, jobs)
    for i, jb in enumerate(jobs):
        px, py, fl = int(jb["px"]), int(jb["py"]), int(jb["flags"])
        pred = oracle_lib.intra_predict(rec, px, py, 16, 16, int(jb["mode"]), int(jb["angle_delta"]), bool(fl & 1),
                                        bool(fl & 2), bool(fl & 4)).ravel()
        resid = src[py:py + 16, px:px + 16].astype(np.int32).ravel() - pred
        lv, tf = oracle_lib.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
        lv = oracle_lib.trellis_optimize_ctx(lv, tf, q, qm, c, int(jb["dcs_ctx"]), 0.05, band_tilt=2.2, n=16)
        rr = oracle_lib.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, qm)
        sse = int(oracle_lib.sse_recon(src, 64, 48, [(px, py)], pred, rr, 16, 16)[0])
        bits = f32(oracle_lib.real_block_bits_bounded(lv, scan, 16, 16, c, 0, int(jb["dcs_ctx"]), int(jb["mode"]),
                                                      abi.TX_DCT_DCT, INF))
        assert res["sse"][i] == sse and f32(res["bits"][i]) == bits and np.array_equal(cf[i], lv), i
        assert f32(res["cost"][i]) == f32(f32(sse) + f32(f32(25.0) * f32(bits + f32(jb["syntax_bits"]))))


# The 5-type TX_16X16 intra set's symbol of each MT_TX_* (cost.rs:101-108).
TX16_SYM = {abi.TX_IDTX: 0, abi.TX_DCT_DCT: 1, abi.TX_ADST_ADST: 2, abi.TX_ADST_DCT: 3, abi.TX_DCT_ADST: 4}


def test_leaf16_refine_oracle_glue(oracle_lib):
    """pick_luma16's winner refinement (partition_search.rs:5252-5474):
    ADST_ADST with the rate bounded by the DCT's rd cost; ADST_DCT / DCT_ADST
    priced unbounded against the running winner, gated on the DCT's SSE;
    IDTX untrellised within tx_guard of the winner's SSE; the tx-type symbols
    of the 5-type set; no V / H."""
    import maroontree_b200 as mt

    src, rec = _frame(64, 48, 71)
    q = oracle_lib.quant_new(60, 8, 15)
    c = synth.synthetic_cdfs(21, n_eob_bins=9)
    prm = mt.split16_params(64, 48, trellis_lambda0=0.05, rd_lambda=14.0, band_tilt=1.9, tx_search=True,
                            tx_guard_shift=4)
    jobs = synth.leaf8_jobs(64, 48, (abi.DC_PRED, abi.H_PRED, abi.D157_PRED, abi.SMOOTH_H_PRED, abi.PAETH_PRED),
                            deltas=(0, 2), seed=5, n=16)
    scan = oracle_lib.default_scan(16)
    f32 = np.float32
    rd = lambda d, b: f32(f32(d) + f32(f32(prm.rd_lambda) * f32(b)))
    bits = lambda cf, t, m, ds, bound: f32(oracle_lib.real_block_bits_bounded(cf, scan, 16, 16, c, 0, ds, m,
                                                                             TX16_SYM[t], bound))
    ref, rcf, _ = oracle_lib.leaf16(src, rec, prm, q, None, c, jobs, refine=True)
    seen = set()
    for i, jb in enumerate(jobs):
        m, ds = int(jb["mode"]), int(jb["dcs_ctx"])
        cf, sse = _cand(oracle_lib, src, rec, prm, q, None, c, jb, abi.TX_DCT_DCT, n=16)
        dct = (sse, bits(cf, abi.TX_DCT_DCT, m, ds, INF))
        best = dct + (abi.TX_DCT_DCT, cf)
        guard = lambda d: d + (d >> prm.tx_guard_shift)
        for t in (abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST, abi.TX_IDTX):
            acf, asse = _cand(oracle_lib, src, rec, prm, q, None, c, jb, t, n=16)
            base = rd(best[0], best[1])
            if t == abi.TX_ADST_ADST:
                ab = bits(acf, t, m, ds, float(f32(f32(base - f32(asse)) / f32(prm.rd_lambda))))
                gate = asse <= guard(dct[0])
            elif t == abi.TX_IDTX:
                ab = bits(acf, t, m, ds, INF)
                gate = asse <= guard(best[0])
            else:
                ab = bits(acf, t, m, ds, INF)
                gate = asse <= guard(dct[0])
            if gate and rd(asse, ab) < base:
                best = (asse, ab, t, acf)
        assert (ref["sse"][i], f32(ref["bits"][i]), ref["tx_type"][i]) == best[:3], i
        assert np.array_equal(rcf[i], best[3])
        seen.add(best[2])
    assert len(seen) >= 3, seen


@pytest.mark.gpu
@pytest.mark.parametrize("refine", [False, True])
@pytest.mark.parametrize("qidx,qm_level,wsse", [(70, 6, 0.0), (116, 15, 1.0), (30, 3, 0.75)])
def test_leaf16_gpu_matches_oracle(mt_lib, oracle_lib, cuda, refine, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    src, rec = _frame(160, 96, qidx + 1)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 16) if qm_level < 15 else None
    c = synth.synthetic_cdfs(qidx + 7, n_eob_bins=9)
    jobs = synth.leaf8_jobs(160, 96, range(13), deltas=(-1, 0, 3), seed=qidx, n=16)
    jobs["py"][4] = 88  # crosses the bottom edge: rejected
    prm = mt.split16_params(160, 96, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.9,
                            wsse_scale=wsse, tx_guard_shift=4, skip_bits=[(2.0, 0.3)] + [(0.0, 0.0)] * 12,
                            vis=(155, 91))
    res, cf, recs = mt_lib.leaf16(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, refine=refine, want_cf=True,
                                  want_rec=True)
    want, wcf, wrec = oracle_lib.leaf16(src, rec, prm, q, qm, c, jobs, refine=refine)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)
    assert res["tx_type"][4] == 255
    if refine:
        assert len(np.unique(res["tx_type"])) >= 4
