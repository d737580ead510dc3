"""The 16x16 leaf's TX_8X8 split trial (split16_luma_try) and its pieces:
trellis_optimize_ctx, the bounded 2-D rate walk, the 1-D (V_DCT / H_DCT)
rate walk and the coefficient result context.

CPU tests pin the oracle: the reference's own trellis validity test
(src/trellis.rs:1054-1101) restated on the oracle, the exactness of the rate
walk's abort bound, the 1-D walk's DC-only form term by term, and the split
trial's glue (quadrant order, progressive contexts, patch prediction) against
an independent composition of the oracle's primitives.  GPU tests compare the
CUDA kernels with the oracle bit for bit, with the default luma TX_8X8 CDFs of
the reference's Cdfs::new(0) (tests/golden/cdfs_luma_tx8_qctx0.json) and with
synthetic ones."""
import json
import os

import numpy as np
import pytest

from maroontree_b200 import abi, synth

GOLDEN_LUMA = os.path.join(os.path.dirname(__file__), "golden", "cdfs_luma_tx8_qctx0.json")
INF = float("inf")


def _icdf(vals, width):
    """src/tables.rs:31-35 icdf: 32768 - v per entry, then the terminal 0."""
    out = np.zeros(width, np.uint16)
    out[:len(vals)] = [32768 - v for v in vals]
    return out


def luma_tx8_cdfs():
    """Cdfs::new(0)'s (TX_8X8, luma) slice as mt_coef_cdfs."""
    g = json.load(open(GOLDEN_LUMA))
    c = abi.CoefCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    arr("txb_skip")[...] = np.stack([_icdf([v], 2) for v in g["skip"]])
    bt = arr("base_tok")
    for k, row in enumerate(g["base_tok"]):
        bt[k] = _icdf(row, 4)
    br = arr("br_tok")
    for k, row in enumerate(g["br_tok"]):
        br[k] = _icdf(row, 4)
    arr("eob_base")[...] = np.stack([_icdf(r, 3) for r in g["eob_base"]])
    arr("eob_hi")[...] = np.stack([_icdf([v], 2) for v in g["eob_hi"]])
    arr("dc_sign")[...] = np.stack([_icdf([v], 2) for v in g["dc_sign"]])
    arr("eob_bin")[...] = _icdf(g["eob_bin_64"], 11)
    arr("eob_bin_1d")[...] = _icdf(g["eob_bin_64_1d"], 11)
    tx = arr("txtp")
    for m, row in enumerate(g["txtp"]):
        tx[m] = _icdf(row, 16)
    return c


def _xorshift(seed):
    state = [seed]

    def nxt():
        s = state[0]
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        state[0] = s
        return s

    return nxt


def random_block(rng, n):
    """The reference test's generator (src/trellis.rs:1044-1053): 1..40 random
    positions with |target| in [0, 6) and the level its rounding."""
    tf = np.zeros(n * n, np.float32)
    cf = np.zeros(n * n, np.int32)
    for _ in range(1 + rng() % 40):
        rc = rng() % (n * n)
        mag = np.float32(rng() % 6) + np.float32(rng() / 18446744073709551615.0)
        sign = 1.0 if rng() & 1 == 0 else -1.0
        tf[rc] = np.float32(sign * mag)
        cf[rc] = int(sign * np.floor(mag + 0.5))
    return tf, cf


@pytest.mark.parametrize("n,cdfs", [(8, "luma"), (16, "synthetic")])
def test_trellis_ctx_output_is_valid(oracle_lib, n, cdfs):
    """trellis.rs:1054-1101 trellis_output_is_valid: zero past the new EOB, no
    magnitude raised, no sign flipped (dc_q 200, ac_q 220, lambda0 0.05)."""
    c = luma_tx8_cdfs() if cdfs == "luma" else synth.synthetic_cdfs(5, n_eob_bins=9)
    q = oracle_lib.quant_new(100, 8, 15)
    q.dc_q, q.ac_q = 200, 220
    scan = oracle_lib.default_scan(n)
    rng = _xorshift(0x2545F4914F6CDD1D)
    changed = 0
    for _ in range(400):
        tf, cf = random_block(rng, n)
        opt = oracle_lib.trellis_optimize_ctx(cf, tf, q, None, c, 0, 0.05, n=n)
        nz = np.nonzero(opt[scan])[0]
        if len(nz):
            assert not opt[scan[nz[-1] + 1:]].any()
        assert np.all(np.abs(opt) <= np.abs(cf))
        assert np.all(np.sign(opt[opt != 0]) == np.sign(cf[opt != 0]))
        changed += int((opt != cf).any())
    assert changed > 0


def test_trellis_ctx_noop_cases(oracle_lib):
    c = luma_tx8_cdfs()
    q = oracle_lib.quant_new(70, 8, 6)
    rng = _xorshift(7)
    tf, cf = random_block(rng, 8)
    assert np.array_equal(oracle_lib.trellis_optimize_ctx(cf, tf, q, None, c, 1, 0.0), cf)
    z = np.zeros(64, np.int32)
    assert not oracle_lib.trellis_optimize_ctx(z, tf, q, None, c, 1, 0.05).any()


def test_bounded_walk_abort_is_exact(oracle_lib):
    """real_block_bits_bounded (rate.rs:149-291): +inf bound is the plain walk;
    a finite return equals it; an abort only happens when the true rate is
    above the bound."""
    c = luma_tx8_cdfs()
    scan = oracle_lib.default_scan(8)
    rng = np.random.default_rng(3)
    aborted = 0
    for k in range(300):
        cf = np.zeros(64, np.int32)
        nnz = rng.integers(1, 40)
        cf[rng.integers(0, 64, nnz)] = rng.integers(-20, 21, nnz)
        full = oracle_lib.real_block_bits_wh(cf, scan, 8, 8, c, k % 7, k % 3, k % 13, 1)
        assert oracle_lib.real_block_bits_bounded(cf, scan, 8, 8, c, k % 7, k % 3, k % 13, 1, INF) == full
        bound = float(np.float32(full * rng.uniform(0.2, 1.2)))
        b = oracle_lib.real_block_bits_bounded(cf, scan, 8, 8, c, k % 7, k % 3, k % 13, 1, bound)
        if b == INF:
            aborted += 1
            assert full > bound
        else:
            assert b == full
    assert aborted > 0


def test_luma_bits_1d_terms(oracle_lib):
    """luma_bits_1d_8x8 (lossy_state.rs:876-1008): the all-zero block is the
    txb_skip(ctx 0) = 1 symbol; a DC-only block adds txb_skip 0, the V/H
    tx-type symbol, eob_pt bin 0 of the 1-D CDF, eob_base[0] and the DC sign
    (plus the base-range ladder from 3)."""
    c = luma_tx8_cdfs()
    cost = oracle_lib.cdf_cost
    z = np.zeros(64, np.int32)
    assert oracle_lib.luma_bits_1d(z, 8, True, c, 1, 0) == cost(np.array(c.txb_skip[0]), 1)
    for vertical in (True, False):
        for dc, mode, dcs in ((1, 0, 0), (-2, 4, 2), (2, 9, 1)):
            cf = z.copy()
            cf[0] = dc
            want = np.float32(cost(np.array(c.txb_skip[0]), 0)) + np.float32(
                cost(np.array(c.txtp[mode]), 2 if vertical else 3))
            want = np.float32(want + np.float32(cost(np.array(c.eob_bin_1d), 0)))
            want = np.float32(want + np.float32(cost(np.array(c.eob_base[0]), abs(dc) - 1)))
            want = np.float32(want + np.float32(cost(np.array(c.dc_sign[dcs]), int(dc < 0))))
            assert oracle_lib.luma_bits_1d(cf, 8, vertical, c, dcs, mode) == want
    # V and H read the coefficients in transposed order: a coefficient in row 0
    # (rc = x * 8) is early in H's walk and late in V's.
    cf = z.copy()
    cf[8 * 5] = 3
    assert oracle_lib.luma_bits_1d(cf, 8, True, c, 0, 0) != oracle_lib.luma_bits_1d(cf, 8, False, c, 0, 0)


def test_coef_res_ctx_values(oracle_lib):
    z = np.zeros(64, np.int32)
    assert oracle_lib.coef_res_ctx(z) == 0x40
    cf = z.copy()
    cf[0], cf[1], cf[8] = -3, 2, 70
    assert oracle_lib.coef_res_ctx(cf) == 63
    cf[0] = 5
    assert oracle_lib.coef_res_ctx(cf) == (63 | 0x80)
    cf = z.copy()
    cf[9] = 4
    assert oracle_lib.coef_res_ctx(cf) == (4 | 0x40)


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 11)
    return src, rec


def _skip_ctx(a, l):
    tbl = [[1, 2, 2, 2, 3], [2, 4, 4, 4, 5], [2, 4, 4, 4, 5], [2, 4, 4, 4, 5], [3, 5, 5, 5, 6]]
    la, ll = (int(a[0]) | int(a[1])) & 0x3F, (int(l[0]) | int(l[1])) & 0x3F
    return tbl[min(la, 4)][min(ll, 4)]


def _dcs(a, l):
    s = sum((int(v) >> 6) - 1 for v in (*a[:2], *l[:2]))
    return (s != 0) + (s > 0)


def _compose_dct_only(oracle_lib, src, rec, prm, q, qm, c, jb):
    """split16_luma_try without the type search and without trellis, composed
    from the oracle's primitives: raster quadrants, each predicted from the
    reconstruction with the earlier quadrants written in, priced in the
    progressive contexts."""
    rec = rec.copy()
    px, py = int(jb["px"]), int(jb["py"])
    a, l = list(jb["a_coef"]), list(jb["l_coef"])
    have_tr, have_bl = bool(jb["flags"] & abi.CAND_HAVE_TR), bool(jb["flags"] & abi.CAND_HAVE_BL)
    ft = bool(jb["flags"] & abi.CAND_FILTER_TYPE)
    scan = oracle_lib.default_scan(8)
    sse, bits, cf4 = 0, np.float32(0), []
    for qi, (sx, sy) in enumerate(((0, 0), (8, 0), (0, 8), (8, 8))):
        bx, by = px + sx, py + sy
        tr, bl = [(py > 0, px > 0), (have_tr, False), (True, have_bl), (False, False)][qi]
        pred = oracle_lib.intra_predict(rec, bx, by, 8, 8, int(jb["mode"]), int(jb["angle_delta"]), tr, bl, ft)
        resid = src[by:by + 8, bx:bx + 8].astype(np.int32).ravel() - pred.ravel()
        cf, _ = oracle_lib.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
        rr = oracle_lib.inv_txfm_dequant(cf, abi.TX_DCT_DCT, q, qm)
        ax, ly = sx // 4, sy // 4
        sk, ds = _skip_ctx(a[ax:ax + 2], l[ly:ly + 2]), _dcs(a[ax:ax + 2], l[ly:ly + 2])
        sse += int(oracle_lib.sse_recon(src, prm.frame_w, prm.frame_h, [(bx, by)], pred.ravel(), rr.ravel(), 8, 8)[0])
        bits = np.float32(bits + np.float32(oracle_lib.real_block_bits_bounded(cf, scan, 8, 8, c, sk, ds,
                                                                                int(jb["mode"]), 1, INF)))
        res = oracle_lib.coef_res_ctx(cf)
        a[ax] = a[ax + 1] = res
        l[ly] = l[ly + 1] = res
        rec[by:by + 8, bx:bx + 8] = np.clip(pred.reshape(8, 8) + rr.reshape(8, 8), 0, 255)
        cf4.append(cf)
    return sse, bits, np.concatenate(cf4), rec[py:py + 16, px:px + 16]


def test_split16_oracle_glue_matches_composition(oracle_lib):
    import maroontree_b200 as mt

    src, rec = _frame(64, 48, 21)
    q = oracle_lib.quant_new(90, 8, 15)
    c = luma_tx8_cdfs()
    prm = mt.split16_params(64, 48, trellis_lambda0=0.0, rd_lambda=25.0)
    jobs = synth.split16_jobs(64, 48, (abi.DC_PRED, abi.D45_PRED, abi.D135_PRED, abi.SMOOTH_PRED, abi.PAETH_PRED),
                              deltas=(0, 2), seed=4)
    res, cf, recs = oracle_lib.split16_luma(src, rec, prm, q, None, c, jobs)
    assert (res["tx_types"] == abi.TX_DCT_DCT).all()
    for i, jb in enumerate(jobs):
        sse, bits, cf4, r16 = _compose_dct_only(oracle_lib, src, rec, prm, q, None, c, jb)
        assert res["sse"][i] == sse and np.float32(res["bits"][i]) == bits, i
        assert np.array_equal(cf[i], cf4) and np.array_equal(recs[i], r16), i


def test_split16_oracle_type_search_and_trellis(oracle_lib):
    """With the type search every quadrant type is one of the seven; the
    trellised result never prices above the untrellised DCT-only one by more
    than what the trial can trade, and the search changes some decisions."""
    import maroontree_b200 as mt

    src, rec = _frame(96, 64, 22)
    q = oracle_lib.quant_new(60, 8, 6)
    qm = oracle_lib.qm_row(6, 0, 8)
    c = luma_tx8_cdfs()
    jobs = synth.split16_jobs(96, 64, range(13), seed=5)
    base = mt.split16_params(96, 64, trellis_lambda0=0.05, rd_lambda=20.0, band_tilt=1.9)
    srch = mt.split16_params(96, 64, trellis_lambda0=0.05, rd_lambda=20.0, band_tilt=1.9, tx_search=True,
                             tx_guard_shift=5)
    r0, _, _ = oracle_lib.split16_luma(src, rec, base, q, qm, c, jobs, threads=4)
    r1, _, _ = oracle_lib.split16_luma(src, rec, srch, q, qm, c, jobs, threads=4)
    assert (r0["tx_types"] == abi.TX_DCT_DCT).all()
    assert np.isin(r1["tx_types"], np.arange(7)).all()
    assert (r1["tx_types"] != abi.TX_DCT_DCT).any()
    # quadrant 0 sees the same contexts and prediction in both runs, so the
    # search can only lower its rd cost
    assert (r1["tx_types"][:, 0] != abi.TX_DCT_DCT).any()


# ---------------------------------------------------------------------------
# GPU parity


def _setup(oracle_lib, w, h, seed, qidx, qm_level, modes=range(13), deltas=(0,)):
    src, rec = _frame(w, h, seed)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8) if qm_level < 15 else None
    jobs = synth.split16_jobs(w, h, modes, deltas, seed=seed)
    return src, rec, q, qm, jobs


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,tilt,cdfs", [(70, 6, 1.9, "luma"), (116, 15, 0.0, "luma"),
                                                      (30, 3, 2.6, "synthetic"), (200, 8, 0.0, "synthetic")])
def test_trellis_ctx_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, tilt, cdfs):
    torch = cuda
    c = luma_tx8_cdfs() if cdfs == "luma" else synth.synthetic_cdfs(qidx, n_eob_bins=7)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8) if qm_level < 15 else None
    rng = np.random.default_rng(qidx)
    n = 3000
    resid = rng.integers(-60, 61, size=(n, 64)).astype(np.int32)
    resid[: n // 3] //= 8  # some sparse blocks
    types = rng.choice([abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_ADST_DCT, abi.TX_DCT_ADST], size=n)
    lv = np.zeros((n, 64), np.int32)
    tf = np.zeros((n, 64), np.float32)
    for i in range(n):
        lv[i], tf[i] = oracle_lib.fwd_txfm_quant(resid[i], int(types[i]), q, qm)
    dcs = rng.integers(0, 3, size=n).astype(np.uint8)
    want = np.stack([oracle_lib.trellis_optimize_ctx(lv[i], tf[i], q, qm, c, int(dcs[i]), 0.05, band_tilt=tilt)
                     for i in range(n)])
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_lv, d_tf, d_dcs = t(lv), t(tf), t(dcs)
    d_costs = t(np.frombuffer(bytes(mt_lib.coef_costs(c)), np.uint8))
    d_qm = t(qm) if qm is not None else None
    mt_lib.trellis_optimize_ctx_device(d_lv, d_tf, d_dcs, n, q, d_qm, d_costs, 0.05, band_tilt=tilt)
    torch.cuda.synchronize()
    got = d_lv.cpu().numpy().view(np.int32).reshape(n, 64)
    assert (want != lv).any()
    bad = np.nonzero((got != want).any(axis=1))[0]
    assert len(bad) == 0, (len(bad), bad[:5])


def _check_split(mt_lib, oracle_lib, src, rec, prm, q, qm, c, jobs):
    res, cf, recs = mt_lib.split16_luma(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True, want_rec=True)
    want, wcf, wrec = oracle_lib.split16_luma(src, rec, prm, q, qm, c, jobs, threads=8)
    assert res.tobytes() == want.tobytes(), np.nonzero(
        (res.view(np.uint8).reshape(len(jobs), -1) != want.view(np.uint8).reshape(len(jobs), -1)).any(axis=1))[0][:5]
    assert np.array_equal(cf, wcf)
    assert np.array_equal(recs, wrec)
    return res


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,search,wsse,cdfs", [
    (70, 6, False, 0.0, "luma"), (70, 6, True, 0.0, "luma"), (116, 15, True, 1.0, "luma"),
    (30, 3, True, 0.75, "synthetic"), (200, 8, False, 0.0, "synthetic")])
def test_split16_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, search, wsse, cdfs):
    import maroontree_b200 as mt

    src, rec, q, qm, jobs = _setup(oracle_lib, 160, 96, qidx, qidx, qm_level, deltas=(-2, 0, 3))
    c = luma_tx8_cdfs() if cdfs == "luma" else synth.synthetic_cdfs(qidx + 1, n_eob_bins=7)
    prm = mt.split16_params(160, 96, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.9 if search else 0.0,
                            wsse_scale=wsse, tx_search=search, tx_guard_shift=5 if search else 4)
    res = _check_split(mt_lib, oracle_lib, src, rec, prm, q, qm, c, jobs)
    if search:
        assert (res["tx_types"] != abi.TX_DCT_DCT).any()


@pytest.mark.gpu
def test_split16_skip_bits_vis_and_rejects(mt_lib, oracle_lib, cuda):
    import maroontree_b200 as mt

    src, rec, q, qm, jobs = _setup(oracle_lib, 96, 64, 9, 90, 6, modes=(0, 1, 3, 9, 12))
    rng = np.random.default_rng(1)
    skip = [(float(np.float32(a)), float(np.float32(b))) for a, b in rng.uniform(0.1, 6.0, size=(13, 2))]
    prm = mt.split16_params(96, 64, trellis_lambda0=0.05, rd_lambda=30.0, band_tilt=1.2, tx_search=True,
                            tx_guard_shift=5, skip_bits=skip, vis=(90, 58), wsse_scale=1.0)
    jobs = jobs.copy()
    jobs["px"][3] = 88  # crosses the right edge: rejected
    jobs["angle_delta"][5] = 2  # a delta on DC: rejected
    res = _check_split(mt_lib, oracle_lib, src, rec, prm, q, qm, luma_tx8_cdfs(), jobs)
    assert (res["tx_types"][3] == 255).all() and (res["tx_types"][5] == 255).all()
    assert res["sse"][3] == 0 and res["bits"][3] == 0
