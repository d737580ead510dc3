"""The 16x16 leaf's 4:2:0 chroma search (pick_uv16_420,
src/coder/block16.rs:980-1381, shipped tuning: uv16_joint, uv8_joint_k 4,
cfl_alpha_rd_steps 0) and uv_mode_bits (src/coder/lossy_state.rs:1302-1349).

CPU tests pin the pieces the picker adds: the default mode CDFs of the library
equal the reference's arrays (tests/golden/cdfs_default.json), the library's
uv_mode_bits equals the oracle's for every (y mode, uv mode) and CfL alpha
pair, and the oracle's picker equals a step-by-step composition of its own
primitives written here (the DC path, CfL with the closed-form alphas, the
joint SATD shortlist sorted by (score, mode, delta), the early stop after U).
GPU tests compare mt_pick_uv16_420 with the oracle bit for bit: totals,
winners, alphas, levels and reconstruction, on synthetic frames (QM / flat,
wSSE, skip pricing, a cropped displayed window, rejected jobs) and on every
16x16 leaf of the 4:2:0 benchmark frames with their chroma quantisers and
the default chroma CDFs."""
import os

import numpy as np
import pytest

from maroontree_b200 import abi, synth

INF = float("inf")
JOINT = [abi.SMOOTH_V_PRED, abi.PAETH_PRED, abi.SMOOTH_PRED, abi.SMOOTH_H_PRED, abi.V_PRED, abi.H_PRED,
         abi.D135_PRED, abi.D113_PRED, abi.D157_PRED, abi.D45_PRED, abi.D67_PRED, abi.D203_PRED]


def _planes(w, h, seed):
    return synth.planes420(synth.generate_rgb(w, h, seed, sigma=4.0, variant="1080p"), seed)


def test_uv_mode_cdfs_default_equal_reference(mt_lib, oracle_lib):
    assert bytes(mt_lib.uv_mode_cdfs_default()) == bytes(oracle_lib.uv_mode_cdfs())


def test_uv_mode_bits_match_oracle(mt_lib, oracle_lib):
    c = mt_lib.uv_mode_costs(mt_lib.uv_mode_cdfs_default())
    oc = oracle_lib.uv_mode_cdfs()
    f32 = np.float32
    for y in range(13):
        for u in range(13):
            assert f32(mt_lib.uv_mode_bits(c, y, u)) == f32(oracle_lib.uv_mode_bits(oc, y, u)), (y, u)
        for au in range(-16, 17):
            for av in range(-16, 17):
                assert f32(mt_lib.uv_mode_bits(c, y, abi.UV_CFL_PRED, (au, av))) == \
                    f32(oracle_lib.uv_mode_bits(oc, y, abi.UV_CFL_PRED, (au, av))), (y, au, av)
    # both alphas 0 is priced as DC
    assert mt_lib.uv_mode_bits(c, 3, abi.UV_CFL_PRED, (0, 0)) == mt_lib.uv_mode_bits(c, 3, abi.DC_PRED)


def _satd_sad_proxy8(src, pred, vw, vh):
    d = np.where((np.arange(8)[None, :] < vw) & (np.arange(8)[:, None] < vh), src.astype(np.int64) - pred, 0)
    sad = int(np.abs(d).sum())
    satd = 0
    h4 = np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]])
    for ty in (0, 4):
        for tx in (0, 4):
            t = d[ty:ty + 4, tx:tx + 4]
            satd += int(np.abs(h4 @ t @ h4.T).sum())
    return sad + (satd >> 2)


def _glue_one(op, src, rec, prm, uvp, q, qm, cd, mc, jb):
    """pick_uv16_420 of one leaf from the oracle's primitives."""
    f32 = np.float32
    cx, cy = int(jb["px"]) // 2, int(jb["py"]) // 2
    fl = int(jb["flags"])
    tr, bl, ft = bool(fl & 1), bool(fl & 2), bool(fl & 4)
    lam = f32(prm.rd_lambda)
    scan = op.default_scan(8)
    cw, ch = src[1].shape[1], src[1].shape[0]
    vw, vh = min(max(prm.vis_w - cx, 0), 8), min(max(prm.vis_h - cy, 0), 8)
    ctx = []
    for pl in range(2):
        a, l = [int(v) for v in jb["a_coef"][pl]], [int(v) for v in jb["l_coef"][pl]]
        sk = 7 + int(a[0] != 0x40 or a[1] != 0x40) + int(l[0] != 0x40 or l[1] != 0x40)
        s = sum((v >> 6) - 1 for v in a + l)
        ctx.append((sk, int(s != 0) + int(s > 0)))

    def plane(pl, pred, tx, keep_dc):
        s = src[1 + pl][cy:cy + 8, cx:cx + 8].astype(np.int32).ravel()
        resid = s - pred.ravel()
        lv, tf = op.fwd_txfm_quant(resid, tx, q, qm)
        lv = op.trellis_optimize_ctx(lv, tf, q, qm, cd, ctx[pl][1], prm.trellis_lambda0, band_tilt=prm.band_tilt, n=8)
        if keep_dc:
            mean = int(np.trunc(resid.sum() / 64))
            if lv[0] == 0 and abs(mean) >= 8:
                lv[0] = 1 if mean > 0 else -1
        rr = op.inv_txfm_dequant(lv, tx, q, qm)
        sse = int(op.sse_recon(src[1 + pl], prm.vis_w, prm.vis_h, [(cx, cy)], pred.ravel(), rr, 8, 8,
                               scale=prm.wsse_scale)[0])
        bits = op.real_block_bits_bounded(lv, scan, 8, 8, cd, ctx[pl][0], ctx[pl][1], -1, 0, INF)
        return f32(f32(sse) + f32(lam * f32(bits)))

    dc = [int(op.intra_predict(rec[1 + pl], cx, cy, 8, 8, abi.DC_PRED)[0, 0]) for pl in range(2)]
    dc_total = f32(0)
    for pl in range(2):
        dc_total = f32(dc_total + plane(pl, np.full((8, 8), dc[pl]), abi.TX_DCT_DCT, True))
    best, mode, delta = dc_total, abi.DC_PRED, 0
    blk = np.array([(cx, cy, (dc[0], dc[1]))], abi.CFL_BLOCK_DTYPE)
    alpha, ac = op.cfl_alpha(rec[0], src[1], src[2], 1, 1, 8, 8, blk, vis=(prm.vis_w, prm.vis_h))
    body = f32(0)
    for pl in range(2):
        diff = int(alpha[0][pl]) * ac[0]
        mag = (np.abs(diff) + 32) >> 6
        pred = np.clip(dc[pl] + np.where(diff < 0, -mag, mag), 0, 255)
        body = f32(body + plane(pl, pred, abi.TX_DCT_DCT, False))
    cfl_total = f32(f32(body + f32(lam * f32(op.uv_mode_bits(mc, int(jb["y_mode"]), abi.UV_CFL_PRED,
                                                             (int(alpha[0][0]), int(alpha[0][1]))))))
                    - f32(lam * f32(op.uv_mode_bits(mc, int(jb["y_mode"]), abi.DC_PRED))))
    if (alpha[0] != 0).any() and cfl_total < best:
        best, mode = cfl_total, abi.UV_CFL_PRED
    allc = []
    for m in JOINT:
        dir_ = abi.V_PRED <= m <= abi.D67_PRED and uvp.angle_deltas
        for d in (range(-3, 4) if dir_ else (0,)):
            sc = 0
            for pl in range(2):
                pp = op.intra_predict(rec[1 + pl], cx, cy, 8, 8, m, d, tr, bl, ft, fw=cw, fh=ch)
                sc += _satd_sad_proxy8(src[1 + pl][cy:cy + 8, cx:cx + 8], pp, vw, vh)
            allc.append((sc, m, d))
    allc.sort()
    txmap = {abi.PAETH_PRED: abi.TX_ADST_ADST, abi.SMOOTH_PRED: abi.TX_ADST_ADST, abi.D135_PRED: abi.TX_ADST_ADST,
             abi.SMOOTH_V_PRED: abi.TX_ADST_DCT, abi.V_PRED: abi.TX_ADST_DCT, abi.D113_PRED: abi.TX_ADST_DCT,
             abi.D67_PRED: abi.TX_ADST_DCT, abi.SMOOTH_H_PRED: abi.TX_DCT_ADST, abi.H_PRED: abi.TX_DCT_ADST,
             abi.D157_PRED: abi.TX_DCT_ADST, abi.D203_PRED: abi.TX_DCT_ADST}
    adc = np.ctypeslib.as_array(mc.angle_delta)
    for _, m, d in allc[:uvp.joint_k]:
        ad = f32(0)
        if abi.V_PRED <= m <= abi.D67_PRED:
            ad = f32(f32(op.cdf_cost(adc[m - abi.V_PRED], d + 3)) - f32(op.cdf_cost(adc[m - abi.V_PRED], 3)))
        total = f32(lam * f32(f32(op.uv_mode_bits(mc, int(jb["y_mode"]), m)) + ad))
        for pl in range(2):
            pp = op.intra_predict(rec[1 + pl], cx, cy, 8, 8, m, d, tr, bl, ft, fw=cw, fh=ch)
            total = f32(total + plane(pl, pp, txmap.get(m, abi.TX_DCT_DCT), True))
            if pl == 0 and total >= best:
                break
        if total < best:
            best, mode, delta = total, m, d
    return best, dc_total, cfl_total, mode, delta, (int(alpha[0][0]), int(alpha[0][1]))


@pytest.mark.parametrize("qidx,qm_level,wsse", [(90, 6, 1.0), (40, 15, 0.0)])
def test_uv16_oracle_glue(oracle_lib, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    op = oracle_lib
    src, rec = _planes(96, 64, qidx)
    cw, ch = src[1].shape[1], src[1].shape[0]
    q = op.quant_new_chroma(qidx, 0, 0, 8, qm_level)
    qm = op.qm_row(qm_level, 1, 8) if qm_level < 15 else None
    cd = op.default_cdfs(op.qcat(qidx), 8, plane=1)
    mc = op.uv_mode_cdfs()
    prm = mt.split16_params(cw, ch, trellis_lambda0=0.05, rd_lambda=0.2 * qidx + 3, band_tilt=0.4, wsse_scale=wsse,
                            vis=(cw - 3, ch - 1))
    uvp = mt.uv16_params(src[0].shape[1], joint_k=4, angle_deltas=True)
    jobs = synth.uv16_jobs(96, 64, qidx)
    res, _, _ = op.pick_uv16_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs)
    f32 = np.float32
    for i, jb in enumerate(jobs):
        best, dct, cflt, mode, delta, al = _glue_one(op, src, rec, prm, uvp, q, qm, cd, mc, jb)
        r = res[i]
        assert (f32(r["total"]), f32(r["dc_total"]), f32(r["cfl_total"])) == (best, dct, cflt), i
        assert (int(r["uv_mode"]), int(r["angle_delta"]), tuple(int(v) for v in r["cfl_alpha"])) == (mode, delta, al)


def _gpu_case(mt, op, src, rec, prm, uvp, q, qm, qctx, jobs, threads):
    cd = op.default_cdfs(qctx, 8, plane=1)
    mc = op.uv_mode_cdfs()
    costs = mt.coef_costs(mt.coef_cdfs_default(qctx, 8, 8, 1))
    mcost = mt.uv_mode_costs(mt.uv_mode_cdfs_default())
    got = mt.pick_uv16_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, costs, mcost, jobs, want_cf=True,
                           want_rec=True)
    want = op.pick_uv16_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs, threads=threads,
                            want_cf=True, want_rec=True)
    assert got[0].tobytes() == want[0].tobytes()
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    return got[0]


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,skip,joint_k,ad", [
    (70, 6, 1.0, False, 4, True), (116, 15, 0.0, True, 4, True), (30, 3, 0.75, False, 7, False),
    (200, 10, 0.0, False, 1, True)])
def test_uv16_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, skip, joint_k, ad):
    src, rec = _planes(320, 192, qidx + 3)
    cw, ch = src[1].shape[1], src[1].shape[0]
    q = oracle_lib.quant_new_chroma(qidx, 0, 0, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 1, 8) if qm_level < 15 else None
    sb = [(float(np.float32(1.5 + 0.1 * k)), float(np.float32(0.2 + 0.05 * k))) for k in range(13)] if skip else None
    prm = mt_lib.split16_params(cw, ch, trellis_lambda0=0.05, rd_lambda=0.25 * qidx + 2, band_tilt=0.9,
                                wsse_scale=wsse, vis=(cw - 5, ch - 2), skip_bits=sb)
    uvp = mt_lib.uv16_params(src[0].shape[1], joint_k=joint_k, angle_deltas=ad)
    jobs = synth.uv16_jobs(320, 192, qidx)
    jobs = np.concatenate([jobs, jobs[:2]])
    jobs["px"][-2] = 312  # the chroma block leaves the plane: rejected
    jobs["y_mode"][-1] = 13  # not a luma mode: rejected
    res = _gpu_case(mt_lib, oracle_lib, src, rec, prm, uvp, q, qm, oracle_lib.qcat(qidx), jobs,
                    os.cpu_count() or 1)
    assert (res["uv_mode"][-2:] == 255).all() and (res["uv_mode"][:-2] != 255).all()
    # the textured chroma gives every kind of winner: DC, CfL, shortlist modes, angle deltas
    kinds = set(int(m) for m in res["uv_mode"][:-2])
    assert {abi.DC_PRED, abi.UV_CFL_PRED} <= kinds and len(kinds) >= 6, kinds
    if ad:
        assert (res["angle_delta"][:-2] != 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["C2q40", "C2q60", "C2q80"])
def test_uv16_at_config(mt_lib, oracle_lib, cuda, name):
    """Every 16x16 leaf of the 4:2:0 benchmark frames: the frame's chroma
    quantiser (delta 0) and QM level, the chroma CDFs of its q context."""
    import configs

    wl = configs.workload(name)
    src, rec = synth.planes420(wl.rgb, wl.qidx)
    cw, ch = src[1].shape[1], src[1].shape[0]
    q = mt_lib.quant_new_chroma(wl.qidx, 0, 0, 8, wl.qm_uv)
    qm = mt_lib.qm_row(wl.qm_uv, 1, 8) if wl.qm_uv < 15 else None
    prm = mt_lib.split16_params(cw, ch, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                band_tilt=0.0, wsse_scale=1.0, vis=(wl.w // 2, wl.h // 2))
    uvp = mt_lib.uv16_params(src[0].shape[1], joint_k=4, angle_deltas=True)
    jobs = synth.uv16_jobs(wl.w, wl.h, wl.qidx)
    _gpu_case(mt_lib, oracle_lib, src, rec, prm, uvp, q, qm, wl.qctx, jobs, configs.THREADS)


# ---- 4:4:4 (pick_uv16_444) ----

def _glue_444(op, src, rec, prm, uvp, q, qm, cd, mc, jb):
    """pick_uv16_444 of one leaf from the oracle's primitives."""
    f32 = np.float32
    cx, cy = int(jb["px"]), int(jb["py"])
    fl = int(jb["flags"])
    tr, bl, ft = bool(fl & 1), bool(fl & 2), bool(fl & 4)
    mlam, dlam = f32(prm.rd_lambda), f32(uvp.dir_lambda)
    scan = op.default_scan(16)
    fw, fh = src[1].shape[1], src[1].shape[0]
    vw, vh = min(max(prm.vis_w - cx, 0), 16), min(max(prm.vis_h - cy, 0), 16)
    ctx = []
    for pl in range(2):
        a, l = [int(v) for v in jb["a_coef"][pl]], [int(v) for v in jb["l_coef"][pl]]
        sk = 7 + int(any(v != 0x40 for v in a)) + int(any(v != 0x40 for v in l))
        s = sum(v >> 6 for v in a + l) - 8
        ctx.append((sk, int(s != 0) + int(s > 0)))

    def plane(pl, pred, tx, keep_dc):
        s = src[1 + pl][cy:cy + 16, cx:cx + 16].astype(np.int32).ravel()
        resid = s - pred.ravel()
        lv, tf = op.fwd_txfm_quant(resid, tx, q, qm)
        lv = op.trellis_optimize(lv, tf, float(q.dc_q), float(q.ac_q), scan, prm.trellis_lambda0)
        if keep_dc:
            mean = int(np.trunc(resid.sum() / 256))
            if lv[0] == 0 and abs(mean) >= 8:
                lv[0] = 1 if mean > 0 else -1
        rr = op.inv_txfm_dequant(lv, tx, q, qm)
        sse = int(op.sse_recon(src[1 + pl], prm.vis_w, prm.vis_h, [(cx, cy)], pred.ravel(), rr, 16, 16,
                               scale=prm.wsse_scale)[0])
        return sse, f32(op.real_block_bits_bounded(lv, scan, 16, 16, cd, ctx[pl][0], ctx[pl][1], -1, 0, INF))

    ym = int(jb["y_mode"])
    dc = [int(op.intra_predict(rec[1 + pl], cx, cy, 16, 16, abi.DC_PRED)[0, 0]) for pl in range(2)]
    dcp = [plane(pl, np.full((16, 16), dc[pl]), abi.TX_DCT_DCT, True) for pl in range(2)]
    blk = np.array([(cx, cy, (dc[0], dc[1]))], abi.CFL_BLOCK_DTYPE)
    alpha, ac = op.cfl_alpha(rec[0], src[1], src[2], 0, 0, 16, 16, blk, vis=(prm.vis_w, prm.vis_h))
    al = (int(alpha[0][0]), int(alpha[0][1]))
    cfp = []
    for pl in range(2):
        diff = al[pl] * ac[0]
        mag = (np.abs(diff) + 32) >> 6
        cfp.append(plane(pl, np.clip(dc[pl] + np.where(diff < 0, -mag, mag), 0, 255), abi.TX_DCT_DCT, False))
    sig = f32(op.uv_mode_bits(mc, ym, abi.UV_CFL_PRED, al))
    dcb = f32(op.uv_mode_bits(mc, ym, abi.DC_PRED))
    dc_total = f32(f32(dcp[0][0] + dcp[1][0]) + f32(mlam * f32(f32(dcp[0][1] + dcp[1][1]) + dcb)))
    cfl_total = f32(f32(cfp[0][0] + cfp[1][0]) + f32(mlam * f32(f32(cfp[0][1] + cfp[1][1]) + sig)))
    use_cfl = cfl_total < dc_total and any(al)
    cur = cfp if use_cfl else dcp
    best = f32(dlam * (sig if use_cfl else dcb))
    for pl in range(2):
        best = f32(best + f32(f32(cur[pl][0]) + f32(dlam * cur[pl][1])))
    mode, delta = abi.DC_PRED, 0
    top = []  # DirectionalTopK, K = 3
    for m in JOINT:
        sc = 0
        for pl in range(2):
            pp = op.intra_predict(rec[1 + pl], cx, cy, 16, 16, m, 0, tr, bl, ft, fw=fw, fh=fh)
            d = np.where((np.arange(16)[None, :] < vw) & (np.arange(16)[:, None] < vh),
                         src[1 + pl][cy:cy + 16, cx:cx + 16].astype(np.int64) - pp, 0)
            h4 = np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]])
            satd = sum(int(np.abs(h4 @ d[ty:ty + 4, tx:tx + 4] @ h4.T).sum()) for ty in range(0, 16, 4)
                       for tx in range(0, 16, 4))
            sc += int(np.abs(d).sum()) + (satd >> 2)
        if len(top) == 3 and sc >= top[-1][0]:
            continue
        pos = len(top) if len(top) < 3 else 2
        if len(top) < 3:
            top.append(None)
        while pos > 0 and sc < top[pos - 1][0]:
            top[pos] = top[pos - 1]
            pos -= 1
        top[pos] = (sc, m)
    txmap = {abi.PAETH_PRED: abi.TX_ADST_ADST, abi.SMOOTH_PRED: abi.TX_ADST_ADST, abi.D135_PRED: abi.TX_ADST_ADST,
             abi.SMOOTH_V_PRED: abi.TX_ADST_DCT, abi.V_PRED: abi.TX_ADST_DCT, abi.D113_PRED: abi.TX_ADST_DCT,
             abi.D67_PRED: abi.TX_ADST_DCT, abi.SMOOTH_H_PRED: abi.TX_DCT_ADST, abi.H_PRED: abi.TX_DCT_ADST,
             abi.D157_PRED: abi.TX_DCT_ADST, abi.D203_PRED: abi.TX_DCT_ADST}

    def price(m, d, etr, ebl, bits):
        total = f32(dlam * f32(bits))
        for pl in range(2):
            pp = op.intra_predict(rec[1 + pl], cx, cy, 16, 16, m, d, etr, ebl, ft, fw=fw, fh=fh)
            sse, b = plane(pl, pp, txmap.get(m, abi.TX_DCT_DCT), True)
            total = f32(total + f32(f32(sse) + f32(dlam * b)))
        return total

    ranked = {m for _, m in top}
    for m in JOINT:
        if m in ranked:
            t = price(m, 0, tr, bl, op.uv_mode_bits(mc, ym, m))
            if t < best:
                best, mode = t, m
    adc = np.ctypeslib.as_array(mc.angle_delta)
    zone2 = {abi.V_PRED: (1, 2, 3), abi.H_PRED: (-3, -2, -1), abi.D113_PRED: (-3, -2, -1, 1, 2, 3),
             abi.D135_PRED: (-3, -2, -1, 1, 2, 3), abi.D157_PRED: (-3, -2, -1, 1, 2, 3)}
    if uvp.angle_deltas and abi.V_PRED <= mode <= abi.D67_PRED:
        m = mode
        base = f32(f32(op.uv_mode_bits(mc, ym, m)) - f32(op.cdf_cost(adc[m - abi.V_PRED], 3)))
        for d in zone2.get(m, ()):
            t = price(m, d, False, False, f32(base + f32(op.cdf_cost(adc[m - abi.V_PRED], d + 3))))
            if t < best:
                best, delta = t, d
    um = mode if mode != abi.DC_PRED else (abi.UV_CFL_PRED if use_cfl else abi.DC_PRED)
    return best, dc_total, cfl_total, um, delta, al


def _case444(mt, op, w, h, seed, qidx, qm_level, wsse, vis_cut=(0, 0), skip=False, ad=True):
    src, rec = synth.planes444(synth.generate_rgb(w, h, seed, sigma=4.0, variant="1080p"), seed)
    q = op.quant_new_chroma(qidx, 0, 0, 8, qm_level)
    qm = op.qm_row(qm_level, 1, 16) if qm_level < 15 else None
    sb = [(float(np.float32(1.5 + 0.1 * k)), float(np.float32(0.2 + 0.05 * k))) for k in range(13)] if skip else None
    prm = mt.split16_params(w, h, trellis_lambda0=0.05, rd_lambda=0.2 * qidx + 3, wsse_scale=wsse,
                            vis=(w - vis_cut[0], h - vis_cut[1]), skip_bits=sb)
    uvp = mt.uv16_params(w, angle_deltas=ad, dir_lambda=0.15 * qidx + 2)
    return src, rec, q, qm, prm, uvp


@pytest.mark.parametrize("qidx,qm_level,wsse", [(90, 6, 1.0), (40, 15, 0.0)])
def test_uv16_444_oracle_glue(oracle_lib, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    op = oracle_lib
    src, rec, q, qm, prm, uvp = _case444(mt, op, 96, 64, qidx + 1, qidx, qm_level, wsse, vis_cut=(3, 1))
    cd = op.default_cdfs(op.qcat(qidx), 16, plane=1)
    mc = op.uv_mode_cdfs()
    jobs = synth.uv16_444_jobs(96, 64, qidx)
    res, _, _ = op.pick_uv16_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs)
    f32 = np.float32
    for i, jb in enumerate(jobs):
        best, dct, cflt, mode, delta, al = _glue_444(op, src, rec, prm, uvp, q, qm, cd, mc, jb)
        r = res[i]
        assert (f32(r["total"]), f32(r["dc_total"]), f32(r["cfl_total"])) == (best, dct, cflt), i
        assert (int(r["uv_mode"]), int(r["angle_delta"]), tuple(int(v) for v in r["cfl_alpha"])) == (mode, delta, al)


def _gpu444(mt, op, src, rec, prm, uvp, q, qm, qctx, jobs, threads):
    cd = op.default_cdfs(qctx, 16, plane=1)
    mc = op.uv_mode_cdfs()
    costs = mt.coef_costs(mt.coef_cdfs_default(qctx, 16, 16, 1))
    mcost = mt.uv_mode_costs(mt.uv_mode_cdfs_default())
    got = mt.pick_uv16_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, costs, mcost, jobs, want_cf=True,
                           want_rec=True)
    want = op.pick_uv16_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs, threads=threads,
                            want_cf=True, want_rec=True)
    assert got[0].tobytes() == want[0].tobytes()
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    return got[0]


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,skip,ad", [(70, 6, 1.0, False, True), (116, 15, 0.0, True, True),
                                                         (30, 3, 0.75, False, False), (200, 10, 0.0, False, True)])
def test_uv16_444_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, skip, ad):
    src, rec, q, qm, prm, uvp = _case444(mt_lib, oracle_lib, 320, 192, qidx + 5, qidx, qm_level, wsse,
                                         vis_cut=(5, 2), skip=skip, ad=ad)
    jobs = synth.uv16_444_jobs(320, 192, qidx)
    jobs = np.concatenate([jobs, jobs[:2]])
    jobs["px"][-2] = 312  # leaves the plane: rejected
    jobs["y_mode"][-1] = 13
    res = _gpu444(mt_lib, oracle_lib, src, rec, prm, uvp, q, qm, oracle_lib.qcat(qidx), jobs, os.cpu_count() or 1)
    assert (res["uv_mode"][-2:] == 255).all() and (res["uv_mode"][:-2] != 255).all()
    kinds = set(int(m) for m in res["uv_mode"][:-2])
    assert abi.DC_PRED in kinds and len(kinds) >= 4, kinds


@pytest.mark.gpu
def test_uv16_444_at_config(mt_lib, oracle_lib, cuda):
    """Every 16x16 leaf of the 4:4:4 benchmark frame C1 (512x512, qindex 70):
    its chroma quantiser and QM level, the chroma TX_16X16 CDFs of its q
    context, the luma and chroma lambdas of its laws."""
    import configs

    wl = configs.workload("C1")
    src, rec = synth.planes444(wl.rgb, wl.qidx)
    q = mt_lib.quant_new_chroma(wl.qidx, 0, 0, 8, wl.qm_uv)
    qm = mt_lib.qm_row(wl.qm_uv, 1, 16) if wl.qm_uv < 15 else None
    prm = mt_lib.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                wsse_scale=1.0)
    uvp = mt_lib.uv16_params(wl.w, angle_deltas=True, dir_lambda=wl.lam.lambda_d)
    jobs = synth.uv16_444_jobs(wl.w, wl.h, wl.qidx)
    _gpu444(mt_lib, oracle_lib, src, rec, prm, uvp, q, qm, wl.qctx, jobs, configs.THREADS)


# ---- the 32x32 leaf at 4:2:0 (pick_uv32_420) ----

def _case32(mt, op, w, h, seed, qidx, qm_level, wsse, skip=False, ad=True):
    src, rec = _planes(w, h, seed)
    cw, ch = src[1].shape[1], src[1].shape[0]
    q = op.quant_new_chroma(qidx, 0, 0, 8, qm_level)
    qm = op.qm_row(qm_level, 1, 16) if qm_level < 15 else None
    sb = [(float(np.float32(1.5 + 0.1 * k)), float(np.float32(0.2 + 0.05 * k))) for k in range(13)] if skip else None
    prm = mt.split16_params(cw, ch, trellis_lambda0=0.05, rd_lambda=0.2 * qidx + 3, band_tilt=0.6, wsse_scale=wsse,
                            vis=(cw - 3, ch - 1), skip_bits=sb)
    uvp = mt.uv16_params(src[0].shape[1], angle_deltas=ad)
    return src, rec, q, qm, prm, uvp


@pytest.mark.parametrize("qidx,qm_level,wsse", [(90, 6, 1.0), (40, 15, 0.0)])
def test_uv32_oracle_accounting(oracle_lib, qidx, qm_level, wsse):
    """The oracle's DC and CfL totals and its winner's total equal the costs
    recomputed from the oracle's primitives (the 4:2:0 context trellis on
    16x16 chroma, the CfL AC of the 32x32 luma); the winner is no worse than
    DC and, unless CfL was refused, CfL."""
    import maroontree_b200 as mt

    op = oracle_lib
    src, rec, q, qm, prm, uvp = _case32(mt, op, 128, 96, qidx + 2, qidx, qm_level, wsse)
    cd = op.default_cdfs(op.qcat(qidx), 16, plane=1)
    mc = op.uv_mode_cdfs()
    jobs = synth.uv16_444_jobs(128, 96, qidx, leaf=32)
    res, _, _ = op.pick_uv32_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs)
    f32 = np.float32
    lam = f32(prm.rd_lambda)
    scan = op.default_scan(16)
    adc = np.ctypeslib.as_array(mc.angle_delta)
    txmap = {abi.PAETH_PRED: abi.TX_ADST_ADST, abi.SMOOTH_PRED: abi.TX_ADST_ADST, abi.D135_PRED: abi.TX_ADST_ADST,
             abi.SMOOTH_V_PRED: abi.TX_ADST_DCT, abi.V_PRED: abi.TX_ADST_DCT, abi.D113_PRED: abi.TX_ADST_DCT,
             abi.D67_PRED: abi.TX_ADST_DCT, abi.SMOOTH_H_PRED: abi.TX_DCT_ADST, abi.H_PRED: abi.TX_DCT_ADST,
             abi.D157_PRED: abi.TX_DCT_ADST, abi.D203_PRED: abi.TX_DCT_ADST}
    cw, ch = src[1].shape[1], src[1].shape[0]
    for i, jb in enumerate(jobs):
        cx, cy, fl, ym = int(jb["px"]) // 2, int(jb["py"]) // 2, int(jb["flags"]), int(jb["y_mode"])
        ctx = []
        for pl in range(2):
            a, l = [int(v) for v in jb["a_coef"][pl]], [int(v) for v in jb["l_coef"][pl]]
            s = sum(v >> 6 for v in a + l) - 8
            ctx.append((7 + int(any(v != 0x40 for v in a)) + int(any(v != 0x40 for v in l)),
                        int(s != 0) + int(s > 0)))

        def plane(pl, pred, tx, keep_dc):
            resid = src[1 + pl][cy:cy + 16, cx:cx + 16].astype(np.int32).ravel() - pred.ravel()
            lv, tf = op.fwd_txfm_quant(resid, tx, q, qm)
            lv = op.trellis_optimize_ctx(lv, tf, q, qm, cd, ctx[pl][1], prm.trellis_lambda0, band_tilt=prm.band_tilt,
                                         n=16)
            if keep_dc:
                mean = int(np.trunc(resid.sum() / 256))
                if lv[0] == 0 and abs(mean) >= 8:
                    lv[0] = 1 if mean > 0 else -1
            rr = op.inv_txfm_dequant(lv, tx, q, qm)
            sse = int(op.sse_recon(src[1 + pl], prm.vis_w, prm.vis_h, [(cx, cy)], pred.ravel(), rr, 16, 16,
                                   scale=prm.wsse_scale)[0])
            bits = f32(op.real_block_bits_bounded(lv, scan, 16, 16, cd, ctx[pl][0], ctx[pl][1], -1, 0, INF))
            return f32(f32(sse) + f32(lam * bits))

        dc = [int(op.intra_predict(rec[1 + pl], cx, cy, 16, 16, abi.DC_PRED)[0, 0]) for pl in range(2)]
        dct = f32(0)
        for pl in range(2):
            dct = f32(dct + plane(pl, np.full((16, 16), dc[pl]), abi.TX_DCT_DCT, True))
        blk = np.array([(cx, cy, (dc[0], dc[1]))], abi.CFL_BLOCK_DTYPE)
        alpha, ac = op.cfl_alpha(rec[0], src[1], src[2], 1, 1, 16, 16, blk, vis=(prm.vis_w, prm.vis_h))
        body = f32(0)
        for pl in range(2):
            diff = int(alpha[0][pl]) * ac[0]
            mag = (np.abs(diff) + 32) >> 6
            body = f32(body + plane(pl, np.clip(dc[pl] + np.where(diff < 0, -mag, mag), 0, 255), abi.TX_DCT_DCT, False))
        cflt = f32(f32(body + f32(lam * f32(op.uv_mode_bits(mc, ym, abi.UV_CFL_PRED, tuple(int(v) for v in alpha[0])))))
                   - f32(lam * f32(op.uv_mode_bits(mc, ym, abi.DC_PRED))))
        r = res[i]
        assert (f32(r["dc_total"]), f32(r["cfl_total"])) == (dct, cflt), i
        assert tuple(int(v) for v in r["cfl_alpha"]) == tuple(int(v) for v in alpha[0])
        m, d = int(r["uv_mode"]), int(r["angle_delta"])
        assert f32(r["total"]) <= dct
        if m == abi.DC_PRED:
            want = dct
        elif m == abi.UV_CFL_PRED:
            want = cflt
        else:
            bits = f32(op.uv_mode_bits(mc, ym, m))
            if d != 0:
                bits = f32(f32(bits - f32(op.cdf_cost(adc[m - abi.V_PRED], 3))) +
                           f32(op.cdf_cost(adc[m - abi.V_PRED], d + 3)))
            want = f32(lam * bits)
            tr, bl = (bool(fl & 1), bool(fl & 2)) if d == 0 else (False, False)
            for pl in range(2):
                pp = op.intra_predict(rec[1 + pl], cx, cy, 16, 16, m, d, tr, bl, bool(fl & 4), fw=cw, fh=ch)
                want = f32(want + plane(pl, pp, txmap.get(m, abi.TX_DCT_DCT), True))
        assert f32(r["total"]) == want, (i, m, d)


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,skip,ad", [(70, 6, 1.0, False, True), (116, 15, 0.0, True, True),
                                                         (30, 3, 0.75, False, False)])
def test_uv32_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, skip, ad):
    src, rec, q, qm, prm, uvp = _case32(mt_lib, oracle_lib, 320, 192, qidx + 9, qidx, qm_level, wsse, skip=skip, ad=ad)
    jobs = synth.uv16_444_jobs(320, 192, qidx, leaf=32)
    jobs = np.concatenate([jobs, jobs[:2]])
    jobs["px"][-2] = 304  # leaves the plane: rejected
    jobs["y_mode"][-1] = 13
    cd = oracle_lib.default_cdfs(oracle_lib.qcat(qidx), 16, plane=1)
    mc = oracle_lib.uv_mode_cdfs()
    costs = mt_lib.coef_costs(mt_lib.coef_cdfs_default(oracle_lib.qcat(qidx), 16, 16, 1))
    mcost = mt_lib.uv_mode_costs(mt_lib.uv_mode_cdfs_default())
    got = mt_lib.pick_uv32_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, costs, mcost, jobs,
                               want_cf=True, want_rec=True)
    want = oracle_lib.pick_uv32_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs,
                                    threads=os.cpu_count() or 1, want_cf=True, want_rec=True)
    assert got[0].tobytes() == want[0].tobytes()
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    assert (got[0]["uv_mode"][-2:] == 255).all()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["C2q40", "C2q80"])
def test_uv32_at_config(mt_lib, oracle_lib, cuda, name):
    import configs

    wl = configs.workload(name)
    src, rec = synth.planes420(wl.rgb, wl.qidx)
    cw, ch = src[1].shape[1], src[1].shape[0]
    q = mt_lib.quant_new_chroma(wl.qidx, 0, 0, 8, wl.qm_uv)
    qm = mt_lib.qm_row(wl.qm_uv, 1, 16) if wl.qm_uv < 15 else None
    prm = mt_lib.split16_params(cw, ch, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                wsse_scale=1.0, vis=(wl.w // 2, wl.h // 2))
    uvp = mt_lib.uv16_params(src[0].shape[1], angle_deltas=True)
    jobs = synth.uv16_444_jobs(wl.w, wl.h, wl.qidx, leaf=32)
    cd = oracle_lib.default_cdfs(wl.qctx, 16, plane=1)
    got = mt_lib.pick_uv32_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm,
                               mt_lib.coef_costs(mt_lib.coef_cdfs_default(wl.qctx, 16, 16, 1)),
                               mt_lib.uv_mode_costs(mt_lib.uv_mode_cdfs_default()), jobs)
    want = oracle_lib.pick_uv32_420(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd,
                                    oracle_lib.uv_mode_cdfs(), jobs, threads=configs.THREADS)
    assert got[0].tobytes() == want[0].tobytes()


# ---- the 32x32 leaf at 4:4:4 (pick_uv32_444) ----

def _case32_444(mt, op, w, h, seed, qidx, qm_level, wsse, skip=False, ad=True):
    src, rec = synth.planes444(synth.generate_rgb(w, h, seed, sigma=4.0, variant="1080p"), seed)
    q = op.quant_new_chroma(qidx, 0, 0, 8, qm_level)
    qm = op.qm_row(qm_level, 1, 32) if qm_level < 15 else None
    sb = [(float(np.float32(1.5 + 0.1 * k)), float(np.float32(0.2 + 0.05 * k))) for k in range(13)] if skip else None
    prm = mt.split16_params(w, h, trellis_lambda0=0.05, rd_lambda=0.2 * qidx + 3, wsse_scale=wsse,
                            vis=(w - 5, h - 2), skip_bits=sb)
    uvp = mt.uv16_params(w, angle_deltas=ad, dir_lambda=0.15 * qidx + 2)
    return src, rec, q, qm, prm, uvp


@pytest.mark.parametrize("qidx,qm_level,wsse", [(90, 6, 1.0), (40, 15, 0.0)])
def test_uv32_444_oracle_accounting(oracle_lib, qidx, qm_level, wsse):
    """The oracle's DC and CfL totals (the planes' costs summed, then the mode
    bits), its winner's total and levels recomputed from primitives: the plain
    trellis over the 1024-entry scan, DCT_DCT for every mode, contexts over
    eight bytes per side."""
    import maroontree_b200 as mt

    op = oracle_lib
    src, rec, q, qm, prm, uvp = _case32_444(mt, op, 128, 96, qidx + 4, qidx, qm_level, wsse)
    cd = op.default_cdfs(op.qcat(qidx), 32, plane=1)
    mc = op.uv_mode_cdfs()
    jobs = synth.uv32_444_jobs(128, 96, qidx)
    res, cfo, _ = op.pick_uv32_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd, mc, jobs, want_cf=True)
    f32 = np.float32
    mlam, dlam = f32(prm.rd_lambda), f32(uvp.dir_lambda)
    scan = op.default_scan(32)
    adc = np.ctypeslib.as_array(mc.angle_delta)
    for i, jb in enumerate(jobs):
        cx, cy, fl, ym = int(jb["px"]), int(jb["py"]), int(jb["flags"]), int(jb["y_mode"])
        ctx = []
        for pl in range(2):
            a, l = [int(v) for v in jb["a_coef"][pl]], [int(v) for v in jb["l_coef"][pl]]
            s = sum(v >> 6 for v in a + l) - 16
            ctx.append((7 + int(any(v != 0x40 for v in a)) + int(any(v != 0x40 for v in l)),
                        int(s != 0) + int(s > 0)))

        def plane(pl, pred, keep_dc):
            resid = src[1 + pl][cy:cy + 32, cx:cx + 32].astype(np.int32).ravel() - pred.ravel()
            lv, tf = op.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
            lv = op.trellis_optimize(lv, tf, float(q.dc_q), float(q.ac_q), scan, prm.trellis_lambda0)
            if keep_dc:
                mean = int(np.trunc(resid.sum() / 1024))
                if lv[0] == 0 and abs(mean) >= 8:
                    lv[0] = 1 if mean > 0 else -1
            rr = op.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, qm)
            sse = int(op.sse_recon(src[1 + pl], prm.vis_w, prm.vis_h, [(cx, cy)], pred.ravel(), rr, 32, 32,
                                   scale=prm.wsse_scale)[0])
            return sse, f32(op.real_block_bits_bounded(lv, scan, 32, 32, cd, ctx[pl][0], ctx[pl][1], -1, 0, INF)), lv

        dc = [int(op.intra_predict(rec[1 + pl], cx, cy, 32, 32, abi.DC_PRED)[0, 0]) for pl in range(2)]
        dcp = [plane(pl, np.full((32, 32), dc[pl]), True) for pl in range(2)]
        blk = np.array([(cx, cy, (dc[0], dc[1]))], abi.CFL_BLOCK_DTYPE)
        alpha, ac = op.cfl_alpha(rec[0], src[1], src[2], 0, 0, 32, 32, blk, vis=(prm.vis_w, prm.vis_h))
        al = (int(alpha[0][0]), int(alpha[0][1]))
        cfp = []
        for pl in range(2):
            diff = al[pl] * ac[0]
            mag = (np.abs(diff) + 32) >> 6
            cfp.append(plane(pl, np.clip(dc[pl] + np.where(diff < 0, -mag, mag), 0, 255), False))
        cost = lambda c: f32(f32(c[0]) + f32(mlam * c[1]))
        dct = f32(f32(f32(cost(dcp[0]) + cost(dcp[1])) + f32(mlam * f32(op.uv_mode_bits(mc, ym, abi.DC_PRED)))))
        cflt = f32(f32(f32(cost(cfp[0]) + cost(cfp[1])) + f32(mlam * f32(op.uv_mode_bits(mc, ym, abi.UV_CFL_PRED, al)))))
        r = res[i]
        assert (f32(r["dc_total"]), f32(r["cfl_total"])) == (dct, cflt), i
        m, d = int(r["uv_mode"]), int(r["angle_delta"])
        if m in (abi.DC_PRED, abi.UV_CFL_PRED):
            cur = cfp if m == abi.UV_CFL_PRED else dcp
            bits = f32(op.uv_mode_bits(mc, ym, abi.UV_CFL_PRED, al) if m == abi.UV_CFL_PRED else
                       op.uv_mode_bits(mc, ym, abi.DC_PRED))
            want = f32(dlam * bits)
            for pl in range(2):
                want = f32(want + f32(f32(cur[pl][0]) + f32(dlam * cur[pl][1])))
            levels = [cur[0][2], cur[1][2]]
        else:
            bits = f32(op.uv_mode_bits(mc, ym, m))
            if d != 0:
                bits = f32(f32(bits - f32(op.cdf_cost(adc[m - abi.V_PRED], 3))) +
                           f32(op.cdf_cost(adc[m - abi.V_PRED], d + 3)))
            want = f32(dlam * bits)
            tr, bl = (bool(fl & 1), bool(fl & 2)) if d == 0 else (False, False)
            levels = []
            for pl in range(2):
                pp = op.intra_predict(rec[1 + pl], cx, cy, 32, 32, m, d, tr, bl, bool(fl & 4), fw=128, fh=96)
                sse, b, lv = plane(pl, pp, True)
                want = f32(want + f32(f32(sse) + f32(dlam * b)))
                levels.append(lv)
        assert f32(r["total"]) == want, (i, m, d)
        assert np.array_equal(cfo[i], np.concatenate(levels)), i


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,skip,ad", [(70, 6, 1.0, False, True), (116, 15, 0.0, True, True),
                                                         (30, 3, 0.75, False, False)])
def test_uv32_444_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, skip, ad):
    src, rec, q, qm, prm, uvp = _case32_444(mt_lib, oracle_lib, 320, 192, qidx + 11, qidx, qm_level, wsse,
                                            skip=skip, ad=ad)
    jobs = synth.uv32_444_jobs(320, 192, qidx)
    jobs = np.concatenate([jobs, jobs[:2]])
    jobs["px"][-2] = 304  # leaves the plane: rejected
    jobs["y_mode"][-1] = 13
    cd = oracle_lib.default_cdfs(oracle_lib.qcat(qidx), 32, plane=1)
    costs = mt_lib.coef_costs(mt_lib.coef_cdfs_default(oracle_lib.qcat(qidx), 32, 32, 1))
    mcost = mt_lib.uv_mode_costs(mt_lib.uv_mode_cdfs_default())
    got = mt_lib.pick_uv32_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, costs, mcost, jobs,
                               want_cf=True, want_rec=True)
    want = oracle_lib.pick_uv32_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd,
                                    oracle_lib.uv_mode_cdfs(), jobs, threads=os.cpu_count() or 1, want_cf=True,
                                    want_rec=True)
    assert got[0].tobytes() == want[0].tobytes()
    assert np.array_equal(got[1], want[1]) and np.array_equal(got[2], want[2])
    assert (got[0]["uv_mode"][-2:] == 255).all()


@pytest.mark.gpu
def test_uv32_444_at_config(mt_lib, oracle_lib, cuda):
    """Every 32x32 leaf of C1 (512x512 4:4:4, qindex 70) with its chroma
    quantiser, QM and lambdas and the chroma TX_32X32 CDFs of its q context."""
    import configs

    wl = configs.workload("C1")
    src, rec = synth.planes444(wl.rgb, wl.qidx)
    q = mt_lib.quant_new_chroma(wl.qidx, 0, 0, 8, wl.qm_uv)
    qm = mt_lib.qm_row(wl.qm_uv, 1, 32) if wl.qm_uv < 15 else None
    prm = mt_lib.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                wsse_scale=1.0)
    uvp = mt_lib.uv16_params(wl.w, angle_deltas=True, dir_lambda=wl.lam.lambda_d)
    jobs = synth.uv32_444_jobs(wl.w, wl.h, wl.qidx)
    cd = oracle_lib.default_cdfs(wl.qctx, 32, plane=1)
    got = mt_lib.pick_uv32_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm,
                               mt_lib.coef_costs(mt_lib.coef_cdfs_default(wl.qctx, 32, 32, 1)),
                               mt_lib.uv_mode_costs(mt_lib.uv_mode_cdfs_default()), jobs)
    want = oracle_lib.pick_uv32_444(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm, cd,
                                    oracle_lib.uv_mode_cdfs(), jobs, threads=configs.THREADS)
    assert got[0].tobytes() == want[0].tobytes()
