"""The 64x64 leaf's luma legs (rd_pick_luma64, src/coder/block64.rs:1812-2012;
TX_64X64 is off in the shipped tuning, so a 64x64 codes four TX_32X32 or,
with tx64_depth2, sixteen TX_16X16):
  * the four-TX_32X32 candidate leg (:1906-1958): quadrants in raster order
    from the running reconstruction, quad_edges' flags, the 32x32 chain in
    each quadrant's dc_sign context, sse x K_PART_LAMBDA and the f32 total;
  * the sixteen-TX_16X16 tx_depth-2 leg (:1983-2010, grid16_luma_pass
    :1670-1805): the transforms in raster order with grid edge flags, the
    coefficient contexts carried from transform to transform (skip_ctx_split
    and dc_sign_ctx_span over four above / four left bytes, coef_res_ctx),
    the DCT_DCT symbol of the mode's TX_16X16 tx-type CDF and the tx_depth
    symbol difference in the total.
CPU tests check the oracle's legs against compositions of its own primitives
written here step by step; GPU tests compare the CUDA legs with the oracle
bit for bit, at the benchmark configurations with the default CDFs."""
import os

import numpy as np
import pytest

from maroontree_b200 import abi, synth

INF = float("inf")


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 19)
    return src, rec


def quad32_jobs(fw, fh, modes, deltas=(0,), seed=0):
    """(64x64 block, mode, delta) jobs of the 64x64 leaf's four-TX_32X32 leg:
    the 64-grid blocks, neighbour flags, random filter types, per-quadrant
    dc_sign contexts and mode / delta bits."""
    rng = np.random.default_rng(seed)
    rows = []
    for py in range(0, fh - 63, 64):
        for px in range(0, fw - 63, 64):
            fl = synth.block_flags(px, py, fw, fh, 64) | (abi.CAND_FILTER_TYPE if rng.random() < 0.5 else 0)
            dcs = rng.integers(0, 3, size=4)
            for m in modes:
                for d in (deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)):
                    rows.append((px, py, m, d, fl, 0, tuple(int(v) for v in dcs), np.float32(rng.random() * 6 + 1),
                                 np.float32(rng.random() * 3 + 0.5)))
    return np.array(rows, abi.QUAD32_JOB_DTYPE)


def test_quad32_oracle_glue(oracle_lib):
    """rd_pick_luma64's four-TX_32X32 leg (block64.rs:1906-1958): quadrants in
    raster order from the running reconstruction with quad_edges' flags, the
    32x32 chain in each quadrant's dc_sign context, sse x K_PART_LAMBDA, and
    the f32 total in the reference's order."""
    import maroontree_b200 as mt

    src, rec = _frame(128, 128, 51)
    q = oracle_lib.quant_new(80, 8, 5)
    qm = oracle_lib.qm_row(5, 0, 32)
    c = oracle_lib.default_cdfs(oracle_lib.qcat(80), 32)
    prm = mt.split16_params(128, 128, trellis_lambda0=0.05, rd_lambda=18.0, band_tilt=1.3, wsse_scale=1.0)
    jobs = quad32_jobs(128, 128, (abi.DC_PRED, abi.V_PRED, abi.D157_PRED, abi.SMOOTH_PRED), deltas=(0, -2), seed=3)
    scan = oracle_lib.default_scan(32)
    f32 = np.float32
    res = oracle_lib.quad32_luma(src, rec, prm, q, qm, c, jobs)
    for i, jb in enumerate(jobs):
        px, py, fl, m, d = int(jb["px"]), int(jb["py"]), int(jb["flags"]), int(jb["mode"]), int(jb["angle_delta"])
        work = rec.copy()
        total = f32(f32(18.0) * jb["mode_bits"])
        if abi.V_PRED <= m <= abi.D67_PRED:
            total = f32(total + f32(f32(18.0) * jb["delta_bits"]))
        edges = [(py > 0, px > 0), (bool(fl & 1), False), (True, bool(fl & 2)), (False, False)]
        for k, (sx, sy) in enumerate(((0, 0), (32, 0), (0, 32), (32, 32))):
            bx, by = px + sx, py + sy
            pred = oracle_lib.intra_predict(work, bx, by, 32, 32, m, d, edges[k][0], edges[k][1], bool(fl & 4)).ravel()
            resid = src[by:by + 32, bx:bx + 32].astype(np.int32).ravel() - pred
            lv, tf = oracle_lib.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
            lv = oracle_lib.trellis_optimize_ctx(lv, tf, q, qm, c, int(jb["dcs_ctx"][k]), 0.05, band_tilt=1.3, n=32)
            rr = oracle_lib.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, qm)
            sse = int(oracle_lib.sse_recon(src, 128, 128, [(bx, by)], pred, rr, 32, 32, scale=1.0)[0])
            bits = f32(oracle_lib.real_block_bits_bounded(lv, scan, 32, 32, c, 0, int(jb["dcs_ctx"][k]), -1, 0, INF))
            assert res["sse"][i][k] == sse and f32(res["bits"][i][k]) == bits, (i, k)
            total = f32(total + f32(f32(f32(sse) * f32(2.775)) + f32(f32(18.0) * bits)))
            work[by:by + 32, bx:bx + 32] = np.clip(pred + rr, 0, 255).reshape(32, 32)
        assert f32(res["total"][i]) == total, i


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse", [(70, 6, 1.0), (116, 15, 0.0), (30, 3, 0.75)])
def test_quad32_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    src, rec = _frame(320, 192, qidx + 9)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 32) if qm_level < 15 else None
    c = oracle_lib.default_cdfs(oracle_lib.qcat(qidx), 32)
    jobs = quad32_jobs(320, 192, range(13), deltas=(-3, 0, 1), seed=qidx)
    jobs["px"][3] = 280  # crosses the right edge: rejected
    prm = mt.split16_params(320, 192, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.9,
                            wsse_scale=wsse, vis=(311, 190))
    res = mt_lib.quad32_luma(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs)
    want = oracle_lib.quad32_luma(src, rec, prm, q, qm, c, jobs, threads=os.cpu_count() or 1)
    assert res.tobytes() == want.tobytes()
    assert np.isinf(res["total"][3]) and np.isfinite(res["total"][0])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["C1", "C2q40", "C2q60", "C2q80"])
def test_quad32_at_config(mt_lib, oracle_lib, cuda, name):
    """Every 64x64 block of the benchmark frames with the 13 modes (angle
    deltas -3 / 0 / 3), the configuration's quantiser, QM and lambdas and the
    default TX_32X32 CDFs."""
    import configs

    wl = configs.workload(name)
    qm = configs.qm(mt_lib, wl, 32)
    c = configs.cdfs(mt_lib, wl, 32)
    jobs = quad32_jobs(wl.w, wl.h, range(13), deltas=(-3, 0, 3), seed=wl.qidx)
    prm = mt_lib.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                band_tilt=0.0, wsse_scale=1.0)
    res = mt_lib.quad32_luma(wl.src, wl.rec, prm, wl.q, qm, mt_lib.coef_costs(c), jobs)
    want = oracle_lib.quad32_luma(wl.src, wl.rec, prm, wl.q, qm, c, jobs, threads=configs.THREADS)
    assert res.tobytes() == want.tobytes()



def grid16_jobs(fw, fh, modes, deltas=(0,), seed=0, zero_ctx=False):
    """(64x64 block, mode, delta) jobs of the sixteen-TX_16X16 leg: random
    neighbour flags and filter types, above / left coefficient-context bytes
    drawn like coef_res_ctx's (cumulative level 0..63 with a dc-sign marker,
    or 0x40 for an uncoded neighbour), mode / delta / tx_depth bits."""
    rng = np.random.default_rng(seed)
    rows = []

    def ctx_bytes():
        if zero_ctx:
            return tuple([0x40] * 16)
        cul = rng.integers(0, 64, size=16)
        sign = rng.choice([0x00, 0x40, 0x80], size=16)
        b = np.where(rng.random(16) < 0.3, 0x40, cul | sign)
        return tuple(int(v) for v in b)

    for py in range(0, fh - 63, 64):
        for px in range(0, fw - 63, 64):
            fl = synth.block_flags(px, py, fw, fh, 64) | (abi.CAND_FILTER_TYPE if rng.random() < 0.5 else 0)
            if rng.random() < 0.3:
                fl ^= rng.integers(0, 4)  # the caller's own neighbour flags
            a, l = ctx_bytes(), ctx_bytes()
            for m in modes:
                for d in (deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)):
                    rows.append((px, py, m, d, fl, 0, a, l, np.float32(rng.random() * 6 + 1),
                                 np.float32(rng.random() * 3 + 0.5), np.float32(rng.random() * 4 - 1)))
    return np.array(rows, abi.GRID16_JOB_DTYPE)


def _skip_table(seed):
    rng = np.random.default_rng(seed)
    return [(float(np.float32(rng.random() * 3 + 0.1)), float(np.float32(rng.random() * 2 + 0.05))) for _ in range(13)]


@pytest.mark.parametrize("skip", [False, True])
def test_grid16_oracle_glue(oracle_lib, skip):
    """grid16_luma_pass step by step: edge flags, skip / dc_sign contexts from
    the carried bytes, the 16x16 chain, coef_res_ctx, and the total's order."""
    import maroontree_b200 as mt

    src, rec = _frame(128, 128, 77)
    q = oracle_lib.quant_new(90, 8, 6)
    qm = oracle_lib.qm_row(6, 0, 16)
    c = oracle_lib.default_cdfs(oracle_lib.qcat(90), 16)
    sb = _skip_table(5) if skip else None
    prm = mt.split16_params(128, 128, trellis_lambda0=0.05, rd_lambda=21.0, band_tilt=0.7, wsse_scale=1.0,
                            skip_bits=sb)
    jobs = grid16_jobs(128, 128, (abi.DC_PRED, abi.H_PRED, abi.D203_PRED, abi.PAETH_PRED), deltas=(0, 2), seed=8)
    scan = oracle_lib.default_scan(16)
    f32 = np.float32
    lam = f32(21.0)
    res, cfo = oracle_lib.grid16_luma(src, rec, prm, q, qm, c, jobs, want_cf=True)
    tbl = [[1, 2, 2, 2, 3], [2, 4, 4, 4, 5], [2, 4, 4, 4, 5], [2, 4, 4, 4, 5], [3, 5, 5, 5, 6]]
    for i, jb in enumerate(jobs):
        px, py, fl, m, d = int(jb["px"]), int(jb["py"]), int(jb["flags"]), int(jb["mode"]), int(jb["angle_delta"])
        a, l = [int(v) for v in jb["a_coef"]], [int(v) for v in jb["l_coef"]]
        work = rec.copy()
        dist = bits = f32(0.0)
        for t in range(16):
            tx, ty = t % 4, t // 4
            bx, by = px + 16 * tx, py + 16 * ty
            tr = (py > 0 and (tx < 3 or bool(fl & 1))) if ty == 0 else tx < 3
            bl = tx == 0 and px > 0 and (ty < 3 or bool(fl & 2))
            pred = oracle_lib.intra_predict(work, bx, by, 16, 16, m, d, tr, bl, bool(fl & 4)).ravel()
            resid = src[by:by + 16, bx:bx + 16].astype(np.int32).ravel() - pred
            la = ll = 0
            for k in range(4):
                la |= a[4 * tx + k]
                ll |= l[4 * ty + k]
            sk = tbl[min(la & 0x3f, 4)][min(ll & 0x3f, 4)]
            s = sum((a[4 * tx + k] >> 6) - 1 + (l[4 * ty + k] >> 6) - 1 for k in range(4))
            ds = int(s != 0) + int(s > 0)
            lv, tf = oracle_lib.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
            lv = oracle_lib.trellis_optimize_ctx(lv, tf, q, qm, c, ds, 0.05, band_tilt=0.7, n=16)
            rr = oracle_lib.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, qm)
            sse = int(oracle_lib.sse_recon(src, 128, 128, [(bx, by)], pred, rr, 16, 16, scale=1.0)[0])
            dist = f32(dist + f32(f32(sse) * f32(2.775)))
            bits = f32(bits + f32(oracle_lib.real_block_bits_bounded(
                lv, scan, 16, 16, c, sk, ds, m, 1, INF, skip_bits=None if sb is None else np.array(sb[sk], np.float32))))
            assert np.array_equal(cfo[i][256 * t:256 * t + 256], lv), (i, t)
            nz = [int(lv[r]) for r in scan if lv[r] != 0]
            if not nz:
                rc = 0x40
            else:
                eob = max(k for k, r in enumerate(scan) if lv[r] != 0)
                cul = sum(abs(int(lv[r])) for r in scan[:eob + 1])
                rc = min(cul, 63) | (0x40 if lv[0] == 0 else (0 if lv[0] < 0 else 0x80))
            a[4 * tx:4 * tx + 4] = [rc] * 4
            l[4 * ty:4 * ty + 4] = [rc] * 4
            work[by:by + 16, bx:bx + 16] = np.clip(pred + rr, 0, 255).reshape(16, 16)
        total = f32(lam * jb["mode_bits"])
        if abi.V_PRED <= m <= abi.D67_PRED:
            total = f32(total + f32(lam * jb["delta_bits"]))
        total = f32(total + f32(dist + f32(lam * bits)))
        total = f32(total + f32(lam * jb["depth_bits"]))
        assert f32(res["dist"][i]) == dist and f32(res["bits"][i]) == bits, i
        assert f32(res["total"][i]) == total, i


def test_grid16_oracle_rejects(oracle_lib):
    import maroontree_b200 as mt

    src, rec = _frame(128, 64, 3)
    q = oracle_lib.quant_new(60, 8, 15)
    c = oracle_lib.default_cdfs(oracle_lib.qcat(60), 16)
    prm = mt.split16_params(128, 64, rd_lambda=9.0)
    jobs = grid16_jobs(128, 64, (abi.DC_PRED, abi.V_PRED), seed=1)
    jobs["px"][0] = 96          # crosses the right edge
    jobs["angle_delta"][1] = 2  # a delta on a non-directional mode
    jobs["mode"][1] = abi.SMOOTH_PRED
    res, _ = oracle_lib.grid16_luma(src, rec, prm, q, None, c, jobs)
    assert np.isinf(res["total"][:2]).all() and (res["sse"][:2] == 0).all()
    assert np.isfinite(res["total"][2:]).all()


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse,skip", [(70, 6, 1.0, False), (116, 15, 0.0, True),
                                                     (30, 3, 0.75, False), (1, 15, 0.0, True)])
def test_grid16_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse, skip):
    import maroontree_b200 as mt

    src, rec = _frame(320, 192, qidx + 31)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 16) if qm_level < 15 else None
    c = oracle_lib.default_cdfs(oracle_lib.qcat(qidx), 16)
    jobs = grid16_jobs(320, 192, range(13), deltas=(-3, 0, 1), seed=qidx)
    jobs["px"][3] = 280  # crosses the right edge: rejected
    prm = mt.split16_params(320, 192, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.1,
                            wsse_scale=wsse, vis=(307, 190), skip_bits=_skip_table(qidx) if skip else None)
    res, cf = mt_lib.grid16_luma(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True)
    want, wcf = oracle_lib.grid16_luma(src, rec, prm, q, qm, c, jobs, threads=os.cpu_count() or 1, want_cf=True)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf)
    assert np.isinf(res["total"][3]) and np.isfinite(res["total"][0])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["C1", "C2q40", "C2q60", "C2q80"])
def test_grid16_at_config(mt_lib, oracle_lib, cuda, name):
    """Every 64x64 block of the benchmark frames with the 13 modes (angle
    deltas -3 / 0 / 3), the configuration's quantiser, QM and lambdas and the
    default TX_16X16 CDFs."""
    import configs

    wl = configs.workload(name)
    qm = configs.qm(mt_lib, wl, 16)
    c = configs.cdfs(mt_lib, wl, 16)
    jobs = grid16_jobs(wl.w, wl.h, range(13), deltas=(-3, 0, 3), seed=wl.qidx)
    prm = mt_lib.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                band_tilt=0.0, wsse_scale=1.0)
    res, _ = mt_lib.grid16_luma(wl.src, wl.rec, prm, wl.q, qm, mt_lib.coef_costs(c), jobs)
    want, _ = oracle_lib.grid16_luma(wl.src, wl.rec, prm, wl.q, qm, c, jobs, threads=configs.THREADS)
    assert res.tobytes() == want.tobytes()
