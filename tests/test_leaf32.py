"""The 32x32 leaf (pick_luma32's mode loop, src/coder/block32.rs:728-836) and
its TX_32X32 pieces: the forward DCT-32 of the reference's butterflies
(dct1d_32_i32 on the 16-point one), the dav1d inverse with the TX_32X32
dequantisation, trellis_optimize_ctx and the rate walk of class 3.

The reference's tests hold no 32x32 known answers, only properties; CPU
tests pin the oracle with them:
  * WC32 is round(65536 / (2 cos((2k+1) pi / 64))) (dct.rs:3846-3851), in the
    oracle's and the device's tables;
  * dct1d_32 of zeros is zeros, of a constant is DC-only within 8, and of a
    sampled sine the DCT-II (AC bins scaled by sqrt 2) within 32
    (dct.rs:4091-4125);
  * forward + quantisation at the finest steps, then the inverse, gives the
    residual back within a few levels;
  * the oracle's leaf32 equals the composition of its primitives.
The oracle writes the inverse in the reference's own forms (constants minus
4096, halved constants with >> 11); the device in single rotations.  GPU
tests compare mt_leaf32 with the oracle bit for bit, at the benchmark
configurations with the default TX_32X32 decision CDFs."""
import math
import os
import re

import numpy as np
import pytest

from maroontree_b200 import abi, synth

INF = float("inf")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _wc32():
    return [int(math.floor(65536.0 / (2.0 * math.cos((2 * k + 1) * math.pi / 64.0)) + 0.5)) for k in range(16)]


def _table(path, name):
    text = open(os.path.join(ROOT, path)).read()
    m = re.search(re.escape(name) + r"\[16\]\s*=\s*\{([^}]*)\}", text)
    return [int(v) for v in re.findall(r"\d+", m.group(1))]


def test_wc32_weights_are_the_formula():
    assert _table("oracle/oracle_chain.cpp", "WC32") == _wc32()
    assert _table("maroontree_b200/csrc/txfm32.cuh", "kWc32") == _wc32()


def test_oracle_dct1d_32_properties(oracle_lib):
    assert np.array_equal(oracle_lib.dct1d_32(np.zeros(32, np.int32)), np.zeros(32, np.int32))
    dc = oracle_lib.dct1d_32(np.full(32, 32, np.int32))
    assert dc[0] != 0 and np.all(np.abs(dc[1:]) <= 8)
    fixed = np.array([int(round(math.sin(i * 0.3) * 128.0)) for i in range(32)], np.int32)
    got = oracle_lib.dct1d_32(fixed)
    # the butterfly's DCT-II: DC the plain sum, each AC bin sqrt(2) x the cosine sum
    n = np.arange(32)
    want = np.array([(1.0 if k == 0 else math.sqrt(2.0)) * np.sum(fixed * np.cos(math.pi * (2 * n + 1) * k / 64.0))
                     for k in range(32)])
    assert np.max(np.abs(got - np.round(want))) <= 32


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_tx32_round_trip(oracle_lib, seed):
    """The finest steps: the inverse of the quantised forward transform is the
    residual within a few levels (at 8 bits, qindex 1 steps 4 / 8)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:32, 0:32]
    resid = np.clip(np.round(60 * np.sin(x * 0.2 + seed) + 40 * np.cos(y * 0.15) + rng.normal(0, 12, (32, 32))),
                    -255, 255).astype(np.int32)
    q = oracle_lib.quant_new(1, 8, 15)
    lv, tf = oracle_lib.fwd_txfm_quant(resid.ravel(), abi.TX_DCT_DCT, q, None)
    back = oracle_lib.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, None)
    err = np.abs(back - resid.ravel())
    assert err.max() <= 4 and err.mean() < 1.5


def _frame(w, h, seed):
    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 19)
    return src, rec


def test_leaf32_oracle_glue(oracle_lib):
    """pick_luma32's candidate (block32.rs:776-836): the 32x32 prediction,
    TX_32X32 DCT_DCT + QM, trellis_optimize_ctx of class 3, the inverse,
    sse_recon, luma_bits with no tx-type symbol + the syntax bits."""
    import maroontree_b200 as mt

    src, rec = _frame(96, 64, 41)
    q = oracle_lib.quant_new(70, 8, 6)
    qm = oracle_lib.qm_row(6, 0, 32)
    c = oracle_lib.default_cdfs(oracle_lib.qcat(70), 32)
    prm = mt.split16_params(96, 64, trellis_lambda0=0.05, rd_lambda=20.0, band_tilt=1.7)
    jobs = synth.leaf8_jobs(96, 64, (abi.DC_PRED, abi.D135_PRED, abi.SMOOTH_PRED, abi.PAETH_PRED), deltas=(0, 2),
                            seed=4, n=32)
    scan = oracle_lib.default_scan(32)
    f32 = np.float32
    res, cf, recs = oracle_lib.leaf32(src, rec, prm, q, qm, c, jobs)
    for i, jb in enumerate(jobs):
        px, py, fl = int(jb["px"]), int(jb["py"]), int(jb["flags"])
        pred = oracle_lib.intra_predict(rec, px, py, 32, 32, int(jb["mode"]), int(jb["angle_delta"]), bool(fl & 1),
                                        bool(fl & 2), bool(fl & 4)).ravel()
        resid = src[py:py + 32, px:px + 32].astype(np.int32).ravel() - pred
        lv, tf = oracle_lib.fwd_txfm_quant(resid, abi.TX_DCT_DCT, q, qm)
        lv = oracle_lib.trellis_optimize_ctx(lv, tf, q, qm, c, int(jb["dcs_ctx"]), 0.05, band_tilt=1.7, n=32)
        rr = oracle_lib.inv_txfm_dequant(lv, abi.TX_DCT_DCT, q, qm)
        sse = int(oracle_lib.sse_recon(src, 96, 64, [(px, py)], pred, rr, 32, 32)[0])
        bits = f32(oracle_lib.real_block_bits_bounded(lv, scan, 32, 32, c, 0, int(jb["dcs_ctx"]), -1, 0, INF))
        assert res["sse"][i] == sse and f32(res["bits"][i]) == bits and np.array_equal(cf[i], lv), i
        assert f32(res["cost"][i]) == f32(f32(sse) + f32(f32(20.0) * f32(bits + f32(jb["syntax_bits"]))))
        assert np.array_equal(recs[i].ravel(), np.clip(pred + rr, 0, 255))
    assert np.count_nonzero(cf) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,wsse", [(70, 6, 0.0), (116, 15, 1.0), (30, 3, 0.75), (1, 15, 0.0)])
def test_leaf32_gpu_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, wsse):
    import maroontree_b200 as mt

    src, rec = _frame(224, 160, qidx + 3)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 32) if qm_level < 15 else None
    c = oracle_lib.default_cdfs(oracle_lib.qcat(qidx), 32)
    jobs = synth.leaf8_jobs(224, 160, range(13), deltas=(-3, 0, 2), seed=qidx, n=32)
    jobs["py"][5] = 144  # crosses the bottom edge: rejected
    prm = mt.split16_params(224, 160, trellis_lambda0=0.05, rd_lambda=0.3 * qidx + 2.0, band_tilt=1.9,
                            wsse_scale=wsse, skip_bits=[(2.5, 0.4)] + [(0.0, 0.0)] * 12, vis=(219, 157))
    res, cf, recs = mt_lib.leaf32(src, rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True, want_rec=True)
    want, wcf, wrec = oracle_lib.leaf32(src, rec, prm, q, qm, c, jobs, threads=os.cpu_count() or 1)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)
    assert res["tx_type"][5] == 255
    assert np.count_nonzero(wcf) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["C1", "C2q40", "C2q60", "C2q80"])
def test_leaf32_at_config(mt_lib, oracle_lib, cuda, name):
    """Every 32x32 block of the benchmark frames with the 13 modes (angle
    deltas -3 / 0 / 3), the configuration's quantiser, QM and lambdas and the
    default TX_32X32 CDFs of its q context."""
    import configs

    wl = configs.workload(name)
    q = wl.q
    qm = configs.qm(mt_lib, wl, 32)
    c = configs.cdfs(mt_lib, wl, 32)
    jobs = synth.leaf8_jobs(wl.w, wl.h, range(13), deltas=(-3, 0, 3), seed=wl.qidx, n=32)
    prm = mt_lib.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.mode_lambda,
                                band_tilt=0.0)
    res, cf, _ = mt_lib.leaf32(wl.src, wl.rec, prm, q, qm, mt_lib.coef_costs(c), jobs, want_cf=True)
    want, wcf, _ = oracle_lib.leaf32(wl.src, wl.rec, prm, q, qm, c, jobs, threads=configs.THREADS)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf)

