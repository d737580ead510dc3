"""GPU parity at the benchmark configurations (C1 512x512 4:4:4 q60, C2
1920x1080 4:2:0 q40 / q60 / q80, tests/configs.py): every RDO kernel family
over every block of the frame, with the quantiser, QM level and lambdas of the
config's laws and the default decision CDFs Cdfs::new(qcat(qindex)) of the
library (pinned against the reference's arrays in test_default_cdfs.py),
compared bit for bit with the oracle on all host cores."""
import numpy as np
import pytest

from configs import NAMES, THREADS, cdfs, qm, workload
from maroontree_b200 import abi, synth

MODES = range(13)
DELTAS = (-3, 0, 3)
pytestmark = pytest.mark.gpu


def _delta_bits(m, d):
    return 0.375 + 0.1 * m + 0.05 * abs(d)


def _chain_prm(mt, wl, n):
    return mt.chain_params(wl.w, wl.h, tx_size=n, trellis_lambda0=wl.lam.trellis_lambda0,
                           mode_lambda=wl.lam.mode_lambda, satd_scale=wl.lam.satd_scale,
                           satd_bridge=wl.lam.satd_bridge)


def _check_level(mt_lib, oracle_lib, wl, n, combos, fn):
    blocks = synth.level_blocks(wl.w, wl.h, n=n, seed=wl.qidx)
    c = cdfs(mt_lib, wl, n)
    prm = _chain_prm(mt_lib, wl, n)
    best, res = fn(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, n), mt_lib.coef_costs(c), blocks, combos,
                   want_results=True)
    cands = synth.candidates_of_level(blocks, combos)
    ref, _, _ = oracle_lib.candidate_chain(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, n), c, cands, threads=THREADS)
    assert res.tobytes() == ref.tobytes()
    win = synth.best_of_level(ref, len(blocks), len(combos))
    assert np.array_equal(best["combo"], win)
    return best


@pytest.mark.parametrize("cfg", NAMES)
def test_level8_at_config(mt_lib, oracle_lib, cuda, cfg):
    wl = workload(cfg)
    combos = synth.level_combos(MODES, abi.TX_2D_SCAN_TYPES, DELTAS, delta_bits=_delta_bits)
    best = _check_level(mt_lib, oracle_lib, wl, 8, combos, mt_lib.rdo_level8)
    assert len(np.unique(best["combo"])) > 20


@pytest.mark.parametrize("cfg", NAMES)
def test_level4_at_config(mt_lib, oracle_lib, cuda, cfg):
    wl = workload(cfg)
    combos = synth.level_combos(MODES, (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX, abi.TX_ADST_DCT,
                                        abi.TX_DCT_ADST), no_trellis_types=(abi.TX_IDTX,))
    _check_level(mt_lib, oracle_lib, wl, 4, combos, mt_lib.rdo_level4)


@pytest.mark.parametrize("cfg", NAMES)
def test_level16_at_config(mt_lib, oracle_lib, cuda, cfg):
    wl = workload(cfg)
    combos = synth.level_combos(MODES, (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX), DELTAS,
                                delta_bits=_delta_bits)
    _check_level(mt_lib, oracle_lib, wl, 16, combos, mt_lib.rdo_level16)


def _leaf_prm(mt, wl, search):
    return mt.split16_params(wl.w, wl.h, trellis_lambda0=wl.lam.trellis_lambda0, rd_lambda=wl.lam.lambda_d,
                             band_tilt=1.9, wsse_scale=1.0, tx_search=search, tx_guard_shift=5 if search else 4)


@pytest.mark.parametrize("cfg", NAMES)
@pytest.mark.parametrize("refine", [False, True])
def test_leaf8_at_config(mt_lib, oracle_lib, cuda, cfg, refine):
    wl = workload(cfg)
    c = cdfs(mt_lib, wl, 8)
    jobs = synth.leaf8_jobs(wl.w, wl.h, [abi.PAETH_PRED, abi.D157_PRED] if refine else MODES, seed=wl.qidx)
    prm = _leaf_prm(mt_lib, wl, wl.sub == 0)
    res, cf, recs = mt_lib.leaf8(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, 8), mt_lib.coef_costs(c), jobs,
                                 refine=refine, want_cf=True, want_rec=True)
    want, wcf, wrec = oracle_lib.leaf8(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, 8), c, jobs, refine=refine,
                                       threads=THREADS)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)


@pytest.mark.parametrize("cfg", NAMES)
@pytest.mark.parametrize("refine", [False, True])
def test_leaf16_at_config(mt_lib, oracle_lib, cuda, cfg, refine):
    wl = workload(cfg)
    c = cdfs(mt_lib, wl, 16)
    jobs = synth.leaf8_jobs(wl.w, wl.h, [abi.SMOOTH_PRED] if refine else MODES, seed=wl.qidx, n=16)
    prm = _leaf_prm(mt_lib, wl, False)
    res, cf, recs = mt_lib.leaf16(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, 16), mt_lib.coef_costs(c), jobs,
                                  refine=refine, want_cf=True, want_rec=True)
    want, wcf, wrec = oracle_lib.leaf16(wl.src, wl.rec, prm, wl.q, qm(mt_lib, wl, 16), c, jobs, refine=refine,
                                        threads=THREADS)
    assert res.tobytes() == want.tobytes()
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)


@pytest.mark.parametrize("cfg", NAMES)
@pytest.mark.parametrize("kind", ["split16", "depth2", "split4tx"])
def test_split_trials_at_config(mt_lib, oracle_lib, cuda, cfg, kind):
    wl = workload(cfg)
    n_tx = 8 if kind == "split16" else 4
    c = cdfs(mt_lib, wl, n_tx)
    jobs = synth.split16_jobs(wl.w, wl.h, MODES, seed=wl.qidx, n=8 if kind == "split4tx" else 16)
    search = kind == "split16" and wl.sub == 0
    prm = _leaf_prm(mt_lib, wl, search)
    q_m = qm(mt_lib, wl, n_tx)
    costs = mt_lib.coef_costs(c)
    if kind == "split16":
        res, cf, recs = mt_lib.split16_luma(wl.src, wl.rec, prm, wl.q, q_m, costs, jobs, want_cf=True, want_rec=True)
        want, wcf, wrec = oracle_lib.split16_luma(wl.src, wl.rec, prm, wl.q, q_m, c, jobs, threads=THREADS)
    elif kind == "depth2":
        res, cf, recs = mt_lib.split16_depth2(wl.src, wl.rec, prm, wl.q, q_m, costs, jobs, want_cf=True,
                                              want_rec=True)
        want, wcf, wrec = oracle_lib.split16_depth2(wl.src, wl.rec, prm, wl.q, q_m, c, jobs, threads=THREADS)
    else:
        res, cf, recs = mt_lib.split4tx(wl.src, wl.rec, prm, wl.q, q_m, costs, jobs, want_cf=True, want_rec=True)
        want, wcf, wrec = oracle_lib.split4tx(wl.src, wl.rec, prm, wl.q, q_m, c, jobs, threads=THREADS)
    bad = (res.view(np.uint8).reshape(len(jobs), -1) != want.view(np.uint8).reshape(len(jobs), -1)).any(axis=1)
    assert not bad.any(), np.nonzero(bad)[0][:5]
    assert np.array_equal(cf, wcf) and np.array_equal(recs, wrec)


@pytest.mark.parametrize("cfg", NAMES)
@pytest.mark.parametrize("n", [4, 8, 16])
def test_mode_beam_at_config(mt_lib, oracle_lib, cuda, cfg, n):
    wl = workload(cfg)
    prm = _chain_prm(mt_lib, wl, n)
    blocks = synth.level_blocks(wl.w, wl.h, n=n, seed=wl.qidx)
    got = mt_lib.mode_beam(wl.src, wl.rec, prm, blocks)
    want = oracle_lib.mode_beam(wl.src, wl.rec, prm, blocks)
    for a, b in zip(got, want):
        assert np.asarray(a).tobytes() == np.asarray(b).tobytes()
