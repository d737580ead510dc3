"""GPU parity of the 8x8 candidate chain and its stage kernels against the
oracle: levels, targets, reconstructions, SATD, bits and costs bit-exact."""
import ctypes as C

import numpy as np
import pytest

from maroontree_b200 import abi, synth

pytestmark = pytest.mark.gpu


def _case(oracle_lib, w, h, seed, qidx, qm_level, modes=range(13), types=abi.TX_2D_SCAN_TYPES, deltas=(0,)):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 100)
    cands = synth.level_candidates(w, h, modes, types, deltas=deltas, seed=seed)
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8)
    cdfs = synth.synthetic_cdfs(seed)
    prm = mt.chain_params(w, h, trellis_lambda0=0.05, mode_lambda=float(qidx) * 0.37 + 1.0, satd_scale=1.25,
                          satd_bridge=0.71)
    return src, rec, cands, q, qm, cdfs, prm


def _compare(a, b, la, lb, ra, rb):
    assert la is not None and np.array_equal(la, lb), "levels differ"
    assert np.array_equal(ra, rb), "reconstructions differ"
    for f in ("satd", "eob"):
        assert np.array_equal(a[f], b[f]), f
    for f in ("distortion", "bits", "cost"):
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), f


@pytest.mark.parametrize("qidx,qm_level", [(70, 6), (116, 1), (35, 8), (200, 15), (20, 15)])
def test_chain_host_api_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level):
    src, rec, cands, q, qm, cdfs, prm = _case(oracle_lib, 128, 96, qidx, qidx, qm_level)
    costs = mt_lib.coef_costs(cdfs)
    a, la, ra = mt_lib.candidate_chain(src, rec, prm, q, qm, costs, cands, True, True)
    b, lb, rb = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, True, True, threads=8)
    _compare(a, b, la, lb, ra, rb)


def test_chain_angle_deltas_and_filter_type(mt_lib, oracle_lib, cuda):
    src, rec, cands, q, qm, cdfs, prm = _case(oracle_lib, 96, 64, 9, 70, 6, deltas=(-3, -2, -1, 1, 2, 3))
    cands["flags"] |= np.where(np.arange(len(cands)) % 3 == 0, abi.CAND_FILTER_TYPE, 0).astype(np.uint8)
    costs = mt_lib.coef_costs(cdfs)
    a, la, ra = mt_lib.candidate_chain(src, rec, prm, q, qm, costs, cands, True, True)
    b, lb, rb = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, True, True, threads=8)
    _compare(a, b, la, lb, ra, rb)


def test_chain_v_h_types_and_skip_bits(mt_lib, oracle_lib, cuda):
    import maroontree_b200 as mt

    src, rec, cands, q, qm, cdfs, prm = _case(oracle_lib, 64, 64, 4, 90, 4, types=range(7))
    prm = mt.chain_params(64, 64, trellis_lambda0=0.0, mode_lambda=9.0, skip_bits=(0.7, 1.9))
    costs = mt_lib.coef_costs(cdfs)
    a, la, ra = mt_lib.candidate_chain(src, rec, prm, q, qm, costs, cands, True, True)
    b, lb, rb = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, True, True, threads=8)
    _compare(a, b, la, lb, ra, rb)


def test_chain_extreme_residuals(mt_lib, oracle_lib, cuda):
    """Saturated sources against flat reconstructions: large levels take the
    trellis's scalar (non-FMA) lanes and the Golomb tails of the rate walk."""
    import maroontree_b200 as mt

    rng = np.random.default_rng(3)
    src = (rng.integers(0, 2, size=(64, 64)) * 255).astype(np.uint16)
    rec = np.full((64, 64), 128, np.uint16)
    cands = synth.level_candidates(64, 64, range(13), range(7), seed=3)
    q = oracle_lib.quant_new(1, 8, 15)
    cdfs = synth.synthetic_cdfs(8)
    prm = mt.chain_params(64, 64, trellis_lambda0=0.05, mode_lambda=3.0)
    costs = mt_lib.coef_costs(cdfs)
    a, la, ra = mt_lib.candidate_chain(src, rec, prm, q, None, costs, cands, True, True)
    b, lb, rb = oracle_lib.candidate_chain(src, rec, prm, q, None, cdfs, cands, True, True, threads=8)
    assert np.abs(lb).max() >= 64
    _compare(a, b, la, lb, ra, rb)


def test_chain_device_api_and_empty_batch(mt_lib, oracle_lib, cuda):
    torch = cuda
    src, rec, cands, q, qm, cdfs, prm = _case(oracle_lib, 64, 64, 5, 70, 6)
    costs = mt_lib.coef_costs(cdfs)
    dev = torch.device("cuda:0")
    d_src = torch.from_numpy(src.astype(np.int16)).to(dev)
    d_rec = torch.from_numpy(rec.astype(np.int16)).to(dev)
    d_qm = torch.from_numpy(qm).to(dev)
    d_costs = torch.from_numpy(np.frombuffer(bytes(costs), np.uint8).copy()).to(dev)
    d_cands = torch.from_numpy(cands.view(np.uint8)).to(dev)
    d_res = torch.zeros(len(cands) * abi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    b, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=8)
    mt_lib.candidate_chain_device(d_src, d_rec, prm, q, d_qm, d_costs, d_cands, len(cands), d_res)
    torch.cuda.synchronize()
    assert d_res.cpu().numpy().tobytes() == b.tobytes()
    d_scr = torch.zeros(mt_lib.chain_scratch_bytes(len(cands)), dtype=torch.uint8, device=dev)
    d_res.zero_()
    mt_lib.candidate_chain_device(d_src, d_rec, prm, q, d_qm, d_costs, d_cands, len(cands), d_res, d_scratch=d_scr)
    torch.cuda.synchronize()
    assert d_res.cpu().numpy().tobytes() == b.tobytes()
    mt_lib.candidate_chain_device(d_src, d_rec, prm, q, d_qm, d_costs, d_cands, 0, d_res)


def test_stage_kernels_match_oracle(mt_lib, oracle_lib, cuda):
    torch = cuda
    lib = mt_lib.load()
    rng = np.random.default_rng(12)
    n = 7 * 300
    resid = rng.integers(-255, 256, size=(n, 64)).astype(np.int32)
    resid[::5] //= 16
    types = np.repeat(np.arange(7, dtype=np.uint8), n // 7)
    q = oracle_lib.quant_new(70, 8, 6)
    qm = oracle_lib.qm_row(6, 0, 8)
    dev = torch.device("cuda:0")
    d_r = torch.from_numpy(resid).to(dev)
    d_t = torch.from_numpy(types).to(dev)
    d_qm = torch.from_numpy(qm).to(dev)
    d_lv = torch.zeros((n, 64), dtype=torch.int32, device=dev)
    d_tf = torch.zeros((n, 64), dtype=torch.float32, device=dev)
    d_out = torch.zeros((n, 64), dtype=torch.int32, device=dev)
    assert lib.mt_fwd_txfm_quant_device(d_r.data_ptr(), d_t.data_ptr(), n, 8, C.byref(q), d_qm.data_ptr(),
                                        d_lv.data_ptr(), d_tf.data_ptr(), None) == 0
    lv_gpu, tf_gpu = d_lv.cpu().numpy(), d_tf.cpu().numpy()
    scan = oracle_lib.default_scan(8)
    for i in range(n):
        cf, tf = oracle_lib.fwd_txfm_quant(resid[i], int(types[i]), q, qm)
        assert np.array_equal(cf, lv_gpu[i]) and np.array_equal(tf.view(np.uint32), tf_gpu[i].view(np.uint32)), i
    assert lib.mt_trellis_optimize_device(d_lv.data_ptr(), d_tf.data_ptr(), n, 8, float(q.dc_q), float(q.ac_q),
                                          0.05, None) == 0
    lv_tr = d_lv.cpu().numpy()
    for i in range(n):
        assert np.array_equal(lv_tr[i], oracle_lib.trellis_optimize(lv_gpu[i], tf_gpu[i], q.dc_q, q.ac_q, scan, 0.05)), i
    assert lib.mt_inv_txfm_dequant_device(d_lv.data_ptr(), d_t.data_ptr(), n, 8, C.byref(q), d_qm.data_ptr(),
                                          d_out.data_ptr(), None) == 0
    out = d_out.cpu().numpy()
    for i in range(n):
        assert np.array_equal(out[i], oracle_lib.inv_txfm_dequant(lv_tr[i], int(types[i]), q, qm)), i


def test_intra_predict_kernel_matches_oracle(mt_lib, oracle_lib, cuda):
    torch = cuda
    import maroontree_b200 as mt

    rng = np.random.default_rng(4)
    w, h = 72, 56
    rec = rng.integers(0, 256, size=(h, w)).astype(np.uint16)
    rec[:, 40:] = rec[:, 40:] // 32 * 32
    cands = synth.level_candidates(w, h, range(13), (1,), deltas=(-3, -2, -1, 0, 1, 2, 3), seed=4)
    cands["flags"] = rng.integers(0, 8, size=len(cands)).astype(np.uint8)
    prm = mt.chain_params(w, h)
    dev = torch.device("cuda:0")
    d_rec = torch.from_numpy(rec.astype(np.int16)).to(dev)
    d_c = torch.from_numpy(cands.view(np.uint8)).to(dev)
    d_o = torch.zeros((len(cands), 64), dtype=torch.int32, device=dev)
    assert mt_lib.load().mt_intra_predict_device(d_rec.data_ptr(), C.byref(prm), d_c.data_ptr(), len(cands),
                                                 d_o.data_ptr(), None) == 0
    out = d_o.cpu().numpy()
    for i, c in enumerate(cands):
        ref = oracle_lib.intra_predict(rec, int(c["px"]), int(c["py"]), 8, 8, int(c["mode"]), int(c["angle_delta"]),
                                       c["flags"] & 1, c["flags"] & 2, c["flags"] & 4)
        assert np.array_equal(out[i], ref.ravel()), (i, c)
