"""GPU parity of the batched RDO level (mt_rdo_level8): every candidate result
bit-exact against the oracle and the per-block winner equal to the first
minimum in evaluation order."""
import numpy as np
import pytest

from maroontree_b200 import abi, synth




def _setup(oracle_lib, w, h, seed, qidx, qm_level, types=abi.TX_2D_SCAN_TYPES, deltas=(0,)):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 7)
    blocks = synth.level_blocks(w, h, seed=seed)
    # nonzero deltas carry an angle-delta symbol cost, as in the proxy's delta pass
    combos = synth.level_combos(range(13), types, deltas, delta_bits=lambda m, d: 0.375 + 0.1 * m + 0.05 * abs(d))
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8)
    cdfs = synth.synthetic_cdfs(seed + 1)
    prm = mt.chain_params(w, h, trellis_lambda0=0.05, mode_lambda=0.3 * qidx + 2.0, satd_scale=1.25, satd_bridge=0.8)
    return src, rec, blocks, combos, q, qm, cdfs, prm


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm_level,deltas", [(70, 6, (0,)), (116, 1, (-3, 0, 3)), (30, 8, (-1, 0, 2))])
def test_level_matches_oracle(mt_lib, oracle_lib, cuda, qidx, qm_level, deltas):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup(oracle_lib, 160, 96, qidx, qidx, qm_level, deltas=deltas)
    best, res = mt_lib.rdo_level8(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    cands = synth.candidates_of_level(blocks, combos)
    ref, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=8)
    assert res.tobytes() == ref.tobytes()
    win = synth.best_of_level(ref, len(blocks), len(combos))
    assert np.array_equal(best["combo"], win)
    ref_w = ref.reshape(len(combos), len(blocks))[win, np.arange(len(blocks))]
    assert np.array_equal(best["cost"].view(np.uint32), ref_w["cost"].view(np.uint32))
    assert np.array_equal(best["bits"].view(np.uint32), ref_w["bits"].view(np.uint32))
    assert np.array_equal(best["eob"], ref_w["eob"])


@pytest.mark.gpu
def test_level_ties_pick_first_combo(mt_lib, oracle_lib, cuda):
    """A flat source and reconstruction make many combos cost the same; the
    winner must be the first of them (strict < in evaluation order)."""
    import maroontree_b200 as mt

    w, h = 64, 64
    src = np.full((h, w), 117, np.uint16)
    rec = np.full((h, w), 117, np.uint16)
    blocks = synth.level_blocks(w, h, seed=2)
    blocks["mode_bits"] = 3.0
    combos = synth.level_combos(range(13), abi.TX_2D_SCAN_TYPES)
    q = oracle_lib.quant_new(70, 8, 15)
    cdfs = synth.synthetic_cdfs(3)
    prm = mt.chain_params(w, h, mode_lambda=5.0)
    best, res = mt_lib.rdo_level8(src, rec, prm, q, None, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    win = synth.best_of_level(res, len(blocks), len(combos))
    assert np.array_equal(best["combo"], win)


@pytest.mark.gpu
def test_level_device_api_matches_host(mt_lib, oracle_lib, cuda):
    torch = cuda
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup(oracle_lib, 96, 64, 5, 70, 6)
    costs = mt_lib.coef_costs(cdfs)
    host_best, host_res = mt_lib.rdo_level8(src, rec, prm, q, qm, costs, blocks, combos, want_results=True)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_best = torch.zeros(len(blocks) * abi.BEST_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_res = torch.zeros(len(blocks) * len(combos) * abi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_keys = torch.zeros(mt_lib.rdo_level8_scratch_bytes(len(blocks), len(combos)), dtype=torch.uint8, device=dev)
    mt_lib.rdo_level8_device(t(src), t(rec), prm, q, t(qm), t(np.frombuffer(bytes(costs), np.uint8)), t(blocks),
                             len(blocks), t(combos), len(combos), d_best, d_res, d_keys)
    torch.cuda.synchronize()
    assert d_best.cpu().numpy().tobytes() == host_best.tobytes()
    assert d_res.cpu().numpy().tobytes() == host_res.tobytes()


@pytest.mark.gpu
def test_level_rejects_out_of_frame_blocks(mt_lib, oracle_lib, cuda):
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup(oracle_lib, 64, 64, 6, 70, 6)
    blocks = blocks.copy()
    blocks["px"][3] = 60  # crosses the right edge
    best, res = mt_lib.rdo_level8(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    r = res.reshape(len(combos), len(blocks))
    assert np.all(r[:, 3]["eob"] == abi.MT_EOB_INVALID)
    assert best["combo"][3] == -1
    assert np.all(best["combo"][np.arange(len(blocks)) != 3] >= 0)


def test_extra_bits_follow_mode_bits_in_oracle(oracle_lib):
    """bits = (luma_bits + mode_bits) + extra_bits, and extra_bits 0 changes nothing."""
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup(oracle_lib, 64, 64, 3, 70, 6, deltas=(-2, 0, 2))
    cands = synth.candidates_of_level(blocks, combos)
    with_bits, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=4)
    plain = cands.copy()
    plain["extra_bits"] = 0.0
    without, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, plain, threads=4)
    nz = cands["extra_bits"] != 0
    assert nz.any() and (~nz).any()
    assert np.array_equal(with_bits["bits"][~nz].view(np.uint32), without["bits"][~nz].view(np.uint32))
    exp = (without["bits"][nz] + cands["extra_bits"][nz]).astype(np.float32)
    assert np.array_equal(with_bits["bits"][nz].view(np.uint32), exp.view(np.uint32))


@pytest.mark.gpu
def test_level_masks_samples_past_the_displayed_frame(mt_lib, oracle_lib, cuda):
    """A frame displayed at 157x93 and coded at 160x96: the right / bottom
    blocks price distortion over the displayed samples only (SrcBlock)."""
    src, rec, blocks, combos, q, qm, cdfs, prm = _setup(oracle_lib, 160, 96, 9, 70, 6, deltas=(-2, 0, 2))
    prm.vis_w, prm.vis_h = 157, 93
    best, res = mt_lib.rdo_level8(src, rec, prm, q, qm, mt_lib.coef_costs(cdfs), blocks, combos, want_results=True)
    cands = synth.candidates_of_level(blocks, combos)
    ref, _, _ = oracle_lib.candidate_chain(src, rec, prm, q, qm, cdfs, cands, threads=8)
    assert res.tobytes() == ref.tobytes()
    full = prm.__class__.from_buffer_copy(prm)
    full.vis_w = full.vis_h = 0
    ref_full, _, _ = oracle_lib.candidate_chain(src, rec, full, q, qm, cdfs, cands, threads=8)
    edge = (cands["px"] + 8 > 157) | (cands["py"] + 8 > 93)
    assert (ref["satd"][edge] != ref_full["satd"][edge]).any()
    assert np.array_equal(ref["satd"][~edge], ref_full["satd"][~edge])
