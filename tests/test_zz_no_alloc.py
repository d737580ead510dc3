"""The allocation-free level entry point (mt_rdo_level8_device_noalloc).

It serves callers that cannot let this library allocate device memory -- a
GPU-memory budget owned by another framework's pool, or a real-time thread
that must not enter the driver's allocator.  The test calls it through the C
ABI twice in a row, on two different levels (the second smaller than the
first, so stale keys left in the shared device array would show), and checks
each per-block result bit-for-bit against mt_rdo_level8_device, which takes
its working storage from the caller.  This file sorts last so a run that stops
at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from maroontree_b200 import abi, synth

pytestmark = pytest.mark.gpu


def _level(oracle_lib, w, h, seed, qidx, qm_level, vis=None):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 3)
    blocks = synth.level_blocks(w, h, seed=seed)
    combos = synth.level_combos(range(13), abi.TX_2D_SCAN_TYPES, deltas=(-3, 0, 3),
                                delta_bits=lambda m, d: 0.25 + 0.125 * abs(d))
    q = oracle_lib.quant_new(qidx, 8, qm_level)
    qm = oracle_lib.qm_row(qm_level, 0, 8)
    costs = mt.coef_costs(synth.synthetic_cdfs(seed))
    prm = mt.chain_params(w, h, trellis_lambda0=0.05, mode_lambda=0.3 * qidx + 2.0, satd_bridge=0.8, vis=vis)
    return src, rec, blocks, combos, q, qm, costs, prm


def _run_both(mt_lib, torch, case):
    src, rec, blocks, combos, q, qm, costs, prm = case
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_src, d_rec, d_qm = t(src), t(rec), t(qm)
    d_costs, d_blocks, d_combos = t(np.frombuffer(bytes(costs), np.uint8)), t(blocks), t(combos)
    nb, nc = len(blocks), len(combos)
    # existing entry point: caller-provided working storage
    d_best_ref = torch.zeros(nb * abi.BEST_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_res = torch.zeros(nb * nc * abi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_keys = torch.zeros(mt_lib.rdo_level8_scratch_bytes(nb, nc), dtype=torch.uint8, device=dev)
    mt_lib.rdo_level8_device(d_src, d_rec, prm, q, d_qm, d_costs, d_blocks, nb, d_combos, nc, d_best_ref, d_res,
                             d_keys)
    # allocation-free entry point, called through the C ABI
    d_best = torch.full((nb * abi.BEST_DTYPE.itemsize,), 0x5A, dtype=torch.uint8, device=dev)
    rc = mt_lib.load().mt_rdo_level8_device_noalloc(
        d_src.data_ptr(), d_rec.data_ptr(), C.byref(prm), C.byref(q), d_qm.data_ptr(), d_costs.data_ptr(),
        d_blocks.data_ptr(), nb, d_combos.data_ptr(), nc, d_best.data_ptr(), None)
    assert rc == abi.MT_OK
    torch.cuda.synchronize()
    ref = d_best_ref.cpu().numpy().view(abi.BEST_DTYPE)
    got = d_best.cpu().numpy().view(abi.BEST_DTYPE)
    return ref, got


def test_noalloc_level_matches_level_entry_point_twice(mt_lib, oracle_lib, cuda):
    first = _level(oracle_lib, 128, 96, 21, 70, 6)
    second = _level(oracle_lib, 64, 64, 22, 116, 1)
    for case in (first, second):
        ref, got = _run_both(mt_lib, cuda, case)
        assert np.all(ref["combo"] >= 0)
        assert got.tobytes() == ref.tobytes()


def test_noalloc_displayed_window_matches_level_entry_point(mt_lib, oracle_lib, cuda):
    """A frame displayed smaller than it is coded takes the masked kernel form."""
    case = _level(oracle_lib, 96, 64, 24, 70, 6, vis=(91, 59))
    ref, got = _run_both(mt_lib, cuda, case)
    assert np.all(ref["combo"] >= 0)
    assert got.tobytes() == ref.tobytes()


def test_noalloc_checks_match_level_entry_point(mt_lib, oracle_lib, cuda):
    """Same input errors and codes as mt_rdo_level8_device (no device work)."""
    src, rec, blocks, combos, q, qm, costs, prm = _level(oracle_lib, 64, 64, 25, 70, 6)
    lib = mt_lib.load()
    for nb, nc in ((70000, 40000), (4, abi.MT_LEVEL_MAX_COMBOS + 1), (-1, 3)):
        a = lib.mt_rdo_level8_device(1, 1, C.byref(prm), C.byref(q), None, 1, 1, nb, 1, nc, 1, 1, 1, None)
        b = lib.mt_rdo_level8_device_noalloc(1, 1, C.byref(prm), C.byref(q), None, 1, 1, nb, 1, nc, 1, None)
        assert a == b != abi.MT_OK, (nb, nc, a, b)


def test_noalloc_rejects_more_blocks_than_its_array(mt_lib, oracle_lib, cuda):
    src, rec, blocks, combos, q, qm, costs, prm = _level(oracle_lib, 64, 64, 23, 70, 6)
    rc = mt_lib.load().mt_rdo_level8_device_noalloc(
        1, 1, C.byref(prm), C.byref(q), None, 1, 1, abi.MT_NOALLOC_MAX_BLOCKS + 1, 1, len(combos), 1, None)
    assert rc == abi.MT_ERR_TOO_LARGE
