"""The proxy's mode beam (proxy_mode_beam's ranking): the oracle's scores equal
a numpy restatement of satd_sad_proxy (src/rd_sse.rs:1143-1176) over the
oracle's predictions, the ranking is the (score, mode) order of the 11
nd_modes, and the CUDA beam equals the oracle for 4x4, 8x8 and 16x16 blocks,
with and without a clipped displayed frame."""
import numpy as np
import pytest

from maroontree_b200 import abi, synth

ND = [abi.DC_PRED, abi.V_PRED, abi.H_PRED, abi.D45_PRED, abi.D135_PRED, abi.D113_PRED, abi.D157_PRED,
      abi.D203_PRED, abi.D67_PRED, abi.SMOOTH_PRED, abi.PAETH_PRED]


def _proxy_np(d):
    """SAD + (SATD >> 2) over 4x4 Hadamard tiles of the residual d (int64)."""
    sad = int(np.abs(d).sum())
    h4 = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]], np.int64)
    satd = 0
    for ty in range(0, d.shape[0], 4):
        for tx in range(0, d.shape[1], 4):
            t = d[ty:ty + 4, tx:tx + 4].astype(np.int64)
            satd += int(np.abs(h4 @ t @ h4.T).sum())
    return sad + (satd >> 2)


def _setup(n, w=96, h=64, seed=3, vis=None):
    import maroontree_b200 as mt

    src = synth.rgb_to_luma(synth.generate_rgb(w, h, seed))
    rec = synth.synthetic_recon(src, seed + 5)
    blocks = synth.level_blocks(w, h, n=n, seed=seed)
    prm = mt.chain_params(w, h, tx_size=n, vis=vis)
    return src, rec, blocks, prm


@pytest.mark.parametrize("n", [4, 8, 16])
def test_oracle_beam_scores_and_order(oracle_lib, n):
    src, rec, blocks, prm = _setup(n)
    scores, modes = oracle_lib.mode_beam(src, rec, prm, blocks)
    for b in range(0, len(blocks), max(1, len(blocks) // 7)):
        bk = blocks[b]
        want = []
        for m in ND:
            pred = oracle_lib.intra_predict(rec, int(bk["px"]), int(bk["py"]), n, n, m, 0,
                                            have_tr=bool(bk["flags"] & 1), have_bl=bool(bk["flags"] & 2),
                                            filter_type=bool(bk["flags"] & 4)).reshape(n, n)
            d = src[bk["py"]:bk["py"] + n, bk["px"]:bk["px"] + n].astype(np.int64) - pred
            want.append((_proxy_np(d), m))
        want.sort()
        assert [s for s, _ in want] == scores[b].tolist()
        assert [m for _, m in want] == modes[b].tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("n,vis", [(4, None), (8, None), (16, None), (8, (93, 61)), (16, (90, 55)), (4, (95, 63))])
def test_mode_beam_matches_oracle(mt_lib, oracle_lib, cuda, n, vis):
    src, rec, blocks, prm = _setup(n, 160, 96, 7, vis)
    ref_s, ref_m = oracle_lib.mode_beam(src, rec, prm, blocks)
    got_s, got_m = mt_lib.mode_beam(src, rec, prm, blocks)
    assert np.array_equal(got_s, ref_s) and np.array_equal(got_m, ref_m)
