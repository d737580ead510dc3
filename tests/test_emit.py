"""Coefficient token emission (mt_emit_coeffs, the square coefficient coders
of src/coeffs.rs) against the oracle's restatement, token for token, over
random transform blocks of every size, plane and context: all-zero blocks,
DC-only blocks, large levels that reach the Golomb tail, dense blocks; and the
CDF slot layout the tokens name against the oracle's own assembly."""
import numpy as np
import pytest

from maroontree_b200 import abi
from maroontree_b200 import entropy as en


def test_slot_layout_matches_oracle(mt_lib, oracle_lib):
    L = en.cdf_layout()
    _, sec = oracle_lib.emit_slots()
    for k in range(4):
        assert L.txb_skip[k] == sec[f"txb_skip{k}"]
        for p in range(2):
            assert L.base_tok[k][p] == sec[f"base_tok{k}{p}"]
            assert L.br_tok[k][p] == sec[f"br_tok{k}{p}"]
            assert L.eob_base[k][p] == sec[f"eob_base{k}{p}"]
            assert L.eob_hi[k][p] == sec[f"eob_hi{k}{p}"]
    assert L.txb_skip[4] == sec["txb_skip4"] and L.base_tok[4][0] == sec["base_tok40"]
    assert L.base_tok[4][1] == -1 and L.eob_base[4][1] == -1 and L.eob_hi[4][1] == -1
    assert (L.dc_sign[0], L.dc_sign[1], L.eob_bin) == (sec["dc_sign0"], sec["dc_sign1"], sec["eob_bin"])
    assert (L.txtp4, L.txtp8, L.txtp16) == (sec["txtp4"], sec["txtp8"], sec["txtp16"])
    for name in ("skip", "part_bl8", "part_split", "kf_y", "uv_mode", "palette_y_mode", "palette_uv_mode", "txsz"):
        assert getattr(L, name) == sec[name], name
    assert L.nslots == mt_lib.load().mt_cdf_slot_count()


def random_blocks(seed, nblocks=600):
    rng = np.random.default_rng(seed)
    blocks = np.zeros(nblocks, abi.COEF_BLOCK_DTYPE)
    levels = []
    off = 0
    for i in range(nblocks):
        lg = int(rng.integers(2, 5))
        n = 1 << lg
        kind = i % 6
        cf = np.zeros(n * n, np.int32)
        if kind == 1:  # DC only
            cf[0] = int(rng.integers(-40, 41)) or 1
        elif kind == 2:  # a few low-frequency coefficients
            for _ in range(int(rng.integers(1, 6))):
                cf[int(rng.integers(0, min(n * n, 20)))] = int(rng.integers(-3, 4))
        elif kind == 3:  # dense, Golomb tails
            mask = rng.random(n * n) < 0.6
            cf[mask] = rng.integers(-400, 401, mask.sum())
        elif kind == 4:  # sparse, anywhere
            mask = rng.random(n * n) < 0.08
            cf[mask] = rng.integers(-20, 21, mask.sum())
        elif kind == 5:  # one huge coefficient
            cf[int(rng.integers(0, n * n))] = int(rng.choice([-1, 1])) * int(rng.integers(15, 9000))
        plane = int(rng.integers(0, 2))
        blocks[i] = (off, lg, plane, int(rng.integers(0, 13)), int(rng.integers(0, 3)), int(rng.integers(0, 13)),
                     int(rng.integers(0, 5 if lg == 4 else 7)), int(plane == 0 and rng.random() < 0.8), 0)
        levels.append(cf)
        off += n * n
    return np.concatenate(levels), blocks


def test_oracle_emission_structure(oracle_lib):
    """Oracle sanity: an all-zero block is one all_zero = 1 symbol; a DC-only
    luma block codes all_zero, the tx type, eob_pt 0, the DC base and sign."""
    cf = np.zeros(64, np.int32)
    b = np.zeros(2, abi.COEF_BLOCK_DTYPE)
    b[0] = (0, 3, 0, 0, 1, 0, 1, 1, 0)
    b[1] = (64, 3, 0, 0, 1, 0, 1, 1, 0)
    cf2 = cf.copy()
    cf2[0] = -2
    toks, off, res = oracle_lib.emit_coeffs(np.concatenate([cf, cf2]), b)
    e, _ = oracle_lib.emit_slots()
    assert list(toks[:1]) == [(e.txb_skip[1] << 8) | 1] and res[0] == 0x40
    t = list(toks[off[1]:off[2]])
    assert t[0] == (e.txb_skip[1] << 8) | 0 and t[1] == (e.txtp8 << 8) | 1
    assert t[2] == ((e.eob_bin + 4) << 8) | 0 and t[3] == (e.eob_base[1][0] << 8) | 1
    assert t[4] == ((e.dc_sign[0] + 1) << 8) | 1 and len(t) == 5 and res[1] == 2


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_emission_matches_oracle(mt_lib, oracle_lib, cuda, seed):
    levels, blocks = random_blocks(seed)
    got = en.emit_coeffs(levels, blocks)
    want = oracle_lib.emit_coeffs(levels, blocks)
    assert np.array_equal(got[1], want[1])
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[2], want[2])
