"""CPU-side checks of the C ABI library: it loads, exports every symbol the
public header declares, and its host helpers (quantiser set-up, QM rows,
scans, CDF bit costs) agree exactly with the oracle.  No device call."""
import os
import re

import numpy as np
import pytest

from maroontree_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "maroontree_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mt_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol(mt_lib):
    lib = mt_lib.load()
    names = header_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(abi.EXPORTED_SYMBOLS)


def test_version(mt_lib):
    assert b"sm_100a" in mt_lib.load().mt_version()


@pytest.mark.parametrize("qidx,level", [(1, 15), (35, 8), (70, 6), (116, 1), (255, 0)])
def test_quant_init_matches_oracle(mt_lib, oracle_lib, qidx, level):
    a = mt_lib.quant_new(qidx, 8, level)
    b = oracle_lib.quant_new(qidx, 8, level)
    assert bytes(a) == bytes(b)
    a = mt_lib.quant_new_chroma(qidx, -5, 12, 8, level)
    b = oracle_lib.quant_new_chroma(qidx, -5, 12, 8, level)
    assert bytes(a) == bytes(b)


def test_quant_rejects_high_bit_depth(mt_lib):
    from maroontree_b200 import MtError

    with pytest.raises(MtError) as e:
        mt_lib.quant_new(70, 10, 6)
    assert e.value.code == abi.MT_ERR_UNSUPPORTED


def test_qm_rows_and_scans_match_oracle(mt_lib, oracle_lib):
    for n in (4, 8, 16, 32):
        assert np.array_equal(mt_lib.default_scan(n), oracle_lib.default_scan(n))
        assert sorted(mt_lib.default_scan(n)) == list(range(n * n))
        for lvl in (0, 6, 14, 15):
            for ch in (0, 1):
                a, b = mt_lib.qm_row(lvl, ch, n), oracle_lib.qm_row(lvl, ch, n)
                assert (a is None) == (b is None)
                if a is not None:
                    assert np.array_equal(a, b)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_coef_costs_match_oracle(mt_lib, oracle_lib, seed):
    from maroontree_b200 import synth

    cdfs = synth.synthetic_cdfs(seed)
    assert bytes(mt_lib.coef_costs(cdfs)) == bytes(oracle_lib.coef_costs(cdfs))


def test_chain_rejects_bad_sizes_without_device(mt_lib):
    """Argument validation happens before any device call."""
    from maroontree_b200 import MtError

    prm = mt_lib.chain_params(64, 64, tx_size=12)
    q = mt_lib.quant_new(70)
    costs = abi.CoefCosts()
    src = np.zeros((64, 64), np.uint16)
    cands = np.zeros(1, abi.CANDIDATE_DTYPE)
    with pytest.raises(MtError) as e:
        mt_lib.candidate_chain(src, src, prm, q, None, costs, cands)
    assert e.value.code == abi.MT_ERR_UNSUPPORTED
    prm = mt_lib.chain_params(64, 64, stride=32)
    with pytest.raises(MtError) as e:
        mt_lib.candidate_chain(src, src, prm, q, None, costs, cands)
    assert e.value.code == abi.MT_ERR_INVALID_INPUT
