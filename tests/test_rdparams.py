"""Frame-level laws of the library against a float32 restatement written
here from the reference's sources, bit for bit over every qindex: quality ->
qindex (src/avif.rs:637-666), the QM level laws (src/quant.rs:122-167, with the
reference's own known answers from its tests at src/quant.rs:466-480) and the
decision lambdas (src/cost.rs:122-148, :286-292, src/partition_rd.rs:30-71,
src/coder/lossy_state.rs:1769-1789, :2396-2408), against the oracle's float32
restatement (oracle/pyoracle.py) bit for bit over every qindex.  No device
call."""
import numpy as np
import pytest

def test_quality_to_q_anchors_and_monotone(mt_lib, oracle_lib):
    assert (mt_lib.quality_to_q(40), mt_lib.quality_to_q(60), mt_lib.quality_to_q(80)) == (116, 70, 35)
    assert mt_lib.quality_to_q(100) == 1 and mt_lib.quality_to_q(0) == 215 and mt_lib.quality_to_q(1) == 215
    qs = [mt_lib.quality_to_q(v) for v in range(1, 101)]
    assert all(a >= b for a, b in zip(qs, qs[1:]))
    # linear between anchors: quality 35 sits halfway between (30, 140) and (40, 116)
    assert mt_lib.quality_to_q(35) == 140 + (116 - 140) * 5 // 10
    assert [mt_lib.quality_to_q(v) for v in range(256)] == [oracle_lib.quality_to_q(v) for v in range(256)]


def test_qm_levels_match_restatement(mt_lib, oracle_lib):
    for sub in (0, 1, 2):
        for q in range(256):
            assert mt_lib.qm_levels(q, sub) == (oracle_lib.qm_level_law(q, sub), oracle_lib.qm_chroma_level_law(q, sub)), (q, sub)
    # the reference's own cases (src/quant.rs:466-480)
    for sub in (1, 2):
        for qi in (20, 12, 7, 1):
            assert mt_lib.qm_levels(qi, sub)[0] == 8
    assert mt_lib.qm_levels(7, 0) == (15, 15)
    assert mt_lib.qm_levels(12, 0)[1] == 2
    # the configs: 4:4:4 q60 and 4:2:0 q40 / q60 / q80
    assert mt_lib.qm_levels(70, 0)[0] == 6
    assert [mt_lib.qm_levels(q, 2)[0] for q in (116, 70, 35)] == [1, 6, 8]


@pytest.mark.parametrize("sub", [0, 1, 2])
def test_lambdas_match_restatement(mt_lib, oracle_lib, sub):
    for q in range(256):
        dcq = int(mt_lib.quant_new(q, 8, 15).dc_q)
        assert bytes(mt_lib.rd_lambdas(q, dcq, sub)) == bytes(oracle_lib.rd_lambdas(q, dcq, sub)), q
    # mlam at qindex 70 4:2:0 for a DC step of 85: mode_lambda_q x the ramped weight, by hand
    got = mt_lib.rd_lambdas(70, 85, 2)
    w = (3.0 + ((72 + 128) / 128 - 3.0) * 70 / 72) * 0.8
    assert abs(got.mode_lambda - 0.009005174719460433 * 85 * 85 * (3.3 + 0.0015 * 85) * w) < 1e-3


def test_lambdas_reject(mt_lib):
    from maroontree_b200 import MtError, abi

    with pytest.raises(MtError) as e:
        mt_lib.rd_lambdas(70, 100, 2, bd=10)
    assert e.value.code == abi.MT_ERR_UNSUPPORTED
    with pytest.raises(MtError):
        mt_lib.rd_lambdas(70, 0, 2)
