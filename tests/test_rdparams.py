"""Frame-level laws of the library against a float32 restatement written
here from the reference's sources, bit for bit over every qindex: quality ->
qindex (src/avif.rs:637-666), the QM level laws (src/quant.rs:122-167, with the
reference's own known answers from its tests at src/quant.rs:466-480) and the
decision lambdas (src/cost.rs:122-148, :286-292, src/partition_rd.rs:30-71,
src/coder/lossy_state.rs:1769-1789, :2396-2408).  No device call."""
import numpy as np
import pytest

f32 = np.float32


def fast_round(v):
    b = np.array([v], f32).view(np.uint32) + np.uint32(1)
    u = b.view(f32)[0]
    magic = f32((1 << 23) + (1 << 22))
    return f32(f32(u + magic) - magic)


def qm_level_law(q, sub):
    qi = f32(q)
    top = f32(8.0) if sub else f32(15.0)
    if qi <= 20:
        return 8 if sub else 15
    if qi <= 48:
        return int(fast_round(f32(top + f32(f32((f32(8.0) - top) * f32(qi - f32(20.0))) / f32(28.0)))))
    if qi >= 128:
        return 0
    return int(fast_round(f32(f32(f32(8.0) * f32(f32(128.0) - qi)) / f32(80.0))))


def qm_chroma_level_law(q, sub):
    if sub:
        return qm_level_law(q, sub)
    pinned = min(2, qm_level_law(q, sub))
    t = f32(np.clip(f32(f32(f32(12.0) - f32(q)) / f32(5.0)), 0, 1))
    if t > 0:
        v = f32(f32(pinned) + f32(f32(f32(15.0) - f32(pinned)) * t))
        return int(np.floor(v + 0.5))  # f32::round of a non-negative value
    return pinned


def mode_lambda_weight(q, sub):
    scale = {2: f32(0.8), 1: f32(0.65), 0: f32(0.6)}[sub]
    w = f32(f32(min(max(((255 - q) * 3) // 4, 0), 72) + 128) * f32(1.0 / 128.0))
    if sub == 1:
        return f32(w * scale)
    r = f32(np.clip(f32(f32(f32(q) - f32(0.0)) / f32(72.0)), 0, 1))
    return f32(f32(f32(3.0) + f32(f32(w - f32(3.0)) * r)) * scale)


def mode_lambda_q(dc_q):
    dc = f32(dc_q)
    mult = f32(f32(3.3) + f32(f32(0.0015) * dc))
    return f32(f32(f32(f32(f32(0.009005174719460433) * f32(1.0)) * dc) * dc) * mult)


def luma_satd_scale(q, sub):
    if sub:
        return f32(1.25)
    qi = f32(q)
    if qi <= 20:
        return f32(2.921556)
    if qi >= 48:
        return f32(1.25)
    return f32(f32(2.921556) + f32(f32(f32(f32(1.25) - f32(2.921556)) * f32(qi - f32(20.0))) / f32(28.0)))


def k_satd(q, sub):
    k = [f32(24.5), f32(21.3), f32(18.2)] if sub else [f32(35.0), f32(21.2), f32(18.1)]
    qi = f32(q)
    if qi <= 28:
        return k[0]
    if qi >= 140:
        return k[2]
    if qi <= 81:
        return f32(k[0] + f32(f32(f32(k[1] - k[0]) * f32(qi - f32(28.0))) / f32(53.0)))
    return f32(k[1] + f32(f32(f32(k[2] - k[1]) * f32(qi - f32(81.0))) / f32(59.0)))


def test_quality_to_q_anchors_and_monotone(mt_lib):
    assert (mt_lib.quality_to_q(40), mt_lib.quality_to_q(60), mt_lib.quality_to_q(80)) == (116, 70, 35)
    assert mt_lib.quality_to_q(100) == 1 and mt_lib.quality_to_q(0) == 215 and mt_lib.quality_to_q(1) == 215
    qs = [mt_lib.quality_to_q(v) for v in range(1, 101)]
    assert all(a >= b for a, b in zip(qs, qs[1:]))
    # linear between anchors: quality 35 sits halfway between (30, 140) and (40, 116)
    assert mt_lib.quality_to_q(35) == 140 + (116 - 140) * 5 // 10


def test_qm_levels_match_restatement(mt_lib):
    for sub in (0, 1, 2):
        for q in range(256):
            assert mt_lib.qm_levels(q, sub) == (qm_level_law(q, sub), qm_chroma_level_law(q, sub)), (q, sub)
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
def test_lambdas_match_restatement(mt_lib, sub):
    for q in range(256):
        dcq = int(mt_lib.quant_new(q, 8, 15).dc_q)
        got = mt_lib.rd_lambdas(q, dcq, sub)
        mlam = f32(mode_lambda_q(dcq) * mode_lambda_weight(q, sub))
        assert np.float32(got.mode_lambda).tobytes() == mlam.tobytes(), q
        assert np.float32(got.lambda_d).tobytes() == f32(mlam / f32(2.775)).tobytes()
        assert got.trellis_lambda0 == np.float32(0.05)
        assert np.float32(got.satd_scale).tobytes() == luma_satd_scale(q, sub).tobytes(), q
        bridge = f32(f32(f32(2.775) / k_satd(q, sub)) * f32(7.130643))
        assert np.float32(got.satd_bridge).tobytes() == bridge.tobytes(), q


def test_lambdas_reject(mt_lib):
    from maroontree_b200 import MtError, abi

    with pytest.raises(MtError) as e:
        mt_lib.rd_lambdas(70, 100, 2, bd=10)
    assert e.value.code == abi.MT_ERR_UNSUPPORTED
    with pytest.raises(MtError):
        mt_lib.rd_lambdas(70, 0, 2)
