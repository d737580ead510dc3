"""Frame CDEF (src/coder/frame_cdef.rs, src/cdef.rs): oracle pins on the CPU
(the weighted SSE against the reference's own test values and a float64
restatement, decisions on frames CDEF cannot help), and bit-exact GPU parity of
the per-block directions, the per-unit distortion tables of all 12 strength
pairs, the strength decision and the filtered planes, for 4:2:0, 4:2:2, 4:4:4
and monochrome frames with odd visible sizes."""
import numpy as np
import pytest

from maroontree_b200 import synth

WSSE_MEAN = np.float32(0.4625)


def _wsse_f64(err):
    """Scalar float64 restatement of the 4x4-DCT weighted SSE."""
    a, b, c = 0.5, 0.653_281_5, 0.270_598_05
    d = np.array([[a, a, a, a], [b, c, -c, -b], [a, -a, -a, a], [c, -b, b, -c]])
    hf, ax, ac1, dg, dc = 0.2, 0.4, 1.0, 0.8, 1.8
    wt = np.array([[dc, ac1, ax, hf], [ac1, dg, hf, hf], [ax, hf, hf, hf], [hf, hf, hf, hf]]) / 0.4625
    h, w = err.shape
    tot = 0.0
    for r in range(0, h, 4):
        for q in range(0, w, 4):
            co = d @ err[r:r + 4, q:q + 4].astype(np.float64) @ d.T
            tot += float((wt * co * co).sum())
    return tot


def test_oracle_wsse_flat_tile_is_weighted_dc(oracle_lib):
    """A flat 4x4 error of 3 is all DC: 4*3 squared times 1.8 / 0.4625."""
    want = 1.8 / 0.4625 * 144.0
    got = oracle_lib.weighted_sse(np.full((4, 4), 3, np.int32))
    assert abs(got - want) < 1e-3 * want


@pytest.mark.parametrize("w,h", [(4, 4), (8, 4), (4, 16), (16, 16), (32, 8), (64, 64), (8, 8), (4, 8)])
def test_oracle_wsse_matches_float64(oracle_lib, w, h):
    i = np.arange(w * h)
    err = (((i * 7919) % 513) - 256).astype(np.int32).reshape(h, w)
    got = oracle_lib.weighted_sse(err)
    want = _wsse_f64(err)
    assert abs(got - want) <= 1e-5 * want
    plain = float((err.astype(np.float64) ** 2).sum())
    assert 0.2 * plain < got < 1.8 * plain


def _prm(mt, w, h, sub, mono, q, slow=True):
    return mt.cdef_params(w, h, sub[0], sub[1], q, mono=mono, slow=slow)


def test_oracle_cdef_leaves_exact_recon_alone(oracle_lib, mt_lib):
    src, _, skip = synth.cdef_inputs(130, 70, 1, 1, False, 4)
    prm = _prm(mt_lib, 130, 70, (1, 1), False, 90)
    out, dec, _ = oracle_lib.cdef_frame(src, src, skip, prm)
    assert dec["bits"] == -1
    assert all(np.array_equal(a, b) for a, b in zip(out, src))


def test_oracle_cdef_all_skip_frame_is_off(oracle_lib, mt_lib):
    src, rec, skip = synth.cdef_inputs(64, 64, 1, 1, False, 5)
    prm = _prm(mt_lib, 64, 64, (1, 1), False, 120)
    out, dec, tabs = oracle_lib.cdef_frame(rec, src, np.ones_like(skip), prm)
    assert dec["bits"] == -1 and not tabs["luma"].any()
    assert all(np.array_equal(a, b) for a, b in zip(out, rec))


def test_oracle_cdef_filters_noisy_frame(oracle_lib, mt_lib):
    """Noisy units get filtered and the luma error drops."""
    src, rec, skip = synth.cdef_inputs(256, 192, 1, 1, False, 6, skip_frac=0.0)
    prm = _prm(mt_lib, 256, 192, (1, 1), False, 120)
    out, dec, _ = oracle_lib.cdef_frame(rec, src, skip, prm)
    assert dec["bits"] >= 0
    e0 = ((rec[0].astype(np.int64) - src[0]) ** 2).sum()
    e1 = ((out[0].astype(np.int64) - src[0]) ** 2).sum()
    assert e1 < e0


def test_cdef_rejects_bad_params(mt_lib):
    from maroontree_b200 import MtError, abi

    src, rec, skip = synth.cdef_inputs(64, 64, 1, 1, False, 1)
    bad = _prm(mt_lib, 64, 64, (1, 1), False, 60)
    bad.disp_w = 50
    with pytest.raises(MtError):
        mt_lib.cdef_frame(rec, src, skip, bad)
    bad = _prm(mt_lib, 64, 64, (0, 1), False, 60)
    with pytest.raises(MtError):
        mt_lib.cdef_frame(rec, src, skip, bad)
    bad = _prm(mt_lib, 64, 64, (1, 1), False, 60)
    bad.bd = 10
    with pytest.raises(MtError) as ei:
        mt_lib.cdef_frame(rec, src, skip, bad)
    assert ei.value.code == abi.MT_ERR_UNSUPPORTED


CASES = [
    # disp_w, disp_h, (sub_x, sub_y), mono, base_q_idx, slow, seed  (oracle's cdef_bits)
    (64, 64, (1, 1), False, 70, True, 20),  # -1: off
    (64, 64, (1, 1), False, 70, True, 25),  # 0
    (203, 117, (1, 1), False, 116, True, 22),  # 1
    (130, 90, (1, 0), False, 200, True, 20),  # 0, 4:2:2
    (97, 131, (0, 0), False, 35, True, 20),  # 1, 4:4:4
    (150, 70, (1, 1), True, 150, True, 21),  # 0, monochrome
    (500, 500, (1, 1), True, 220, True, 20),  # 1, monochrome
    (256, 200, (1, 1), False, 255, False, 21),  # 0, the fast candidate list
    (640, 480, (1, 1), False, 20, True, 20),  # 3
    (640, 480, (0, 0), False, 10, True, 24),  # 2
    (1920, 1080, (1, 1), False, 70, True, 3),
    (1280, 720, (0, 0), False, 50, True, 26),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}-{c[2]}-{'mono' if c[3] else 'col'}-q{c[4]}")
def test_cdef_tables_match_oracle(mt_lib, oracle_lib, cuda, case):
    import torch

    w, h, sub, mono, q, slow, seed = case
    src, rec, skip = synth.cdef_inputs(w, h, sub[0], sub[1], mono, seed)
    prm = _prm(mt_lib, w, h, sub, mono, q, slow)
    _, _, want = oracle_lib.cdef_frame(rec, src, skip, prm)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).astype(np.int16) if a.dtype == np.uint16 else a).cuda()
    d_rec, d_src = [dev(p) for p in rec], [dev(p) for p in src]
    nb, nu = skip.size, want["luma"].shape[0]
    dirs = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    vars_ = torch.zeros(nb, dtype=torch.int32, device="cuda")
    tabs = [torch.zeros((nu, 12), dtype=torch.int64, device="cuda") for _ in range(3)]
    ch = (lambda a, i: None) if mono else (lambda a, i: a[i].data_ptr())
    rc = mt_lib.load().mt_cdef_tables_device(d_rec[0].data_ptr(), ch(d_rec, 1), ch(d_rec, 2), d_src[0].data_ptr(),
                                             ch(d_src, 1), ch(d_src, 2), dev(skip).data_ptr(), prm, dirs.data_ptr(),
                                             vars_.data_ptr(), tabs[0].data_ptr(), tabs[1].data_ptr(),
                                             tabs[2].data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert np.array_equal(dirs.cpu().numpy(), want["dirs"])
    assert np.array_equal(vars_.cpu().numpy(), want["vars"])
    for k, name in enumerate(["luma", "u", "v"]):
        if mono and k:
            continue
        assert np.array_equal(tabs[k].cpu().numpy(), want[name]), name


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}-{c[2]}-{'mono' if c[3] else 'col'}-q{c[4]}")
def test_cdef_frame_matches_oracle(mt_lib, oracle_lib, cuda, case):
    w, h, sub, mono, q, slow, seed = case
    src, rec, skip = synth.cdef_inputs(w, h, sub[0], sub[1], mono, seed)
    prm = _prm(mt_lib, w, h, sub, mono, q, slow)
    want_planes, want_dec, _ = oracle_lib.cdef_frame(rec, src, skip, prm)
    got_planes, got_dec = mt_lib.cdef_frame(rec, src, skip, prm)
    assert got_dec["bits"] == want_dec["bits"]
    assert got_dec["strengths"] == want_dec["strengths"]
    assert np.array_equal(got_dec["grid"], want_dec["grid"])
    for a, b in zip(got_planes, want_planes):
        assert np.array_equal(a, b)
