"""Deblocking filter (src/loopfilter.rs filter_plane, as src/coder/frame_deblock.rs
drives it per plane): oracle known answers and order properties on the CPU,
bit-exact GPU parity with the oracle on AV1-shaped block geometry, on the
reference's own mixed-geometry pattern (edges whose taps overlap), at 1080p,
and through the device entry point on a stream."""
import ctypes as C

import numpy as np
import pytest

from maroontree_b200 import synth


def _geometry(vis_w, vis_h, seed):
    w, h = (vis_w + 7) & ~7, (vis_h + 7) & ~7
    bw, bh, ve, he, bid = synth.partition_maps(w // 4, h // 4, seed)
    return w, h, bw, bh, ve, he, synth.blocky_plane(w, h, bid, seed)


def _mixed_geometry():
    """The edge-map pattern of the reference's batch-coalescing test
    (src/loopfilter.rs tests): block sizes and edge flags that ignore each
    other, so neighbouring edges' taps overlap."""
    W, H = 264, 88
    nc4, nr4 = W // 4, H // 4
    r4, c4 = np.mgrid[0:nr4, 0:nc4]
    sizes = np.array([1, 2, 4, 8], np.uint8)
    bw = sizes[(r4 + 2 * c4) & 3]
    bh = sizes[(2 * r4 + c4) & 3]
    ve = ((c4 >= 2) & (c4 + 2 < nc4) & ((3 * r4 + c4) % 5 <= 2)).astype(np.uint8)
    he = ((r4 >= 2) & (r4 + 2 < nr4) & ((r4 + 3 * c4) % 5 <= 2)).astype(np.uint8)
    i = np.arange(W * H)
    img = ((((i % W) // 8 + (i // W) // 8) & 31) * 4 + 64).astype(np.uint16).reshape(H, W)
    return W, H, bw, bh, ve, he, img


def test_oracle_explicit_edge_at_unaligned_origin(oracle_lib):
    """An explicitly flagged vertical edge at x = 12 inside 8-wide blocks is
    filtered; under the alignment rule (12/4 = 3 is not a multiple of 2) it is not."""
    w, h = 32, 4
    px = np.full((h, w), 110, np.uint16)
    px[:, :12] = 100
    bw = np.full((1, w // 4), 2, np.uint8)
    bh = np.ones((1, w // 4), np.uint8)
    ve = np.zeros((1, w // 4), np.uint8)
    ve[0, 3] = 1
    out = oracle_lib.deblock_plane(px, w, h, bw, bh, 32, 7, True, ve, None)
    assert not np.array_equal(out, px)
    assert np.array_equal(out[:, :8], px[:, :8]) and np.array_equal(out[:, 16:], px[:, 16:])
    assert np.array_equal(oracle_lib.deblock_plane(px, w, h, bw, bh, 32, 7, True), px)


def test_oracle_wide_filter_known_answer(oracle_lib):
    """A 1-step edge between two 16-wide flat blocks at level 32 takes the
    16-wide smoothing filter: (sum of the 15-tap window + 8) >> 4 per sample."""
    w, h = 32, 4
    px = np.full((h, w), 101, np.uint16)
    px[:, :16] = 100
    bw = np.full((1, 8), 4, np.uint8)
    out = oracle_lib.deblock_plane(px, w, h, bw, bw, 32, 0, True)
    row = out[0, 10:22].tolist()
    # p5..q5 of p = 100 x7, q = 101 x7 under the 16-wide taps (AV1 spec 7.14.6.4).
    window = [100] * 7 + [101] * 7
    taps = [
        [7, 2, 2, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0], [5, 2, 2, 2, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0],
        [4, 1, 2, 2, 2, 1, 1, 1, 1, 1, 0, 0, 0, 0], [3, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 0, 0, 0],
        [2, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 0, 0], [1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1, 0],
        [0, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 1, 1], [0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 1, 2],
        [0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 1, 1, 3], [0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 1, 4],
        [0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 5], [0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 7],
    ]
    expect = [(sum(t * v for t, v in zip(tp, window)) + 8) >> 4 for tp in taps]
    assert row == expect
    assert np.all(out == out[0:1])


def test_oracle_level_zero_is_identity(oracle_lib):
    w, h, bw, bh, ve, he, px = _geometry(77, 45, 3)
    assert np.array_equal(oracle_lib.deblock_plane(px, 77, 45, bw, bh, 0, 0, True, ve, he), px)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_two_pass_order_equals_superblock_order(oracle_lib, seed):
    """On AV1-shaped geometry, filtering all vertical edges then all horizontal
    edges (one superblock row spanning the frame) gives the reference's
    per-superblock-row samples: the order the GPU passes use."""
    rng = np.random.default_rng(seed)
    vis_w, vis_h = int(rng.integers(8, 260)), int(rng.integers(8, 300))
    w, h, bw, bh, ve, he, px = _geometry(vis_w, vis_h, seed)
    luma = seed % 3 != 0
    level, sharp = int(rng.choice([8, 24, 40, 63])), int(rng.integers(0, 8))
    flags = (ve, he) if seed % 2 else (None, None)
    sb = oracle_lib.deblock_plane(px, vis_w, vis_h, bw, bh, level, sharp, luma, *flags, sb_rows4=16 if luma else 8)
    whole = oracle_lib.deblock_plane(px, vis_w, vis_h, bw, bh, level, sharp, luma, *flags, sb_rows4=1 << 20)
    assert np.array_equal(sb, whole)
    assert not np.array_equal(sb, px)


def test_deblock_rejects_bad_input(mt_lib):
    from maroontree_b200 import MtError, abi

    w, h, bw, bh, ve, he, px = _geometry(64, 64, 1)
    with pytest.raises(MtError):
        mt_lib.deblock_plane(px, 64, 64, bw, bh, 64, 0, True)
    with pytest.raises(MtError):
        mt_lib.deblock_plane(px, 64, 64, bw, bh, 10, 8, True)
    with pytest.raises(MtError):
        mt_lib.deblock_plane(px, 65, 64, bw, bh, 10, 0, True)
    lib = mt_lib.load()
    odd = np.zeros((6, 6), np.uint16)
    m = np.ones((2, 2), np.uint8)
    assert lib.mt_deblock_plane(odd.ctypes.data, 6, 6, 6, 6, m.ctypes.data, m.ctypes.data, None, None, 2, 10, 0, 1,
                                8) == abi.MT_ERR_INVALID_INPUT
    assert lib.mt_deblock_plane(odd.ctypes.data, 8, 8, 8, 8, m.ctypes.data, m.ctypes.data, None, None, 2, 10, 0, 1,
                                10) == abi.MT_ERR_UNSUPPORTED


def test_deblock_rejects_superblock_crossing_edge(mt_lib):
    """A 16-wide horizontal edge on the last 4-row of a 64-row superblock row
    (outside AV1 block geometry) is refused by the host entry point, which
    checks the maps before touching the device."""
    from maroontree_b200 import MtError, abi

    w, h = 64, 128
    nc4, nr4 = w // 4, h // 4
    bw = np.full((nr4, nc4), 4, np.uint8)
    bh = np.full((nr4, nc4), 4, np.uint8)
    he = np.zeros((nr4, nc4), np.uint8)
    he[15, 4] = 1
    px = np.full((h, w), 100, np.uint16)
    with pytest.raises(MtError) as ei:
        mt_lib.deblock_plane(px, w, h, bw, bh, 30, 0, True, None, he)
    assert ei.value.code == abi.MT_ERR_UNSUPPORTED


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(16))
def test_deblock_matches_oracle(mt_lib, oracle_lib, cuda, seed):
    rng = np.random.default_rng(1000 + seed)
    vis_w, vis_h = int(rng.integers(1, 400)), int(rng.integers(1, 300))
    w, h, bw, bh, ve, he, px = _geometry(vis_w, vis_h, 1000 + seed)
    luma = seed % 4 != 0
    level, sharp = int(rng.choice([1, 6, 16, 31, 47, 63])), int(rng.integers(0, 8))
    flags = (ve, he) if seed % 2 else (None, None)
    want = oracle_lib.deblock_plane(px, vis_w, vis_h, bw, bh, level, sharp, luma, *flags, sb_rows4=16 if luma else 8)
    got = mt_lib.deblock_plane(px, vis_w, vis_h, bw, bh, level, sharp, luma, *flags)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("level,sharp", [(32, 7), (63, 0), (12, 3)])
def test_deblock_overlapping_taps_match_oracle(mt_lib, oracle_lib, cuda, level, sharp):
    W, H, bw, bh, ve, he, img = _mixed_geometry()
    want = oracle_lib.deblock_plane(img, W, H, bw, bh, level, sharp, True, ve, he)
    got = mt_lib.deblock_plane(img, W, H, bw, bh, level, sharp, True, ve, he)
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("luma", [True, False])
def test_deblock_1080p_device_entry(mt_lib, oracle_lib, cuda, luma):
    """Full-size planes through mt_deblock_plane_device on a side stream."""
    import torch

    from maroontree_b200 import abi

    vis_w, vis_h = (1920, 1080) if luma else (960, 540)
    w, h, bw, bh, ve, he, px = _geometry(vis_w, vis_h, 77 + luma)
    level = 36 if luma else 20
    want = oracle_lib.deblock_plane(px, vis_w, vis_h, bw, bh, level, 2, luma, ve, he, sb_rows4=16 if luma else 8)
    d_px = torch.from_numpy(px.astype(np.int16)).cuda()
    maps = [torch.from_numpy(np.ascontiguousarray(m)).cuda() for m in (bw, bh, ve, he)]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        rc = mt_lib.load().mt_deblock_plane_device(d_px.data_ptr(), w, h, vis_w, vis_h, *[m.data_ptr() for m in maps],
                                                    bw.shape[1], level, 2, int(luma), 8, C.c_void_p(s.cuda_stream))
    s.synchronize()
    assert rc == abi.MT_OK
    got = d_px.cpu().numpy().view(np.uint16)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("q,sub,want", [(70, 2, (8, 4, 7)), (255, 0, (31, 25, 7)), (5, 2, (0, 0, 7)), (9, 2, (1, 1, 7)),
                                        (120, 1, (15, 12, 7)), (0, 0, (0, 0, 7))])
def test_loop_filter_levels_known_answers(mt_lib, oracle_lib, q, sub, want):
    """src/obu.rs:306-334: luma round(q/8) (max 40); chroma round((q/10) x 0.5
    in 4:2:0, x 1 otherwise), at least 1 while luma filters (max 32)."""
    sx, sy = (1, 1) if sub == 2 else ((1, 0) if sub == 1 else (0, 0))
    assert mt_lib.loop_filter_levels(q, sx, sy) == want
    assert oracle_lib.loop_filter_levels(q, sub) == want


def test_loop_filter_levels_all_q_match_oracle(mt_lib, oracle_lib):
    for q in range(256):
        for sx, sy in ((0, 0), (1, 0), (1, 1)):
            assert mt_lib.loop_filter_levels(q, sx, sy) == oracle_lib.loop_filter_levels(q, sx + sy)


def _frame_inputs(disp_w, disp_h, sx, sy, mono, seed):
    w8, h8 = (disp_w + 7) & ~7, (disp_h + 7) & ~7
    pw, ph, pv, pt, bid = synth.partition_maps(w8 // 4, h8 // 4, seed)
    tx = synth.transform_maps(pw, ph, bid, seed + 1)
    planes = [synth.blocky_plane(w8, h8, bid, seed)]
    if not mono:
        cb = bid[::1 << sy, ::1 << sx]
        planes += [synth.blocky_plane(w8 >> sx, h8 >> sy, cb, seed + 2), synth.blocky_plane(w8 >> sx, h8 >> sy, cb, seed + 3)]
    return planes, tx, (pw, ph)


@pytest.mark.gpu
@pytest.mark.parametrize("disp_w,disp_h,sx,sy,mono,q", [
    (64, 64, 1, 1, False, 70), (203, 117, 1, 1, False, 180), (130, 90, 1, 0, False, 120), (97, 131, 0, 0, False, 255),
    (150, 70, 1, 1, True, 100), (1920, 1080, 1, 1, False, 70)])
def test_deblock_frame_matches_oracle(mt_lib, oracle_lib, cuda, disp_w, disp_h, sx, sy, mono, q):
    planes, tx, pred = _frame_inputs(disp_w, disp_h, sx, sy, mono, disp_w + q)
    ly, luv, _ = mt_lib.loop_filter_levels(q, sx, sy)
    want = oracle_lib.deblock_frame(planes, disp_w, disp_h, sx, sy, tx, pred, ly, luv, luv, mono)
    got = mt_lib.deblock_frame(planes, disp_w, disp_h, sx, sy, tx, pred, ly, luv, luv, mono)
    for a, b, c in zip(got, want, planes):
        assert np.array_equal(a, b)
        assert not np.array_equal(b, c)


@pytest.mark.gpu
@pytest.mark.parametrize("mono", [True, False])
def test_deblock_frame_overlapping_taps_match_oracle(mt_lib, oracle_lib, cuda, mono):
    """The frame entry on the reference's mixed-geometry maps (edges whose
    taps overlap): the classify pass sends the frame to the two-pass kernels,
    which keep each run in the reference's order."""
    W, H, bw, bh, ve, he, img = _mixed_geometry()
    tx = (bw, bh, ve, he)
    pred = (np.full_like(bw, 2), np.full_like(bh, 2))
    planes = [img]
    if not mono:
        planes += [img[::2, ::2].copy(), (255 - img[::2, ::2]).astype(np.uint16)]
    for q in (60, 200):
        ly, luv, _ = mt_lib.loop_filter_levels(q, 1, 1)
        want = oracle_lib.deblock_frame(planes, W, H, 1, 1, tx, pred, ly, luv, luv, mono)
        got = mt_lib.deblock_frame(planes, W, H, 1, 1, tx, pred, ly, luv, luv, mono)
        for a, b, c in zip(got, want, planes):
            assert np.array_equal(a, b)
        assert not np.array_equal(want[0], planes[0])


@pytest.mark.gpu
@pytest.mark.parametrize("disp_w,disp_h,sx,sy", [(1031, 517, 0, 0), (4096, 256, 1, 1)])
def test_deblock_frame_tiles_match_oracle(mt_lib, oracle_lib, cuda, disp_w, disp_h, sx, sy):
    """The fused tile kernel across many 64x64 tiles and ragged frame edges,
    against the oracle's frame-wide two-pass deblocking."""
    planes, tx, pred = _frame_inputs(disp_w, disp_h, sx, sy, False, disp_w + disp_h)
    ly, luv, _ = mt_lib.loop_filter_levels(150, sx, sy)
    want = oracle_lib.deblock_frame(planes, disp_w, disp_h, sx, sy, tx, pred, ly, luv, luv, False)
    got = mt_lib.deblock_frame(planes, disp_w, disp_h, sx, sy, tx, pred, ly, luv, luv, False)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def _device_deblock(mt_lib, planes, disp_w, disp_h, sx, sy, tx, pred, lv, to):
    """mt_deblock_frame_device (in place) or mt_deblock_frame_device_to (from
    separate input planes, which must come back unchanged) on the GPU."""
    import torch
    from maroontree_b200 import abi

    lib = mt_lib.load()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).astype(np.int16)).cuda()
    src = [dev(p) for p in planes]
    out = [torch.zeros_like(p) for p in src] if to else [p.clone() for p in src]
    maps = [torch.from_numpy(np.ascontiguousarray(m, np.uint8)).cuda() for m in list(tx) + list(pred)]
    g = abi.DeblockFrameParams()
    g.w8, g.h8 = planes[0].shape[1], planes[0].shape[0]
    g.disp_w, g.disp_h, g.sub_x, g.sub_y, g.mono, g.bd = disp_w, disp_h, sx, sy, 0, 8
    scr = torch.empty(lib.mt_deblock_frame_scratch_bytes(C.byref(g)), dtype=torch.uint8, device="cuda")
    args = [m.data_ptr() for m in maps] + [C.byref(g), *lv, scr.data_ptr(), None]
    if to:
        rc = lib.mt_deblock_frame_device_to(*[p.data_ptr() for p in src], *[p.data_ptr() for p in out], *args)
    else:
        rc = lib.mt_deblock_frame_device(*[p.data_ptr() for p in out], *args)
    torch.cuda.synchronize()
    assert rc == 0
    if to:
        for a, b in zip(src, planes):
            assert np.array_equal(a.cpu().numpy().view(np.uint16), b)
    return [p.cpu().numpy().view(np.uint16) for p in out]


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_deblock_frame_device_to_equals_in_place(mt_lib, oracle_lib, cuda, mixed):
    """The out-of-place entry gives the in-place entry's planes and leaves its
    input planes as they were, on the fused path and on the two-pass path of
    maps with overlapping taps."""
    if mixed:
        W, H, bw, bh, ve, he, img = _mixed_geometry()
        planes, tx, pred = [img, img[::2, ::2].copy(), img[::2, ::2].copy()], (bw, bh, ve, he), (bw, bh)
        dw, dh = W, H
    else:
        dw, dh = 515, 333
        planes, tx, pred = _frame_inputs(dw, dh, 1, 1, False, 5)
    lv = mt_lib.loop_filter_levels(120, 1, 1)[:2]
    lv = (lv[0], lv[1], lv[1])
    a = _device_deblock(mt_lib, planes, dw, dh, 1, 1, tx, pred, lv, to=False)
    b = _device_deblock(mt_lib, planes, dw, dh, 1, 1, tx, pred, lv, to=True)
    want = oracle_lib.deblock_frame(planes, dw, dh, 1, 1, tx, pred, *lv, False)
    for x, y, z in zip(a, b, want):
        assert np.array_equal(x, y) and np.array_equal(x, z)
