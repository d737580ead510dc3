"""Adaptive-quantisation grid (precompute_aq_grid / aq_sb_target): the oracle
pinned to the reference's own AQ tests (src/coder/aq_tests.rs:559-730), the
dark-weight power table pinned to this C library, and the CUDA grid bit-exact
against the oracle (every cell and both tile means)."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from maroontree_b200 import abi, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _params(w8, h8, q, bd=8, vb=True, dark=True, tiling=(0, 0), octile=6, boost_only=False, strength=1.0):
    p = abi.AqParams()
    p.w8, p.h8 = w8, h8
    p.tile_cols_log2, p.tile_rows_log2 = tiling
    p.base_q_idx, p.bd, p.variance_boost, p.dark_aq = q, bd, int(vb), int(dark)
    p.octile, p.boost_only, p.strength = octile, int(boost_only), strength
    return p


def _serial_frame(w=200, h=136):
    """The mixed dark-gradient / texture / flat frame of aq_grid_matches_serial
    (src/coder/aq_tests.rs:564-580)."""
    r = np.arange(h)[:, None]
    c = np.arange(w)[None, :]
    base = ((r * 255) // h) // 3
    tex = np.where(((r // 32 + c // 32) % 3) == 0, ((r * 7 + c * 13) % 53) - 26, 0)
    return np.clip(base + tex, 0, 255).astype(np.uint16)


def _stripes(mean, shift=0):
    c = np.arange(64)[None, :].repeat(64, 0)
    return ((mean + np.where((c // 4) % 2 == 0, 12, -12)) << shift).astype(np.uint16)


def _tiles(prm):
    sbr, sbc = (prm.h8 + 63) // 64, (prm.w8 + 63) // 64
    cs = -(-sbc // (1 << prm.tile_cols_log2))
    rs = -(-sbr // (1 << prm.tile_rows_log2))
    for y0 in range(0, sbr, rs):
        for x0 in range(0, sbc, cs):
            yield y0, min(y0 + rs, sbr), x0, min(x0 + cs, sbc)


def _walk_ok(cells, prm):
    """aq_begin_sb's serial accumulator over each tile's raster order
    (src/coder/lossy_state.rs:3904-3935) reproduces every cell."""
    for y0, y1, x0, x1 in _tiles(prm):
        cur = prm.base_q_idx
        for sy in range(y0, y1):
            for sx in range(x0, x1):
                c = cells[sy, sx]
                d = int(c["target"]) - cur  # fast_round(d / 4): half away from zero
                st = max(-12, min(12, (1 if d > 0 else -1) * ((abs(d) + 2) // 4)))
                nq = min(max(cur + st * 4, 1), 255)
                if (c["prev"], c["newq"], c["steps"]) != (cur, nq, st):
                    return False
                cur = nq
    return True


# ---- oracle pins (CPU) -------------------------------------------------------


def test_dark_protection_targets_dark_structure_only(oracle_lib):
    """src/coder/aq_tests.rs:665-706."""
    d_dark = oracle_lib.dark_protection(_stripes(36), 190)
    assert d_dark > 0
    assert oracle_lib.dark_protection(_stripes(180), 190) == 0
    assert oracle_lib.dark_protection(np.full((64, 64), 24, np.uint16), 190) == 0
    assert oracle_lib.dark_protection(_stripes(36), 60) == 0
    assert oracle_lib.dark_protection(_stripes(36), 190, enabled=False) == 0


def test_dark_protection_bitdepth_normalized(oracle_lib):
    """src/coder/aq_tests.rs:708-730 (and the same at 12 bits)."""
    d8 = oracle_lib.dark_protection(_stripes(36), 190)
    assert d8 > 0
    assert oracle_lib.dark_protection(_stripes(36, 2), 190, bd=10) == d8
    assert oracle_lib.dark_protection(_stripes(36, 4), 190, bd=12) == d8


def test_fast_round_and_log1p(oracle_lib):
    lib = oracle_lib.load()
    assert [lib.or_fast_round(v) for v in (2.5, -2.5, 1.4, -1.6, 0.0, 7.0)] == [3.0, -3.0, 1.0, -2.0, 0.0, 7.0]
    for d in (0.0, 1e-6, 0.37, 1.0, 255.0, 1e4, 6.5e7):
        got = lib.or_dirty_log1pf(d)
        assert abs(got - np.log1p(d)) <= 2e-6 * max(1.0, np.log1p(d)), d


def test_tiling_spec_min(oracle_lib):
    """plan_tiling with one target tile: one tile up to 4096 wide and 2304
    superblocks, then the minimum column / row split."""
    assert oracle_lib.tiling_spec_min(1920, 1080) == (0, 0)
    assert oracle_lib.tiling_spec_min(512, 512) == (0, 0)
    assert oracle_lib.tiling_spec_min(4096, 4096) == (0, 1)
    assert oracle_lib.tiling_spec_min(8192, 1080) == (1, 0)
    assert oracle_lib.tiling_spec_min(16384, 16384) == (2, 3)


def test_library_tiling_matches_oracle(mt_lib, oracle_lib):
    for w, h in [(1920, 1080), (4096, 4096), (8192, 1080), (16384, 16384), (64, 64), (4104, 2312)]:
        assert mt_lib.tiling_spec_min(w, h) == oracle_lib.tiling_spec_min(w, h)


@pytest.mark.parametrize("vb", [False, True])
@pytest.mark.parametrize("q", [60, 140, 220])
def test_oracle_grid_matches_serial(oracle_lib, vb, q):
    """src/coder/aq_tests.rs:559-618: the grid equals the serial accumulator walk."""
    y = _serial_frame()
    prm = _params(200, 136, q, vb=vb)
    cells, refs = oracle_lib.aq_grid(y, prm)
    assert _walk_ok(cells, prm)
    assert np.all((cells["newq"] >= 1) & (np.abs(cells["steps"]) <= 12))
    # The frame carries dark, flat and textured SBs: the targets are not all equal.
    assert len(set(cells["target"].ravel().tolist())) > 2


def test_dark_pow_table_pinned_to_this_c_library():
    """The committed exception table is what gen_dark_pow_table.py derives from
    the C library the oracle links (glibc powf)."""
    sys.path.insert(0, os.path.join(ROOT, "maroontree_b200", "csrc"))
    try:
        import gen_dark_pow_table as gen
    finally:
        sys.path.pop(0)
    committed = open(gen.OUT).read()
    saved = gen.OUT
    tmp = os.path.join(os.path.dirname(saved), "_dark_pow_check.h")
    try:
        gen.OUT = tmp
        gen.generate()
        fresh = open(tmp).read()
    finally:
        gen.OUT = saved
        if os.path.exists(tmp):
            os.remove(tmp)
    assert fresh == committed


def test_dark_pow_table_entries_match_oracle(oracle_lib):
    text = open(os.path.join(ROOT, "maroontree_b200", "csrc", "dark_pow_table.h")).read()
    def arr(name):
        body = text.split(name)[1].split("{")[1].split("}")[0]
        return np.array([int(v, 0) for v in re.findall(r"0x[0-9a-f]+|\d+", body)], np.int64)

    xs, rs, bk = arr("kDarkPowX"), arr("kDarkPowR"), arr("kDarkPowB")
    assert len(xs) == len(rs) > 1000 and np.all(np.diff(xs) > 0)
    got = oracle_lib.dark_pow(xs.astype(np.uint32).view(np.float32)).view(np.uint32)
    assert np.array_equal(got, rs.astype(np.uint32))
    # the bucket index: entry i sits in bucket (x - 0x3f800000) >> 12
    b = (xs - 0x3F800000) >> 12
    assert np.array_equal(bk[b] <= np.arange(len(xs)), np.ones(len(xs), bool))
    assert np.all(np.arange(len(xs)) < bk[b + 1]) and bk[-1] == len(xs) and bk[0] == 0


# ---- CUDA parity (GPU) ---------------------------------------------------------


def _cases():
    rgb = synth.generate_rgb(1920, 1080, 3, variant="1080p")
    y1080 = synth.rgb_to_luma(rgb)
    rng = np.random.default_rng(11)
    y10 = np.clip(synth.rgb_to_luma(synth.generate_rgb(328, 200, 7)).astype(np.int32) * 4 +
                  rng.integers(-6, 7, (200, 328)), 0, 1023).astype(np.uint16)
    # 12 bits: dark, very busy superblocks whose Laplacian sums pass 2^24 sample
    # units (the reference's f32 sums round there), among white noise.
    y12 = rng.integers(0, 4096, (136, 264)).astype(np.int64)
    r, c = np.mgrid[0:64, 0:64]
    c1, c2 = (r + c) % 2, (r // 2 + c // 2) % 2
    for k, a in enumerate((600, 1600, 1000, 1180)):
        y12[:64, 64 * k:64 * k + 64] = a * c1 + (1780 - a) * c2 + rng.integers(-3, 4, (64, 64))
    y12[64:128, :64] //= 24
    y12 = np.clip(y12, 0, 4095).astype(np.uint16)
    serial = _serial_frame()
    return {
        "serial": serial, "c2": y1080, "y10": y10, "y12": y12,
    }


_CASES = None


def _case(name):
    global _CASES
    if _CASES is None:
        _CASES = _cases()
    return _CASES[name]


GPU_CASES = [
    ("serial", 60, 8, True, True, (0, 0)),
    ("serial", 140, 8, True, True, (0, 0)),
    ("serial", 220, 8, True, True, (0, 0)),
    ("serial", 60, 8, False, True, (0, 0)),
    ("serial", 140, 8, False, True, (0, 0)),
    ("serial", 220, 8, False, True, (0, 0)),
    ("c2", 116, 8, True, True, (0, 0)),   # 1080p q40: dark protection active
    ("c2", 70, 8, True, True, (0, 0)),    # 1080p q60
    ("c2", 35, 8, True, True, (0, 0)),    # 1080p q80: the cut-side top ease
    ("c2", 116, 8, False, True, (1, 1)),  # classic AQ, four tiles
    ("c2", 200, 8, True, True, (2, 0)),   # three column tiles (ragged last)
    ("y10", 150, 10, True, True, (0, 0)),
    ("y12", 150, 12, True, True, (0, 0)),
    ("y12", 150, 12, False, True, (0, 1)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,q,bd,vb,dark,tiling", GPU_CASES)
def test_aq_grid_matches_oracle(mt_lib, oracle_lib, cuda, name, q, bd, vb, dark, tiling):
    y = _case(name)
    h8, w8 = y.shape
    prm = _params(w8, h8, q, bd=bd, vb=vb, dark=dark, tiling=tiling)
    ref_cells, ref_refs = oracle_lib.aq_grid(y, prm)
    cells, refs = mt_lib.aq_grid(y, prm)
    assert refs.view(np.uint32).tolist() == ref_refs.view(np.uint32).tolist()
    assert cells.tobytes() == ref_cells.tobytes()
    assert _walk_ok(cells, prm)


@pytest.mark.gpu
def test_aq_grid_variants_match_oracle(mt_lib, oracle_lib, cuda):
    """Octile, boost-only and strength knobs."""
    y = _case("serial")
    for kw in ({"octile": 1}, {"octile": 8}, {"boost_only": True}, {"strength": 2.5}, {"strength": -1.0},
               {"dark": False}):
        prm = _params(200, 136, 140, **kw)
        a, ra = oracle_lib.aq_grid(y, prm)
        b, rb = mt_lib.aq_grid(y, prm)
        assert a.tobytes() == b.tobytes(), kw
        assert ra.tobytes() == rb.tobytes(), kw


@pytest.mark.gpu
def test_aq_grid_device_api_matches_host(mt_lib, cuda):
    torch = cuda
    y = _case("c2")
    prm = _params(1920, 1080, 116)
    host_cells, host_refs = mt_lib.aq_grid(y, prm)
    dev = torch.device("cuda:0")
    d_y = torch.from_numpy(y.view(np.int16).copy()).to(dev)
    d_cells = torch.zeros(host_cells.size * 4, dtype=torch.uint8, device=dev)
    d_refs = torch.zeros(host_refs.size, dtype=torch.float32, device=dev)
    d_scr = torch.zeros(mt_lib.aq_grid_scratch_bytes(prm), dtype=torch.uint8, device=dev)
    for _ in range(2):  # the scratch is reused as is between calls
        mt_lib.aq_grid_device(d_y, prm, d_cells, d_refs, d_scr)
        torch.cuda.synchronize()
        assert d_cells.cpu().numpy().tobytes() == host_cells.tobytes()
        assert d_refs.cpu().numpy().tobytes() == host_refs.tobytes()


@pytest.mark.gpu
def test_aq_grid_rejects_bad_input(mt_lib, cuda):
    import ctypes as C

    lib = mt_lib.load()
    y = np.zeros((64, 8192), np.uint16)
    cells = np.zeros(4096, abi.AQ_CELL_DTYPE)
    refs = np.zeros(256, np.float32)
    for bad in (_params(200, 64, 60, bd=9), _params(204, 64, 60), _params(200, 64, 300),
                _params(200, 64, 60, tiling=(7, 0)),
                _params(8192, 64, 60)):  # one tile 128 superblocks wide
        assert lib.mt_aq_grid(y.ctypes.data, C.byref(bad), cells.ctypes.data, refs.ctypes.data) != 0
    assert lib.mt_aq_grid(y.ctypes.data, C.byref(_params(8192, 64, 60, tiling=(1, 0))), cells.ctypes.data,
                          refs.ctypes.data) == 0


@pytest.mark.gpu
def test_dark_pow_exhaustive(mt_lib, oracle_lib, cuda):
    """Every binary32 x in (1, 4.5]: the device power equals the C library's powf."""
    torch = cuda
    lo = np.array([1.0], np.float32).view(np.uint32)[0] + 1
    hi = np.array([4.5], np.float32).view(np.uint32)[0]
    xs = np.arange(lo, hi + 1, dtype=np.uint32).view(np.float32)
    ref = oracle_lib.dark_pow(xs)
    dev = torch.device("cuda:0")
    d_x = torch.from_numpy(xs).to(dev)
    d_o = torch.empty_like(d_x)
    mt_lib.dark_pow_device(d_x, d_o, xs.size)
    torch.cuda.synchronize()
    got = d_o.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
