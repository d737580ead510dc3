"""Screen-content frame gate (screen_frame_gate): the oracle pinned to the
reference's window-hash test (src/coder/block64.rs:2818-2843) and the gate's
own invariants, and the CUDA gate equal to the oracle on every counter and
verdict (photo, text, UI and mixed frames; both index grids; 8/10-bit)."""
import numpy as np
import pytest

from maroontree_b200 import synth


def _xorshift_plane(w, h, seed=0x12345678, mod=1024):
    """The pseudo-random plane of rolling_hash_matches_direct."""
    out = np.empty(w * h, np.uint16)
    s = seed
    for i in range(w * h):
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        out[i] = s % mod
    return out.reshape(h, w)


def _hash8_py(luma, x, y):
    hp, hq = 0x9E3779B1, 0x85EBCA77
    c = 0
    for j in range(8):
        r = 0
        for i in range(8):
            r = (r * hp + int(luma[y + j, x + i]) + 1) & 0xFFFFFFFF
        c = (c * hq + r) & 0xFFFFFFFF
    h = c
    h ^= h >> 16
    h = (h * 0x7FEB352D) & 0xFFFFFFFF
    h ^= h >> 15
    h = (h * 0x846CA68B) & 0xFFFFFFFF
    return h ^ (h >> 16)


def test_hash8_matches_definition(oracle_lib):
    luma = _xorshift_plane(37, 29)
    for x, y in [(0, 0), (5, 3), (29, 21), (13, 17)]:
        assert oracle_lib.hash8(luma, x, y) == _hash8_py(luma, x, y)


def test_gate_on_photo_stops_at_prescreen(oracle_lib):
    y = synth.rgb_to_luma(synth.generate_rgb(640, 360, 3))
    r = oracle_lib.screen_gate(y, 1, 1, 116)
    assert r["copy_stage"] == 0 and r["ibc_pays"] == 0 and r["few_colour"] == 0
    assert r["blocks16"] == 40 * 22


def test_gate_on_text_finds_copies(oracle_lib):
    y = synth.screen_luma(640, 360, 6, photo_frac=0.0)
    r = oracle_lib.screen_gate(y, 0, 0, 116)
    assert r["copy_stage"] == 1 and r["few_colour"] == 1 and r["copied"] >= 4 and r["ibc_pays"] == 1
    assert 0 < r["dup8"] < r["nonflat8"]


def test_gate_tiny_frames(oracle_lib):
    for w, h in [(8, 8), (8, 64), (64, 8)]:
        r = oracle_lib.screen_gate(np.zeros((h, w), np.uint16), 1, 1, 60)
        assert all(v == 0 for v in r.values())


def _frames():
    photo = synth.rgb_to_luma(synth.generate_rgb(1920, 1080, 3, variant="1080p"))
    mixed = synth.screen_luma(1920, 1080, 5, photo_frac=0.3)
    text = synth.screen_luma(640, 360, 6, photo_frac=0.0)
    half = synth.screen_luma(512, 512, 8, photo_frac=0.5)
    odd = synth.screen_luma(200, 136, 9, photo_frac=0.4)  # 16x16 grid narrower than the frame
    ui10 = synth.screen_luma(320, 240, 10, photo_frac=0.3, bd=10)
    little = synth.screen_luma(1280, 720, 11, photo_frac=0.95)  # a few text rows over a photo
    return {"photo": photo, "mixed": mixed, "text": text, "half": half, "odd": odd, "ui10": ui10, "little": little}


_F = None


def _frame(name):
    global _F
    if _F is None:
        _F = _frames()
    return _F[name]


GPU_CASES = [
    ("photo", 1, 1, 116, 8), ("mixed", 1, 1, 116, 8), ("mixed", 0, 0, 70, 8), ("mixed", 1, 0, 35, 8),
    ("text", 0, 0, 116, 8), ("text", 1, 1, 4, 8), ("half", 0, 0, 200, 8), ("odd", 1, 1, 116, 8),
    ("ui10", 1, 1, 150, 10), ("little", 1, 1, 116, 8), ("little", 1, 1, 250, 8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,sx,sy,q,bd", GPU_CASES)
def test_screen_gate_matches_oracle(mt_lib, oracle_lib, cuda, name, sx, sy, q, bd):
    y = _frame(name)
    ref = oracle_lib.screen_gate(y, sx, sy, q, bd)
    got = mt_lib.screen_gate(y, sx, sy, q, bd)
    assert got == ref


@pytest.mark.gpu
def test_screen_gate_device_api_reuses_scratch(mt_lib, oracle_lib, cuda):
    import ctypes as C

    from maroontree_b200 import abi

    torch = cuda
    lib = mt_lib.load()
    dev = torch.device("cuda:0")
    y1, y2 = _frame("text"), _frame("half")
    prm1 = mt_lib.screen_gate_params(y1.shape[1], y1.shape[0], 0, 0, 116)
    prm2 = mt_lib.screen_gate_params(y2.shape[1], y2.shape[0], 0, 0, 200)
    n = max(lib.mt_screen_gate_scratch_bytes(C.byref(prm1)), lib.mt_screen_gate_scratch_bytes(C.byref(prm2)))
    scr = torch.full((n,), 0xAB, dtype=torch.uint8, device=dev)  # stale contents must not matter
    for y, prm, q in [(y1, prm1, 116), (y2, prm2, 200), (y1, prm1, 116)]:
        d_y = torch.from_numpy(y.view(np.int16).copy()).to(dev)
        r = abi.ScreenGateResult()
        assert lib.mt_screen_gate_device(d_y.data_ptr(), C.byref(prm), scr.data_ptr(), C.byref(r), None) == 0
        assert r.as_dict() == oracle_lib.screen_gate(y, 0, 0, q)
