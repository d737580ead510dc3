"""Decision distortion of reconstructed blocks (sse_recon): the oracle's plain
SSE equals numpy, its weighted SSE weighs a constant tile by the DC weight
(1.8 / 0.4625 of the 4x4 orthonormal DCT energy), and the CUDA distortion
equals the oracle bit for bit (plain and weighted, square and rectangular
sizes, clipped displayed windows)."""
import numpy as np
import pytest


def _blocks(w, h, n, fw=96, fh=64, seed=0):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, 256, (fh, fw)).astype(np.uint16)
    px = rng.integers(0, fw // 4, n) * 4
    py = rng.integers(0, fh // 4, n) * 4
    px = np.minimum(px, fw - w)
    py = np.minimum(py, fh - h)
    pos = np.stack([px, py], 1).astype(np.uint16)
    pred = rng.integers(-20, 276, (n, h, w)).astype(np.int32)
    resid = rng.integers(-40, 41, (n, h, w)).astype(np.int32)
    return src, pos, pred, resid


def test_oracle_plain_sse_equals_numpy(oracle_lib):
    src, pos, pred, resid = _blocks(8, 8, 20)
    got = oracle_lib.sse_recon(src, 90, 60, pos, pred, resid, 8, 8)
    for b in range(20):
        x, y = int(pos[b, 0]), int(pos[b, 1])
        vw, vh = max(0, min(90 - x, 8)), max(0, min(60 - y, 8))
        rec = np.clip(pred[b] + resid[b], 0, 255)[:vh, :vw]
        d = src[y:y + vh, x:x + vw].astype(np.int64) - rec
        assert got[b] == int((d * d).sum())


def test_oracle_weighted_sse_of_a_flat_tile(oracle_lib):
    for c in (1, 3, -7, 20):
        err = np.full((4, 4), c, np.int32)
        got = oracle_lib.weighted_sse(err)
        want = (1.8 / 0.4625) * 16.0 * c * c
        assert abs(got - want) <= 1e-5 * want


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(4, 4), (8, 8), (16, 16), (8, 16), (16, 4), (32, 32), (64, 64)])
@pytest.mark.parametrize("scale", [0.0, 1.0, 0.7])
def test_sse_recon_matches_oracle(mt_lib, oracle_lib, cuda, w, h, scale):
    fw, fh = 160, 128
    src, pos, pred, resid = _blocks(w, h, 64, fw, fh, seed=w * 100 + h)
    for vis in ((fw, fh), (fw - 5, fh - 3), (fw - 9, fh - 13)):
        ref = oracle_lib.sse_recon(src, vis[0], vis[1], pos, pred, resid, w, h, scale)
        got = mt_lib.sse_recon(src, vis[0], vis[1], pos, pred, resid, w, h, scale)
        assert np.array_equal(got, ref), (vis, np.nonzero(got != ref))
    got0 = mt_lib.sse_recon(src, fw, fh, pos, pred, None, w, h, scale)
    assert np.array_equal(got0, oracle_lib.sse_recon(src, fw, fh, pos, pred, None, w, h, scale))
