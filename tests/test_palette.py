"""Lossy luma palette candidates (src/coder/palette.rs, src/kmeans.rs).

The oracle is pinned by the reference's own palette tests, restated:
histogram_kmeans_palette_basics (palette.rs:2260-2316), the DP review cases
and the brute-force optimality check (:2444-2505), the nearest-index tie rule
(kmeans.rs:213-257) and palette_color_ctx_nb against the map form
(:2362-2393).  The GPU tests compare the device kernels' candidates, maps
and index bits with the oracle bit for bit."""
import itertools

import numpy as np
import pytest

from maroontree_b200 import abi, synth


def hist_sse(hist, centers):
    return sum(c * min((v - m) ** 2 for m in centers) for v, c in hist)


def test_histogram_and_exact_palette(oracle_lib):
    import maroontree_b200 as mt

    plane = np.zeros((32, 32), np.uint16)
    for y in range(16):
        for x in range(16):
            plane[y + 4, x + 4] = [10, 80, 150, 220][(x // 4 + y // 4) % 4]
    vals, cnts = oracle_lib.block_color_histogram(plane, 4, 4, 16, 16)
    assert vals.tolist() == [10, 80, 150, 220] and cnts.sum() == 256
    cands, maps = oracle_lib.luma_palette(plane, 16, 16, [(4, 4)], mt.palette_opts())
    exact = cands[0][2]  # 4 colours
    assert exact["n_colors"] == 4 and exact["colors"][:4].tolist() == [10, 80, 150, 220]
    recon = np.asarray(exact["colors"][:4])[maps[0, 2]]
    assert np.array_equal(recon, plane[4:20, 4:20])
    assert cands[0][0]["n_colors"] == 2  # lossy: 2 colours over 4 values
    assert cands[0][9]["n_colors"] == 0  # dominant colours need fewer colours than values
    flat = np.full((32, 32), 7, np.uint16)
    assert oracle_lib.block_color_histogram(flat, 4, 4, 16, 16) is None
    noisy = ((np.arange(32 * 32) * 37) % 251).astype(np.uint16).reshape(32, 32)
    assert oracle_lib.block_color_histogram(noisy, 0, 0, 16, 16) is None


def test_dp_review_cases(oracle_lib):
    a = [(0, 90), (80, 5), (100, 5)]
    assert oracle_lib.dp_palette_center_sets(a, 2)[0] == [0, 90]
    assert hist_sse(a, [0, 90]) == 1000
    b = [(51, 11), (169, 7), (181, 18), (222, 16), (241, 15)]
    assert oracle_lib.dp_palette_center_sets(b, 2)[0] == [51, 207]
    assert hist_sse(b, [51, 207]) == 43_216
    assert hist_sse(b, [139, 231]) == 126_032


def test_dp_centers_are_optimal(oracle_lib):
    seed = [0x12345677]

    def rnd():
        s = seed[0]
        s ^= (s << 13) & 0xFFFFFFFF
        s ^= s >> 17
        s ^= (s << 5) & 0xFFFFFFFF
        seed[0] = s
        return s

    def best(hist, k):
        if k == 1:
            w = sum(c for _, c in hist)
            m = (sum(v * c for v, c in hist) + w // 2) // w
            return hist_sse(hist, [m])
        return min(best(hist[:i], k - 1) + best(hist[i:], 1) for i in range(k - 1, len(hist)))

    for _ in range(120):
        h = 2 + rnd() % 9
        vals = []
        while len(vals) < h:
            v = rnd() % 256
            if v not in vals:
                vals.append(v)
        vals.sort()
        hist = [(v, 1 + rnd() % 40) for v in vals]
        sets = oracle_lib.dp_palette_center_sets(hist, 8)
        for n in range(2, 9):
            s = sets[n - 2]
            if n > h:
                assert s == []
                continue
            assert len(s) == n and all(p < q for p, q in zip(s, s[1:]))
            assert hist_sse(hist, s) == best(hist, n), (hist, n)


def test_nearest_indices_ties_and_tails(oracle_lib):
    w, h, stride = 29, 5, 48
    u = ((np.arange(stride * 16) * 37) % 4096).astype(np.uint16)
    u[2 * stride + 3], u[2 * stride + 4] = 0, 4095
    plane = u.reshape(16, stride)
    centers = [0, 4095, 2048, 2048, 1]
    for k in range(1, 6):
        got = oracle_lib.luma_nearest_indices(plane, 3, 2, w, h, centers[:k])
        blk = plane[2:2 + h, 3:3 + w].astype(np.int64).reshape(-1, 1)
        want = np.argmin((blk - np.asarray(centers[:k], np.int64)) ** 2, axis=1)  # first minimum
        assert np.array_equal(got, want), k


def test_color_ctx_nb_matches_map(oracle_lib):
    rng = np.random.default_rng(3)
    for n in range(2, 9):
        for _ in range(4):
            m = rng.integers(0, n, (6, 7)).astype(np.uint8)
            for y, x in itertools.product(range(6), range(7)):
                if (y, x) == (0, 0):
                    continue
                l = int(m[y, x - 1]) if x else None
                up = int(m[y - 1, x]) if y else None
                ul = int(m[y - 1, x - 1]) if x and y else 0
                assert oracle_lib.palette_color_ctx(m, 7, y, x) == oracle_lib.palette_color_ctx_nb(l, up, ul,
                                                                                                   int(m[y, x]))
    assert oracle_lib.palette_color_ctx_nb(1, 1, 1, 1) == (4, 0)
    assert oracle_lib.palette_color_ctx_nb(2, 5, 7, 3) == (1, 5)  # scored 2, 5, 7; then 0, 1, 3


def test_dirty_log2f(oracle_lib):
    for k in range(2, 9):
        assert abs(oracle_lib.dirty_log2f(float(k)) - np.log2(k)) < 1e-5


def _costs(seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.15, 7.0, (7, 5, 8)).astype(np.float32)


def _grid(fw, fh, w, h):
    ys, xs = np.meshgrid(np.arange(0, fh - h + 1, h), np.arange(0, fw - w + 1, w), indexing="ij")
    return np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.uint16)


def test_oracle_nearest_and_smoothing_glue(oracle_lib):
    """lossy_luma_palette_from_centers without the Viterbi: the nearest map,
    then smooth_palette_map in raster order (palette.rs:1173-1216)."""
    import maroontree_b200 as mt

    src = synth.screen_luma(64, 64, 5)
    pos = _grid(64, 64, 16, 16)
    cands, maps = oracle_lib.luma_palette(src, 16, 16, pos, mt.palette_opts(smooth_t=24, smooth_guard=True,
                                                                            color_costs=_costs(1)))
    checked = 0
    for b, (px, py) in enumerate(pos):
        for s in range(abi.PALETTE_SLOTS):
            cd = cands[b, s]
            if cd["n_colors"] == 0:
                continue
            c = [int(v) for v in cd["colors"][:cd["n_colors"]]]
            m = oracle_lib.luma_nearest_indices(src, int(px), int(py), 16, 16, c).reshape(16, 16).astype(int)
            blk = src[py:py + 16, px:px + 16].astype(int)
            for y in range(16):
                for x in range(16):
                    v, i0 = blk[y, x], m[y, x]
                    d0 = abs(v - c[i0])
                    if d0 == 0:
                        continue
                    best, best_d = i0, d0 + 24
                    if x and m[y, x - 1] != i0 and abs(v - c[m[y, x - 1]]) <= best_d:
                        best, best_d = m[y, x - 1], abs(v - c[m[y, x - 1]])
                    if y and m[y - 1, x] not in (i0, best) and abs(v - c[m[y - 1, x]]) < best_d:
                        best = m[y - 1, x]
                    m[y, x] = best
            assert np.array_equal(maps[b, s], m), (b, s)
            checked += 1
    assert checked > 20


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,bd,mode", [(8, 8, 8, "viterbi"), (16, 16, 8, "viterbi"), (16, 16, 8, "smooth"),
                                         (32, 32, 10, "viterbi"), (64, 64, 8, "smooth"), (16, 8, 8, "plain"),
                                         (32, 16, 12, "smooth"), (64, 64, 10, "viterbi")])
def test_luma_palette_gpu_matches_oracle(mt_lib, oracle_lib, cuda, w, h, bd, mode):
    src = synth.screen_luma(192, 128, w + h + bd, bd=bd)
    pos = _grid(192, 128, w, h)
    pos[1] = (192 - w + 4, 0)  # crosses the right edge: empty slots
    opts = mt_lib.palette_opts(smooth_t=24 if mode == "smooth" else 0, smooth_guard=True,
                               viterbi_lambda=21.5 if mode == "viterbi" else 0.0, color_costs=_costs(w * h + bd))
    cands, maps = mt_lib.luma_palette(src, w, h, pos, opts, bd=bd, want_maps=True)
    wc, wm = oracle_lib.luma_palette(src, w, h, pos, opts, bd=bd)
    assert cands.tobytes() == wc.tobytes()
    assert np.array_equal(maps, wm)
    assert (cands["n_colors"][1] == 0).all()
    assert (cands["hist_len"] > 0).sum() > len(pos) // 4
