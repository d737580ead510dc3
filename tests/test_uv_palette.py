"""UV palette candidates (exact_uv_palette, uv_pair_histogram,
lossy_uv_palette_from_hist, viterbi_uv_palette_map: src/coder/palette.rs:199-431,
:1053-1076; uv_nearest_indices: src/kmeans.rs:37-68).

The reference holds no test of its own for these functions, so the oracle is
pinned here against the properties the functions define and against a short
numpy restatement of the lossy centres:
- exact palettes equal the sorted set of the block's pairs, with a lossless map;
- dominant-pair candidates are the most frequent pairs;
- k-means candidates come from the weighted-quantile starts and the Lloyd passes;
- nearest maps take the first closest centre;
- each Viterbi row costs no more than the nearest row under the same row above.

The GPU tests compare the device kernel's candidates and maps with the oracle
bit for bit."""
import numpy as np
import pytest


def _costs(seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.15, 7.0, (7, 5, 8)).astype(np.float32)


def _planes(fw, fh, w, h, seed, bd=8):
    """Screen-like chroma: per block either flat, 2..8 exact pairs, pairs with
    sparse noise (lossy), or textured (many pairs)."""
    rng = np.random.default_rng(seed)
    top = (1 << bd) - 1
    u = np.zeros((fh, fw), np.uint16)
    v = np.zeros((fh, fw), np.uint16)
    kinds = []
    for by in range(0, fh - h + 1, h):
        for bx in range(0, fw - w + 1, w):
            kind = int(rng.integers(0, 4))
            kinds.append(kind)
            if kind == 0:
                u[by:by + h, bx:bx + w] = rng.integers(0, top + 1)
                v[by:by + h, bx:bx + w] = rng.integers(0, top + 1)
                continue
            k = int(rng.integers(2, 9)) if kind == 1 else int(rng.integers(3, 12))
            pu = rng.integers(0, top + 1, k)
            pv = rng.integers(0, top + 1, k)
            pv[-1] = pv[0] if k > 2 else pv[-1]  # a shared V value: the pair order needs U
            idx = rng.integers(0, k, (h, w))
            bu, bv = pu[idx], pv[idx]
            if kind == 2:
                noise = rng.random((h, w)) < 0.15
                bu = np.where(noise, np.clip(bu + rng.integers(-6, 7, (h, w)), 0, top), bu)
                bv = np.where(noise, np.clip(bv + rng.integers(-6, 7, (h, w)), 0, top), bv)
            elif kind == 3:
                bu = rng.integers(0, top + 1, (h, w))
            u[by:by + h, bx:bx + w] = bu
            v[by:by + h, bx:bx + w] = bv
    return u, v, kinds


def _grid(fw, fh, w, h):
    ys, xs = np.meshgrid(np.arange(0, fh - h + 1, h), np.arange(0, fw - w + 1, w), indexing="ij")
    return np.stack([xs.ravel(), ys.ravel()], axis=1).astype(np.uint16)


def _opts(lam, seed):
    import maroontree_b200 as mt
    return mt.palette_opts(viterbi_lambda=lam, color_costs=_costs(seed))


def _hist(bu, bv):
    pairs, counts = np.unique(np.stack([bu.ravel(), bv.ravel()], 1).astype(np.int64), axis=0, return_counts=True)
    return [tuple(map(int, p)) for p in pairs], [int(c) for c in counts]


def _kmeans_centres(pairs, counts, colors):
    """lossy_uv_palette_from_hist's k-means leg, restated in numpy terms."""
    if len(pairs) < 2 or colors > len(pairs):
        return None
    if colors == len(pairs):
        return sorted(pairs)
    total = sum(counts)
    cum = np.cumsum(counts)
    init = []
    for i in range(colors):
        target = (2 * i + 1) * total // (2 * colors)
        e = int(np.searchsorted(cum, target, side="right"))
        init.append(pairs[min(e, len(pairs) - 1)])
    init = [p for j, p in enumerate(init) if j == 0 or p != init[j - 1]]
    if len(init) != colors:
        return None
    P = np.array(pairs, np.int64)
    W = np.array(counts, np.int64)
    for _ in range(8):
        c = np.array(init, np.int64)
        d = ((P[:, None, :] - c[None, :, :]) ** 2).sum(-1)
        a = d.argmin(1)
        for i in range(len(init)):
            m = a == i
            n = int(W[m].sum())
            if n:
                init[i] = (int((P[m, 0] * W[m]).sum() + n // 2) // n, int((P[m, 1] * W[m]).sum() + n // 2) // n)
        init = sorted(set(init))
        if len(init) != colors:
            return None
    return init


def _top_centres(pairs, counts, colors):
    if len(pairs) < 2 or colors > len(pairs):
        return None
    order = sorted(range(len(pairs)), key=lambda e: (-counts[e], pairs[e]))
    return sorted(pairs[e] for e in order[:colors])


def _cand_pairs(cd):
    n = int(cd["n_colors"])
    return [(int(cd["u"][i]), int(cd["v"][i])) for i in range(n)]


@pytest.mark.parametrize("w,h", [(8, 8), (16, 16), (4, 8), (32, 32)])
def test_oracle_candidates_pinned(oracle_lib, w, h):
    fw, fh = 8 * max(w, 8), 6 * max(h, 8)
    u, v, kinds = _planes(fw, fh, w, h, w * 7 + h)
    pos = _grid(fw, fh, w, h)
    cands, maps = oracle_lib.uv_palette(u, v, w, h, pos, _opts(0.0, 3))
    seen = set()
    for b, (px, py) in enumerate(pos):
        bu, bv = u[py:py + h, px:px + w].astype(np.int64), v[py:py + h, px:px + w].astype(np.int64)
        pairs, counts = _hist(bu, bv)
        cb, mb = cands[b], maps[b]
        if 2 <= len(pairs) <= 8:
            seen.add("exact")
            assert cb[0]["exact"] == 1 and _cand_pairs(cb[0]) == pairs
            pu = np.array([p[0] for p in pairs])[mb[0]]
            pv = np.array([p[1] for p in pairs])[mb[0]]
            assert np.array_equal(pu, bu) and np.array_equal(pv, bv)
            assert (cb["n_colors"][1:] == 0).all() and not mb[1:].any()
            continue
        assert (cb["exact"] == 0).all()
        want = [_kmeans_centres(pairs, counts, 8), _kmeans_centres(pairs, counts, 4), _top_centres(pairs, counts, 8),
                _top_centres(pairs, counts, 4)]
        for s in range(4):
            if want[s] is None:
                assert cb[s]["n_colors"] == 0 and not mb[s].any()
                seen.add("empty")
                continue
            seen.add("lossy")
            assert _cand_pairs(cb[s]) == want[s], (b, s)
            c = np.array(want[s], np.int64)
            d = (bu[..., None] - c[:, 0]) ** 2 + (bv[..., None] - c[:, 1]) ** 2
            assert np.array_equal(mb[s], d.argmin(-1)), (b, s)  # argmin: the first closest centre
    assert seen == {"exact", "lossy", "empty"}


def _row_cost(oracle_lib, row, above, dist, lam, costs, y):
    tot = 0.0
    for x, i in enumerate(row):
        tot += float(dist[x, i])
        if x == 0 and y == 0:
            continue
        l = None if x == 0 else int(row[x - 1])
        up = None if y == 0 else int(above[x])
        ul = int(above[x - 1]) if (x > 0 and y > 0) else 0
        ctx, sym = oracle_lib.palette_color_ctx_nb(l, up, ul, int(i))
        n = dist.shape[1]
        tot += lam * float(costs[n - 2][ctx][sym])
    return tot


def test_oracle_viterbi_rows_beat_nearest(oracle_lib):
    w = h = 8
    u, v, _ = _planes(64, 48, w, h, 11)
    pos = _grid(64, 48, w, h)
    lam, costs = 37.0, _costs(5)
    cands, maps = oracle_lib.uv_palette(u, v, w, h, pos, _opts(lam, 5))
    checked = 0
    for b, (px, py) in enumerate(pos):
        bu, bv = u[py:py + h, px:px + w].astype(np.int64), v[py:py + h, px:px + w].astype(np.int64)
        for s in range(4):
            cd = cands[b, s]
            if cd["n_colors"] == 0 or cd["exact"]:
                continue
            c = np.array(_cand_pairs(cd), np.int64)
            dist = ((bu[..., None] - c[:, 0]) ** 2 + (bv[..., None] - c[:, 1]) ** 2).astype(np.float64)
            near = dist.argmin(-1)
            m = maps[b, s]
            assert m.max() < len(c)
            for y in range(h):
                above = m[y - 1] if y else None
                vit = _row_cost(oracle_lib, m[y], above, dist[y], lam, costs, y)
                alt = _row_cost(oracle_lib, near[y], above, dist[y], lam, costs, y)
                assert vit <= alt * (1 + 1e-5) + 1e-3, (b, s, y)
            checked += 1
    assert checked > 10


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,bd,lam", [(4, 4, 8, 0.0), (8, 8, 8, 29.0), (16, 16, 8, 0.0), (16, 16, 10, 55.5),
                                        (32, 32, 8, 18.25), (8, 16, 12, 0.0), (32, 32, 10, 0.0), (16, 8, 8, 41.0)])
def test_uv_palette_gpu_matches_oracle(mt_lib, oracle_lib, cuda, w, h, bd, lam):
    fw, fh = 12 * w, 8 * h
    u, v, _ = _planes(fw, fh, w, h, w * h + bd, bd=bd)
    pos = _grid(fw, fh, w, h)
    opts = mt_lib.palette_opts(viterbi_lambda=lam, color_costs=_costs(w + h + bd))
    cands, maps = mt_lib.uv_palette(u, v, w, h, pos, opts, want_maps=True)
    wc, wm = oracle_lib.uv_palette(u, v, w, h, pos, opts)
    assert cands.tobytes() == wc.tobytes()
    assert np.array_equal(maps, wm)
    assert (cands["exact"][:, 0] == 1).any() and (cands["n_colors"][:, 3] > 0).any()
