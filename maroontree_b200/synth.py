"""Seeded synthetic inputs for the intra RD path.

The reference measures on a private image corpus that is not available here,
so images come from a seeded generator with the shapes the benchmark names:
a sum of six 2-D sinusoids (1-40 cycles/image, random phase, amplitude <= 60)
over mid-grey, twelve hard-edged rectangles (six axis-aligned, six rotated)
in uniform colours, then Gaussian noise, rounded half away from zero and
clamped to 0..255.  The 1080p variant adds a 64-px-period texture band and a
smooth gradient quadrant.  A xoshiro128** stream drives every draw.
"""
import numpy as np

from . import abi


class Xoshiro128ss:
    """xoshiro128** (Blackman & Vigna) seeded through splitmix32."""

    def __init__(self, seed):
        s = []
        z = seed & 0xFFFFFFFF
        for _ in range(4):
            z = (z + 0x9E3779B9) & 0xFFFFFFFF
            t = z
            t = ((t ^ (t >> 16)) * 0x85EBCA6B) & 0xFFFFFFFF
            t = ((t ^ (t >> 13)) * 0xC2B2AE35) & 0xFFFFFFFF
            s.append(t ^ (t >> 16))
        self.s = s

    def next_u32(self):
        s = self.s
        r = (((s[1] * 5) & 0xFFFFFFFF) << 7 | ((s[1] * 5) & 0xFFFFFFFF) >> 25) & 0xFFFFFFFF
        r = (r * 9) & 0xFFFFFFFF
        t = (s[1] << 9) & 0xFFFFFFFF
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 11) | (s[3] >> 21)) & 0xFFFFFFFF
        return r

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * (self.next_u32() / 4294967296.0)

    def randint(self, lo, hi):  # inclusive
        return lo + self.next_u32() % (hi - lo + 1)


def generate_rgb(w, h, seed, sigma=4.0, variant="plain"):
    """Interleaved u8 RGB image (h, w, 3)."""
    rng = Xoshiro128ss(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.full((3, h, w), 128.0)
    for _ in range(6):
        f = rng.uniform(1.0, 40.0)
        th = rng.uniform(0.0, np.pi)
        arg = 2 * np.pi * f * (np.cos(th) * xx / w + np.sin(th) * yy / h)
        for c in range(3):
            a = rng.uniform(0.0, 60.0)
            ph = rng.uniform(0.0, 2 * np.pi)
            img[c] += a * np.sin(arg + ph)
    for k in range(12):
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        sw, sh = rng.uniform(w / 32, w / 4), rng.uniform(w / 32, w / 4)
        ang = rng.uniform(0.0, np.pi) if k >= 6 else 0.0
        col = [rng.randint(0, 255) for _ in range(3)]
        ca, sa = np.cos(ang), np.sin(ang)
        u = (xx - cx) * ca + (yy - cy) * sa
        v = -(xx - cx) * sa + (yy - cy) * ca
        m = (np.abs(u) <= sw / 2) & (np.abs(v) <= sh / 2)
        for c in range(3):
            img[c][m] = col[c]
    if variant == "1080p":
        band = (yy >= 256) & (yy < 384)
        tex = 40 * np.sin(2 * np.pi * xx / 64) * np.sin(2 * np.pi * yy / 64)
        for c in range(3):
            img[c][band] += tex[band]
        q = (xx >= w // 2) & (yy >= h // 2)
        g = 255.0 * ((xx - w // 2) + (yy - h // 2)) / (w / 2 + h / 2)
        for c in range(3):
            img[c][q] = g[q]
    noise_rng = np.random.default_rng(rng.next_u32())
    img = img + noise_rng.normal(0.0, sigma, size=img.shape)
    img = np.where(img >= 0, np.floor(img + 0.5), np.ceil(img - 0.5))
    return np.clip(img, 0, 255).astype(np.uint8).transpose(1, 2, 0).copy()


def rgb_to_luma(rgb):
    """Q13 BT.601 luma of the reference's CSC (src/encoder.rs:113-127, :403-409)."""
    r = rgb[..., 0].astype(np.int32)
    g = rgb[..., 1].astype(np.int32)
    b = rgb[..., 2].astype(np.int32)
    y = (2449 * r + 4809 * g + 934 * b + 4096) >> 13
    return np.clip(y, 0, 255).astype(np.uint16)


def synthetic_recon(src, seed, amp=3):
    """A reconstruction snapshot: the source plus small seeded coding error."""
    rng = np.random.default_rng(seed)
    noise = rng.integers(-amp, amp + 1, size=src.shape)
    return np.clip(src.astype(np.int32) + noise, 0, 255).astype(np.uint16)


def _rand_cdf(rng, nsym, width):
    cuts = np.sort(rng.integers(1, 32768, size=nsym - 1))[::-1]
    out = np.zeros(width, np.uint16)
    out[: nsym - 1] = cuts
    return out


def synthetic_cdfs(seed, n_eob_bins=7, n_txtp=7):
    """A valid decision-CDF slice (strictly decreasing inverse CDFs ending in 0)."""
    rng = np.random.default_rng(seed)
    c = abi.CoefCdfs()
    flat = {}
    flat["txb_skip"] = np.stack([_rand_cdf(rng, 2, 2) for _ in range(13)])
    flat["base_tok"] = np.stack([_rand_cdf(rng, 4, 4) for _ in range(42)])
    flat["br_tok"] = np.stack([_rand_cdf(rng, 4, 4) for _ in range(21)])
    flat["eob_base"] = np.stack([_rand_cdf(rng, 3, 3) for _ in range(4)])
    flat["eob_hi"] = np.stack([_rand_cdf(rng, 2, 2) for _ in range(11)])
    flat["eob_bin"] = _rand_cdf(rng, n_eob_bins, 11)
    flat["dc_sign"] = np.stack([_rand_cdf(rng, 2, 2) for _ in range(3)])
    flat["txtp"] = np.stack([_rand_cdf(rng, n_txtp, 16) for _ in range(13)])
    for k, v in flat.items():
        arr = np.ctypeslib.as_array(getattr(c, k))
        arr[...] = v.reshape(arr.shape)
    return c


def block_flags(px, py, fw, fh, n=8):
    """Deterministic neighbour availability for a block on the n-grid."""
    bx, by = px // n, py // n
    have_tr = py > 0 and px + n < fw and (bx % 2 == 0 or by % 2 == 0)
    have_bl = px > 0 and py + n < fh and (bx % 2 == 1 and by % 2 == 0)
    return (abi.CAND_HAVE_TR if have_tr else 0) | (abi.CAND_HAVE_BL if have_bl else 0)


def level_candidates(fw, fh, modes, tx_types, deltas=(0,), n=8, seed=0):
    """All (block, mode, angle delta, tx type) candidates of one 8x8 level,
    block-major then mode, delta, type (the order the reference's mode loops
    evaluate within a block)."""
    rng = np.random.default_rng(seed)
    bxs = np.arange(0, fw - n + 1, n)
    bys = np.arange(0, fh - n + 1, n)
    combos = []
    for m in modes:
        ds = deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)
        for d in ds:
            for t in tx_types:
                combos.append((m, d, t))
    nb = len(bxs) * len(bys)
    out = np.zeros(nb * len(combos), abi.CANDIDATE_DTYPE)
    py_g, px_g = np.meshgrid(bys, bxs, indexing="ij")
    px_f, py_f = px_g.ravel(), py_g.ravel()
    flags = np.array([block_flags(int(x), int(y), fw, fh, n) for x, y in zip(px_f, py_f)], np.uint8)
    k = len(combos)
    out["px"] = np.repeat(px_f, k)
    out["py"] = np.repeat(py_f, k)
    cm = np.array(combos, np.int32)
    out["mode"] = np.tile(cm[:, 0], nb)
    out["angle_delta"] = np.tile(cm[:, 1], nb)
    out["tx_type"] = np.tile(cm[:, 2], nb)
    out["flags"] = np.repeat(flags, k)
    out["dcs_ctx"] = rng.integers(0, 3, size=nb).repeat(k)
    out["skip_ctx"] = 0
    out["mode_bits"] = (rng.random(len(out)) * 6 + 1).astype(np.float32)
    return out


def level_blocks(fw, fh, n=8, seed=0):
    """Block records of one 8x8 level (raster order) with deterministic
    neighbour flags, contexts and mode-signalling bits."""
    rng = np.random.default_rng(seed)
    bys, bxs = np.meshgrid(np.arange(0, fh - n + 1, n), np.arange(0, fw - n + 1, n), indexing="ij")
    px, py = bxs.ravel(), bys.ravel()
    out = np.zeros(len(px), abi.BLOCK8_DTYPE)
    out["px"], out["py"] = px, py
    out["flags"] = [block_flags(int(x), int(y), fw, fh, n) for x, y in zip(px, py)]
    out["dcs_ctx"] = rng.integers(0, 3, size=len(px))
    out["skip_ctx"] = 0
    out["mode_bits"] = (rng.random((len(px), 13)) * 6 + 1).astype(np.float32)
    return out


def level_combos(modes, tx_types, deltas=(0,)):
    """(mode, angle delta, tx type) combos in the reference's evaluation order
    (mode, then delta, then type)."""
    rows = []
    for m in modes:
        ds = deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)
        for d in ds:
            for t in tx_types:
                rows.append((m, d, t, 0))
    return _combos(rows)


def _combos(rows):
    out = np.zeros(len(rows), abi.COMBO_DTYPE)
    for i, (m, d, t, _) in enumerate(rows):
        out[i] = (m, d, t, 0)
    return out


def candidates_of_level(blocks, combos):
    """The candidate list a level launch evaluates, combo-major (index c * nblocks + b)."""
    nb, nc = len(blocks), len(combos)
    out = np.zeros(nb * nc, abi.CANDIDATE_DTYPE)
    out["px"] = np.tile(blocks["px"], nc)
    out["py"] = np.tile(blocks["py"], nc)
    out["mode"] = np.repeat(combos["mode"], nb)
    out["angle_delta"] = np.repeat(combos["angle_delta"], nb)
    out["tx_type"] = np.repeat(combos["tx_type"], nb)
    out["flags"] = np.tile(blocks["flags"], nc)
    out["dcs_ctx"] = np.tile(blocks["dcs_ctx"], nc)
    out["skip_ctx"] = np.tile(blocks["skip_ctx"], nc)
    out["mode_bits"] = blocks["mode_bits"][np.tile(np.arange(nb), nc), np.repeat(combos["mode"], nb)]
    return out


def best_of_level(results, nblocks, ncombos):
    """Per-block argmin of combo-major results with the first-minimum rule."""
    cost = results["cost"].reshape(ncombos, nblocks)
    return np.argmin(cost, axis=0)
