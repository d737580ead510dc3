"""Seeded synthetic inputs for the intra RD path.

The reference measures on a private image corpus that is not available here,
so images come from a seeded generator with the shapes the benchmark names:
a sum of six 2-D sinusoids (1-40 cycles/image, random phase, amplitude <= 60)
over mid-grey, twelve hard-edged rectangles (six axis-aligned, six rotated)
in uniform colours, then Gaussian noise, rounded half away from zero and
clamped to 0..255.  The 1080p variant adds a 64-px-period texture band and a
smooth gradient quadrant.  The large variant (the 4096x4096 frame) keeps the
noise to the left half and makes the right half piecewise constant: a grid
of cells with seeded cut positions, each in one uniform colour.  A
xoshiro128** stream drives every draw.
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
    half = None
    if variant == "large":
        half = xx >= w // 2
        xs = np.sort(np.array([w // 2] + [int(rng.uniform(w // 2, w)) for _ in range(15)] + [w]))
        ys = np.sort(np.array([0] + [int(rng.uniform(0, h)) for _ in range(15)] + [h]))
        cx = np.searchsorted(xs, xx[0], side="right") - 1
        cy = np.searchsorted(ys, yy[:, 0], side="right") - 1
        cols = np.array([[rng.randint(0, 255) for _ in range(3)] for _ in range(len(xs) * len(ys))], np.float64)
        cell = cy[:, None] * len(xs) + cx[None, :]
        for c in range(3):
            img[c][half] = cols[cell, c][half]
    noise_rng = np.random.default_rng(rng.next_u32())
    noise = noise_rng.normal(0.0, sigma, size=img.shape)
    if half is not None:
        noise[:, half] = 0.0
    img = img + noise
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
    # drawn last so the fields above keep their values for a given seed
    flat["eob_bin_1d"] = _rand_cdf(rng, n_eob_bins, 11)
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


def level_combos(modes, tx_types, deltas=(0,), no_trellis_types=(), delta_bits=None):
    """(mode, angle delta, tx type) combos in the reference's evaluation order
    (mode, then delta, then type); types in no_trellis_types carry
    MT_COMBO_NO_TRELLIS.  delta_bits(mode, delta) -> the angle-delta symbol
    cost of a nonzero delta (the proxy's delta pass); 0 for delta 0."""
    rows = []
    for m in modes:
        ds = deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)
        for d in ds:
            extra = float(delta_bits(m, d)) if (delta_bits is not None and d != 0) else 0.0
            for t in tx_types:
                rows.append((m, d, t, abi.COMBO_NO_TRELLIS if t in no_trellis_types else 0, extra))
    return _combos(rows)


def _combos(rows):
    out = np.zeros(len(rows), abi.COMBO_DTYPE)
    for i, row in enumerate(rows):
        out[i] = tuple(row) + (0.0,) * (5 - len(row))
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
    no_tr = np.where(combos["flags"] & abi.COMBO_NO_TRELLIS, abi.CAND_NO_TRELLIS, 0).astype(np.uint8)
    out["flags"] = np.tile(blocks["flags"], nc) | np.repeat(no_tr, nb)
    out["dcs_ctx"] = np.tile(blocks["dcs_ctx"], nc)
    out["skip_ctx"] = np.tile(blocks["skip_ctx"], nc)
    out["mode_bits"] = blocks["mode_bits"][np.tile(np.arange(nb), nc), np.repeat(combos["mode"], nb)]
    out["extra_bits"] = np.repeat(combos["bits"], nb)
    return out


def best_of_level(results, nblocks, ncombos):
    """Per-block argmin of combo-major results with the first-minimum rule."""
    cost = results["cost"].reshape(ncombos, nblocks)
    return np.argmin(cost, axis=0)


# ---------------------------------------------------------------------------
# Block geometry and reconstructions for the in-loop filters.

def partition_maps(nc4, nr4, seed, sb4=16, split_bias=0.55):
    """Random AV1-shaped block geometry over an nr4 x nc4 grid of 4x4 cells.

    Each sb4 x sb4 superblock is partitioned recursively with the AV1
    partition types (NONE, SPLIT, HORZ, VERT, HORZ_4, VERT_4 and the 3-way
    HORZ_A/B, VERT_A/B); blocks are clipped to the grid.  Returns
    (bw4, bh4, vedge4, hedge4, block_id): u8 block width / height in 4-sample
    units per cell, u8 flags where a block starts at the cell's column / row,
    and an int32 block index per cell."""
    rng = np.random.default_rng(seed)
    bw4 = np.zeros((nr4, nc4), np.uint8)
    bh4 = np.zeros((nr4, nc4), np.uint8)
    ve = np.zeros((nr4, nc4), np.uint8)
    he = np.zeros((nr4, nc4), np.uint8)
    bid = np.full((nr4, nc4), -1, np.int32)
    count = [0]

    def put(r, c, h, w):
        if r >= nr4 or c >= nc4:
            return
        r1, c1 = min(r + h, nr4), min(c + w, nc4)
        bw4[r:r1, c:c1] = w
        bh4[r:r1, c:c1] = h
        ve[r:r1, c] = 1
        he[r, c:c1] = 1
        bid[r:r1, c:c1] = count[0]
        count[0] += 1

    def node(r, c, s):
        if r >= nr4 or c >= nc4:
            return
        kinds = ["none"]
        if s > 1:
            kinds += ["split", "horz", "vert", "horz_a", "horz_b", "vert_a", "vert_b"]
        if s >= 4:
            kinds += ["horz_4", "vert_4"]
        if s > 1 and rng.random() < split_bias:
            kind = "split"
        else:
            kind = kinds[int(rng.integers(len(kinds)))]
        hs = s // 2
        if kind == "none":
            put(r, c, s, s)
        elif kind == "split":
            for dr in (0, hs):
                for dc in (0, hs):
                    node(r + dr, c + dc, hs)
        elif kind == "horz":
            put(r, c, hs, s)
            put(r + hs, c, hs, s)
        elif kind == "vert":
            put(r, c, s, hs)
            put(r, c + hs, s, hs)
        elif kind == "horz_4":
            for k in range(4):
                put(r + k * s // 4, c, s // 4, s)
        elif kind == "vert_4":
            for k in range(4):
                put(r, c + k * s // 4, s, s // 4)
        elif kind == "horz_a":
            put(r, c, hs, hs)
            put(r, c + hs, hs, hs)
            put(r + hs, c, hs, s)
        elif kind == "horz_b":
            put(r, c, hs, s)
            put(r + hs, c, hs, hs)
            put(r + hs, c + hs, hs, hs)
        elif kind == "vert_a":
            put(r, c, hs, hs)
            put(r + hs, c, hs, hs)
            put(r, c + hs, s, hs)
        else:  # vert_b
            put(r, c, s, hs)
            put(r, c + hs, hs, hs)
            put(r + hs, c + hs, hs, hs)

    for r in range(0, nr4, sb4):
        for c in range(0, nc4, sb4):
            node(r, c, sb4)
    return bw4, bh4, ve, he, bid


def blocky_plane(w, h, block_id, seed, maxv=255):
    """A reconstruction-like plane: per block a flat level, a gentle ramp or
    texture, with small steps between neighbouring blocks, so that every branch
    of the loop filter (flat 16 / flat 8 / 6 / narrow with and without high
    edge variance, and rejected lines) is reached."""
    rng = np.random.default_rng(seed)
    nb = int(block_id.max()) + 1
    base = np.clip(128 + np.cumsum(rng.integers(-6, 7, nb)), 16, maxv - 16)
    style = rng.integers(0, 5, nb)
    gx = rng.integers(-2, 3, nb)
    gy = rng.integers(-2, 3, nb)
    cell = np.repeat(np.repeat(block_id, 4, axis=0), 4, axis=1)
    ch, cw = cell.shape
    full = np.zeros((h, w), np.int64)
    bidp = np.full((h, w), 0, np.int64)
    bidp[:min(h, ch), :min(w, cw)] = cell[:min(h, ch), :min(w, cw)]
    bidp[bidp < 0] = 0
    yy, xx = np.mgrid[0:h, 0:w]
    b = bidp
    v = base[b].astype(np.int64)
    s = style[b]
    v = v + np.where(s == 1, rng.integers(-1, 2, (h, w)), 0)
    v = v + np.where(s == 2, (gx[b] * (xx % 16) + gy[b] * (yy % 16)) // 4, 0)
    v = v + np.where(s == 3, rng.integers(-12, 13, (h, w)), 0)
    v = v + np.where(s == 4, rng.integers(-3, 4, (h, w)), 0)
    full[:] = np.clip(v, 0, maxv)
    return full.astype(np.uint16)


def cdef_inputs(disp_w, disp_h, sub_x, sub_y, mono, seed, skip_frac=0.3, rgb=None):
    """Source and reconstruction planes plus a per-8x8 skip map for the frame
    CDEF: luma from the synthetic RGB image (or the given disp_h x disp_w
    image), chroma a contrast-reduced copy of it; the reconstruction adds
    seeded error whose amplitude varies per 64x64 unit (0 .. 12, with or
    without block-edge ringing), so that CDEF helps some units and not others.
    Planes are edge-padded to multiples of 8."""
    w8, h8 = (disp_w + 7) & ~7, (disp_h + 7) & ~7
    rng = np.random.default_rng(seed)
    y = rgb_to_luma(generate_rgb(disp_w, disp_h, seed) if rgb is None else rgb).astype(np.int32)
    y = np.pad(y, ((0, h8 - disp_h), (0, w8 - disp_w)), mode="edge")
    planes = [y]
    if not mono:
        sub = y[::1 << sub_y, ::1 << sub_x]
        planes.append(np.clip(128 + (sub - 128) // 3, 0, 255))
        planes.append(np.clip(128 - (sub - 128) // 4, 0, 255))
    src, rec = [], []
    uc, ur = (w8 + 63) // 64, (h8 + 63) // 64
    amp_u = rng.choice([0, 1, 2, 4, 7, 12], size=(ur, uc))
    ring_u = rng.choice([0, 1, 3], size=(ur, uc))
    for k, p in enumerate(planes):
        sx, sy = (0, 0) if k == 0 else (sub_x, sub_y)
        h, w = p.shape
        yy, xx = np.mgrid[0:h, 0:w]
        amp = amp_u[(yy << sy) // 64, (xx << sx) // 64]
        noise = np.round(rng.uniform(-1, 1, size=p.shape) * amp).astype(np.int32)
        ring = np.where(((xx % (8 >> sx)) == 0) | ((yy % (8 >> sy)) == 0),
                        ring_u[(yy << sy) // 64, (xx << sx) // 64] * amp // 2, 0)
        src.append(p.astype(np.uint16))
        rec.append(np.clip(p + noise + ring, 0, 255).astype(np.uint16))
    skip8 = (rng.random((h8 // 8, w8 // 8)) < skip_frac).astype(np.uint8)
    if uc * ur > 1:
        skip8[:8, :8] = 1  # one all-skip unit
    return src, rec, skip8


def transform_maps(bw4, bh4, block_id, seed, split_p=0.4):
    """Luma transform-block maps inside the prediction blocks of
    ``partition_maps``: each block of at least 8x8 is split into a 2x2 grid of
    transforms with probability split_p (tx_depth 1).  Returns (tw4, th4,
    tv4, tt4) like the prediction maps."""
    rng = np.random.default_rng(seed)
    nr4, nc4 = bw4.shape
    tw, th = bw4.copy(), bh4.copy()
    tv = np.zeros_like(bw4)
    tt = np.zeros_like(bw4)
    nb = int(block_id.max()) + 1
    split = rng.random(nb) < split_p
    seen = np.zeros(nb, bool)
    for r in range(nr4):
        for c in range(nc4):
            b = block_id[r, c]
            if b < 0 or seen[b]:
                continue
            seen[b] = True
            w, h = int(bw4[r, c]), int(bh4[r, c])
            sw, sh = (w // 2, h // 2) if (split[b] and w >= 2 and h >= 2) else (w, h)
            for dr in range(0, h, sh):
                for dc in range(0, w, sw):
                    r0, c0 = r + dr, c + dc
                    if r0 >= nr4 or c0 >= nc4:
                        continue
                    r1, c1 = min(r0 + sh, nr4), min(c0 + sw, nc4)
                    tw[r0:r1, c0:c1] = sw
                    th[r0:r1, c0:c1] = sh
                    tv[r0:r1, c0] = 1
                    tt[r0, c0:c1] = 1
    return tw, th, tv, tt


def screen_luma(w, h, seed, photo_frac=0.3, glyph_px=(8, 12), bd=8):
    """Screen-content luma (u16, h x w): flat UI panels, rows of text drawn from a
    small glyph alphabet (exact repeats at arbitrary offsets, with an
    antialiasing level), and a photographic patch (the generator's luma)."""
    rng = np.random.default_rng(seed)
    top = (1 << bd) - 1
    img = np.full((h, w), int(0.92 * top), np.int32)
    # UI panels
    for _ in range(6):
        x0, y0 = rng.integers(0, w), rng.integers(0, h)
        img[y0:y0 + rng.integers(16, h // 3 + 17), x0:x0 + rng.integers(16, w // 3 + 17)] = int(rng.integers(0, top + 1))
    # glyph alphabet: binary masks with an antialiased edge level
    gw, gh = glyph_px
    glyphs = []
    for _ in range(24):
        m = (rng.random((gh, gw)) < 0.35).astype(np.int32)
        aa = (rng.random((gh, gw)) < 0.15).astype(np.int32)
        glyphs.append((m, aa))
    ink, mid = int(0.1 * top), int(0.5 * top)
    y = 4
    while y + gh < h * (1 - photo_frac):
        x = int(rng.integers(0, 24))
        while x + gw < w:
            if rng.random() < 0.8:
                m, aa = glyphs[int(rng.integers(0, len(glyphs)))]
                blk = img[y:y + gh, x:x + gw]
                blk[aa == 1] = mid
                blk[m == 1] = ink
            x += gw + int(rng.integers(0, 3))
        y += gh + int(rng.integers(2, 6))
    # photographic patch at the bottom
    ph = int(h * photo_frac)
    if ph > 0:
        lum = rgb_to_luma(generate_rgb(w, ph, int(seed) + 1)).astype(np.int32)
        img[h - ph:, :] = lum << (bd - 8)
    return np.clip(img, 0, top).astype(np.uint16)


def coef_ctx_bytes(rng, n):
    """Valid coefficient result context bytes (coef_res_ctx form): 0x40 for an
    all-zero neighbour, else min(cumulative level, 63) | dc-sign marker."""
    cul = rng.integers(1, 64, size=n)
    dcb = rng.choice(np.array([0x00, 0x40, 0x80]), size=n)
    zero = rng.random(n) < 0.3
    return np.where(zero, 0x40, cul | dcb).astype(np.uint8)


def split16_jobs(fw, fh, modes, deltas=(0,), seed=0, n=16):
    """(n x n block, mode, delta) jobs of the split trials (n = 16:
    split16_luma_try / split16_depth2_try, 8: split4tx_try), mode-major (every
    block for one (mode, delta), then the next), with deterministic neighbour
    flags and random coefficient contexts per block."""
    rng = np.random.default_rng(seed)
    bys, bxs = np.meshgrid(np.arange(0, fh - n + 1, n), np.arange(0, fw - n + 1, n), indexing="ij")
    px, py = bxs.ravel(), bys.ravel()
    nb = len(px)
    flags = np.array([block_flags(int(x), int(y), fw, fh, n) for x, y in zip(px, py)], np.uint8)
    flags |= np.where(rng.random(nb) < 0.5, abi.CAND_FILTER_TYPE, 0).astype(np.uint8)
    a_coef = coef_ctx_bytes(rng, nb * 4).reshape(nb, 4)
    l_coef = coef_ctx_bytes(rng, nb * 4).reshape(nb, 4)
    rows = []
    for m in modes:
        for d in (deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)):
            for b in range(nb):
                rows.append((px[b], py[b], m, d, flags[b], 0, a_coef[b], l_coef[b]))
    return np.array(rows, abi.SPLIT16_JOB_DTYPE)


def planes420(rgb, seed):
    """Source and reconstruction planes of a 4:2:0 frame from an RGB image:
    luma by rgb_to_luma, U and V the blue and red channels averaged over each
    2x2 cell's diagonal pair (textured chroma with real edges, so every kind
    of chroma mode can win); each reconstruction is the plane plus a seeded
    +-3 coding error.  Returns ([Y, U, V], [Y', U', V'])."""
    c = np.asarray(rgb).astype(np.int32)
    y = rgb_to_luma(np.asarray(rgb, np.uint8))
    u = ((c[0::2, 0::2, 2] + c[1::2, 1::2, 2] + 1) >> 1).astype(np.uint16)
    v = ((c[0::2, 0::2, 0] + c[1::2, 1::2, 0] + 1) >> 1).astype(np.uint16)
    src = [y, u, v]
    rec = [synthetic_recon(p, seed + 7 + k) for k, p in enumerate(src)]
    return src, rec


def planes444(rgb, seed):
    """Source and reconstruction planes of a 4:4:4 frame from an RGB image:
    luma by rgb_to_luma, U the blue and V the red channel, each reconstruction
    the plane plus a seeded +-3 coding error."""
    c = np.asarray(rgb)
    src = [rgb_to_luma(np.asarray(rgb, np.uint8)), c[:, :, 2].astype(np.uint16), c[:, :, 0].astype(np.uint16)]
    rec = [synthetic_recon(p, seed + 7 + k) for k, p in enumerate(src)]
    return src, rec


def uv16_444_jobs(w, h, seed, every=1, leaf=16):
    """16x16-leaf jobs of the 4:4:4 chroma search (mt_uv16_444_job), as
    uv16_jobs with four coefficient-context bytes per plane and side; leaf=32:
    the 32x32 leaves of the 4:2:0 search pick_uv32_420 (same layout)."""
    rng = np.random.default_rng(seed)
    rows = []
    for py in range(0, h - leaf + 1, leaf):
        for px in range(0, w - leaf + 1, leaf):
            if rng.random() > 1.0 / every:
                continue
            fl = block_flags(px, py, w, h, leaf) | (abi.CAND_FILTER_TYPE if rng.random() < 0.5 else 0)
            ctx = coef_ctx_bytes(rng, 16)
            rows.append((px, py, int(rng.integers(0, 13)), fl, ctx[:8].reshape(2, 4), ctx[8:].reshape(2, 4), (0, 0)))
    return np.array(rows, abi.UV16_444_JOB_DTYPE)


def uv32_444_jobs(w, h, seed):
    """32x32-leaf jobs of the 4:4:4 chroma search (mt_uv32_444_job): eight
    coefficient-context bytes per plane and side."""
    rng = np.random.default_rng(seed)
    rows = []
    for py in range(0, h - 31, 32):
        for px in range(0, w - 31, 32):
            fl = block_flags(px, py, w, h, 32) | (abi.CAND_FILTER_TYPE if rng.random() < 0.5 else 0)
            ctx = coef_ctx_bytes(rng, 32)
            rows.append((px, py, int(rng.integers(0, 13)), fl, ctx[:16].reshape(2, 8), ctx[16:].reshape(2, 8), (0, 0)))
    return np.array(rows, abi.UV32_444_JOB_DTYPE)


def uv16_jobs(w, h, seed, every=1):
    """16x16-leaf jobs of the 4:2:0 chroma search (mt_uv16_job): every
    16x16 leaf of a w x h frame (or about one in `every`), a random luma
    winner mode, deterministic neighbour flags with a random chroma filter
    type, coefficient-context bytes shaped like coef_res_ctx's."""
    rng = np.random.default_rng(seed)
    rows = []
    for py in range(0, h - 15, 16):
        for px in range(0, w - 15, 16):
            if rng.random() > 1.0 / every:
                continue
            fl = block_flags(px, py, w, h, 16) | (abi.CAND_FILTER_TYPE if rng.random() < 0.5 else 0)
            ctx = coef_ctx_bytes(rng, 8)
            rows.append((px, py, int(rng.integers(0, 13)), fl, ctx[:4].reshape(2, 2), ctx[4:].reshape(2, 2), (0, 0)))
    return np.array(rows, abi.UV16_JOB_DTYPE)


def leaf64_jobs(fw, fh, modes, deltas=(0,), seed=0, grid=False):
    """(64x64 block, mode, delta) jobs of the 64x64 leaf's legs, mode-major:
    the four-TX_32X32 leg (mt_quad32_job: random per-quadrant dc_sign contexts)
    or, grid=True, the sixteen-TX_16X16 leg (mt_grid16_job: above / left
    coefficient-context bytes shaped like coef_res_ctx's, tx_depth bits)."""
    rng = np.random.default_rng(seed)
    bys, bxs = np.meshgrid(np.arange(0, fh - 63, 64), np.arange(0, fw - 63, 64), indexing="ij")
    px, py = bxs.ravel(), bys.ravel()
    nb = len(px)
    flags = np.array([block_flags(int(x), int(y), fw, fh, 64) for x, y in zip(px, py)], np.uint8)
    flags |= np.where(rng.random(nb) < 0.5, abi.CAND_FILTER_TYPE, 0).astype(np.uint8)

    def ctx_bytes():
        b = rng.integers(0, 64, size=(nb, 16)) | rng.choice([0x00, 0x40, 0x80], size=(nb, 16))
        return np.where(rng.random((nb, 16)) < 0.3, 0x40, b).astype(np.uint8)

    a, l = ctx_bytes(), ctx_bytes()
    dcs = rng.integers(0, 3, size=(nb, 4)).astype(np.uint8)
    rows = []
    for m in modes:
        for d in (deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)):
            mb = (rng.random(nb) * 6 + 1).astype(np.float32)
            db = (rng.random(nb) * 3 + 0.5).astype(np.float32)
            xb = (rng.random(nb) * 4 - 1).astype(np.float32)
            for b in range(nb):
                if grid:
                    rows.append((px[b], py[b], m, d, flags[b], 0, a[b], l[b], mb[b], db[b], xb[b]))
                else:
                    rows.append((px[b], py[b], m, d, flags[b], 0, dcs[b], mb[b], db[b]))
    return np.array(rows, abi.GRID16_JOB_DTYPE if grid else abi.QUAD32_JOB_DTYPE)


def leaf8_jobs(fw, fh, modes, deltas=(0,), seed=0, n=8):
    """(n x n block, mode, delta) jobs of the leaf luma searches (n = 8 or 16),
    mode-major, with deterministic neighbour flags, random dc_sign contexts and
    syntax bits."""
    rng = np.random.default_rng(seed)
    bys, bxs = np.meshgrid(np.arange(0, fh - n + 1, n), np.arange(0, fw - n + 1, n), indexing="ij")
    px, py = bxs.ravel(), bys.ravel()
    nb = len(px)
    flags = np.array([block_flags(int(x), int(y), fw, fh, n) for x, y in zip(px, py)], np.uint8)
    flags |= np.where(rng.random(nb) < 0.5, abi.CAND_FILTER_TYPE, 0).astype(np.uint8)
    dcs = rng.integers(0, 3, size=nb)
    rows = []
    for m in modes:
        for d in (deltas if abi.V_PRED <= m <= abi.D67_PRED else (0,)):
            syn = (rng.random(nb) * 6 + 1).astype(np.float32)
            for b in range(nb):
                rows.append((px[b], py[b], m, d, flags[b], dcs[b], syn[b]))
    return np.array(rows, abi.LEAF8_JOB_DTYPE)
