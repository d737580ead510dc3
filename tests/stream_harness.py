"""A sequential 4:4:4 intra coder over 8x8 blocks, for conformance tests:
every block is predicted, transformed, quantised and reconstructed by the
candidate chain (the library's CUDA kernel or the oracle), its coefficients are
coded by the token emitter (library or oracle), and the library's packer,
headers and container turn the tokens into an AVIF file.  A real AV1 decoder
(dav1d through Pillow's libavif) must then reproduce the coder's own
reconstruction exactly.  The block syntax around the coefficients (partition,
skip, modes, palette and filter-intra flags, tx_depth) follows the AV1 syntax
and the reference's context rules (src/coder/superblock.rs:711-990,
src/coder/block8.rs:2620-2700, src/coder/lossy_state.rs:1408-1415,
:4021-4051, src/coeffs.rs:2917-2920).

The picture is coded with the identity matrix (RGB as G, B, R planes), full
range, so the decoder's RGB output is the reconstruction itself.  With
filters=True the frame also carries the shipped loop-filter levels and the
oracle's CDEF decision (strengths in the frame header, each superblock's
cdef_idx inserted at its read_cdef() point by the library's filter replay), and
the expected output is the oracle's deblocked and CDEF-filtered planes.
"""
import io

import numpy as np

from maroontree_b200 import abi, synth
from maroontree_b200 import container as ct
from maroontree_b200 import entropy as en

INTRA_MODE_CTX = [0, 1, 2, 3, 4, 4, 4, 4, 3, 0, 1, 2, 0]  # src/intrapred.rs:1088
SMOOTH = (9, 10, 11)
TYPES = (abi.TX_IDTX, abi.TX_DCT_DCT, abi.TX_V_DCT, abi.TX_H_DCT, abi.TX_ADST_ADST, abi.TX_ADST_DCT,
         abi.TX_DCT_ADST)


def res_ctx_of(cf_colmajor, cls=0):
    """The coefficient context byte a transform block leaves (src/coeffs.rs):
    min(sum of |levels| up to eob, 63) | dc-sign bits; 0x40 when all zero.
    The sum runs in the class's own order (the 2-D scan, or the 1-D classes'
    row / column order)."""
    cf = np.asarray(cf_colmajor)
    if not cf.any():
        return 0x40
    if cls == 0:
        scan = SCAN8
    elif cls == 1:
        scan = [((i & 7) << 3) | (i >> 3) for i in range(64)]
    else:
        scan = list(range(64))
    nz = [i for i in range(64) if cf[scan[i]] != 0]
    cul = int(sum(abs(int(cf[scan[i]])) for i in range(nz[-1] + 1)))
    dcb = 0x40 if cf[0] == 0 else (0 if cf[0] < 0 else 0x80)
    return min(cul, 63) | dcb


SCAN8 = [0, 8, 1, 2, 9, 16, 24, 17, 10, 3, 4, 11, 18, 25, 32, 40, 33, 26, 19, 12, 5, 6, 13, 20, 27, 34, 41, 48, 56,
         49, 42, 35, 28, 21, 14, 7, 15, 22, 29, 36, 43, 50, 57, 58, 51, 44, 37, 30, 23, 31, 38, 45, 52, 59, 60, 53, 46,
         39, 47, 54, 61, 62, 55, 63]


class Coder:
    def __init__(self, mt, po, rgb, qidx, qm_level, gpu, seed=0, filters=False, pick="random", qm_uv=None):
        self.mt, self.po, self.gpu, self.filters, self.pick = mt, po, gpu, filters, pick
        self.qm_uv = qm_level if qm_uv is None else qm_uv
        self.h, self.w = rgb.shape[:2]
        assert self.w % 64 == 0 and self.h % 64 == 0
        # identity matrix: Y = G, U = B, V = R
        self.src = [rgb[..., 1].astype(np.uint16), rgb[..., 2].astype(np.uint16), rgb[..., 0].astype(np.uint16)]
        self.rec = [np.zeros((self.h, self.w), np.uint16) for _ in range(3)]
        self.qidx, self.qm_level = qidx, qm_level
        self.q = [mt.quant_new(qidx, 8, qm_level)] + [mt.quant_new_chroma(qidx, 0, 0, 8, self.qm_uv)] * 2
        self.qm = mt.qm_row(qm_level, 0, 8) if qm_level < 15 else None
        self.qmc = mt.qm_row(self.qm_uv, 1, 8) if (qm_level < 15 or self.qm_uv < 15) else None
        self.lam = mt.rd_lambdas(qidx, self.q[0].dc_q, 0)
        self.costs = mt.coef_costs(mt.coef_cdfs_default(mt.qcat(qidx), 8, 8, 0))
        self.cdfs = mt.coef_cdfs_default(mt.qcat(qidx), 8, 8, 0)
        self.rng = np.random.default_rng(seed)
        self.L = en.cdf_layout()
        n4c, n4r, n8c, n8r = self.w // 4, self.h // 4, self.w // 8, self.h // 8
        self.a_part, self.l_part = np.zeros(n8c, np.uint8), np.zeros(n8r, np.uint8)
        self.a_skip, self.l_skip = np.zeros(n4c, np.uint8), np.zeros(n4r, np.uint8)
        self.a_mode, self.l_mode = np.zeros(n4c, np.uint8), np.zeros(n4r, np.uint8)
        self.a_tx, self.l_tx = np.full(n4c, -1, np.int8), np.full(n4r, -1, np.int8)
        self.a_coef = [np.full(n4c, 0x40, np.uint8) for _ in range(3)]
        self.l_coef = [np.full(n4r, 0x40, np.uint8) for _ in range(3)]
        self.sbs = []          # per SB: list of token lists / ('coef', k) placeholders
        self.coef_blocks = []  # (levels, COEF_BLOCK record) in coding order

    def tok(self, slot, s):
        return (int(slot) << 8) | int(s)

    def part_ctx(self, bl, x8, y8):
        sh = 4 - bl
        return ((int(self.a_part[x8]) >> sh) & 1) + (((int(self.l_part[y8]) >> sh) & 1) << 1)

    def chain(self, plane, px, py, mode, delta, tx, flags):
        prm = self.mt.chain_params(self.w, self.h, tx_size=8, mode_lambda=20.0, satd_bridge=0.7)
        cand = np.zeros(1, abi.CANDIDATE_DTYPE)
        cand["px"], cand["py"], cand["mode"], cand["angle_delta"] = px, py, mode, delta
        cand["tx_type"], cand["flags"] = tx, flags
        q, qm = self.q[plane], (self.qm if plane == 0 else self.qmc)
        if self.gpu:
            _, lv, ro = self.mt.candidate_chain(self.src[plane], self.rec[plane], prm, q, qm, self.costs, cand,
                                                True, True)
        else:
            _, lv, ro = self.po.candidate_chain(self.src[plane], self.rec[plane], prm, q, qm, self.cdfs, cand,
                                                True, True)
        self.rec[plane][py:py + 8, px:px + 8] = ro[0].reshape(8, 8)
        return lv[0]

    def best(self, px, py, flags):
        lam = self.lam
        prm = self.mt.chain_params(self.w, self.h, tx_size=8, trellis_lambda0=lam.trellis_lambda0,
                                   mode_lambda=lam.mode_lambda, satd_scale=lam.satd_scale, satd_bridge=lam.satd_bridge)
        cands = np.zeros(13 * 7, abi.CANDIDATE_DTYPE)
        cands["px"], cands["py"], cands["flags"] = px, py, flags
        cands["mode"] = np.repeat(np.arange(13), 7)
        cands["tx_type"] = np.tile(np.array(TYPES), 13)
        res, _, _ = self.po.candidate_chain(self.src[0], self.rec[0], prm, self.q[0], self.qm, self.cdfs, cands)
        k = int(np.argmin(res["cost"]))
        return int(cands["mode"][k]), 0, int(cands["tx_type"][k])

    def block8(self, out, x8, y8, thr, lhb):
        px, py = x8 * 8, y8 * 8
        bx4, by4 = px // 4, py // 4
        have_tr = thr and y8 > 0 and px + 8 < self.w
        have_bl = lhb and x8 > 0 and py + 8 < self.h
        mode = int(self.rng.integers(0, 13))
        delta = int(self.rng.integers(-3, 4)) if 1 <= mode <= 8 else 0
        tx = int(TYPES[int(self.rng.integers(0, 7))])
        ft = (py > 0 and self.a_mode[bx4] in SMOOTH) or (px > 0 and self.l_mode[by4] in SMOOTH)
        flags = (abi.CAND_HAVE_TR if have_tr else 0) | (abi.CAND_HAVE_BL if have_bl else 0)
        if self.pick == "best":  # the lowest-cost (mode, type) of the chain at delta 0
            mode, delta, tx = self.best(px, py, flags | (abi.CAND_FILTER_TYPE if ft else 0))
        L = self.L
        out.append(self.tok(L.skip + int(self.a_skip[bx4]) + int(self.l_skip[by4]), 0))  # skip = 0
        self.a_skip[bx4:bx4 + 2] = 0
        self.l_skip[by4:by4 + 2] = 0
        yctx = INTRA_MODE_CTX[self.a_mode[bx4]] * 5 + INTRA_MODE_CTX[self.l_mode[by4]]
        out.append(self.tok(L.kf_y + yctx, mode))
        if 1 <= mode <= 8:
            out.append(self.tok(L.angle_delta + mode - 1, delta + 3))
        out.append(self.tok(L.uv_mode + 13 + mode, 0))  # UV_DC_PRED, CfL allowed at 8x8
        if mode == 0:
            out.append(self.tok(L.palette_y_mode + 0, 0))  # has_palette_y, bsize ctx 0, ctx 0
        out.append(self.tok(L.palette_uv_mode + 0, 0))  # has_palette_uv (UV is DC)
        if mode == 0:
            out.append(self.tok(L.filter_intra + 3, 0))  # use_filter_intra, BLOCK_8X8
        ctx = int(self.l_tx[by4] >= 1) + int(self.a_tx[bx4] >= 1)
        out.append(self.tok(L.txsz + 0 * 3 + ctx, 0))  # tx_depth 0: TX_8X8
        self.a_tx[bx4:bx4 + 2] = 1
        self.l_tx[by4:by4 + 2] = 1
        for plane in range(3):
            lv = self.chain(plane, px, py, mode if plane == 0 else 0, delta if plane == 0 else 0,
                            tx if plane == 0 else abi.TX_DCT_DCT,
                            flags | (abi.CAND_FILTER_TYPE if (ft and plane == 0) else 0))
            a, l = self.a_coef[plane], self.l_coef[plane]
            s = sum(int(v) >> 6 for v in a[bx4:bx4 + 2]) + sum(int(v) >> 6 for v in l[by4:by4 + 2]) - 4
            dcs = int(s != 0) + int(s > 0)
            skip_ctx = 0 if plane == 0 else 7 + int((a[bx4:bx4 + 2] != 0x40).any()) + int((l[by4:by4 + 2] != 0x40).any())
            rec = np.zeros(1, abi.COEF_BLOCK_DTYPE)
            cls = 0 if plane or tx not in (abi.TX_V_DCT, abi.TX_H_DCT) else (1 if tx == abi.TX_V_DCT else 2)
            rec[0] = (0, 3, int(plane > 0), skip_ctx, dcs, mode, tx, int(plane == 0), cls)
            out.append(("coef", len(self.coef_blocks)))
            self.coef_blocks.append((lv.astype(np.int32), rec))
            r = res_ctx_of(lv, cls)
            a[bx4:bx4 + 2] = r
            l[by4:by4 + 2] = r
        self.a_mode[bx4:bx4 + 2] = mode
        self.l_mode[by4:by4 + 2] = mode

    def node(self, out, bl, x8, y8, sz8, thr, lhb):
        if sz8 > 1:
            out.append(self.tok(self.L.part_split + (bl - 1) * 4 + self.part_ctx(bl, x8, y8), 3))
            h = sz8 // 2
            for cx, cy, t, l in ((x8, y8, True, True), (x8 + h, y8, thr, False), (x8, y8 + h, True, lhb),
                                 (x8 + h, y8 + h, False, False)):
                self.node(out, bl + 1, cx, cy, h, t, l)
        else:
            out.append(self.tok(self.L.part_bl8 + self.part_ctx(4, x8, y8), 0))  # PARTITION_NONE
            self.block8(out, x8, y8, thr, lhb)
            self.a_part[x8] = 0x1E
            self.l_part[y8] = 0x1E

    def encode(self):
        for sy in range(0, self.h, 64):
            for sx in range(0, self.w, 64):
                out = []
                self.node(out, 1, sx // 8, sy // 8, 8, True, False)
                self.sbs.append(out)
        levels = np.concatenate([lv for lv, _ in self.coef_blocks])
        blocks = np.concatenate([r for _, r in self.coef_blocks])
        blocks["cf_offset"] = np.arange(len(blocks)) * 64
        if self.gpu:
            toks, offs, _ = en.emit_coeffs(levels, blocks)
        else:
            toks, offs, _ = self.po.emit_coeffs(levels, blocks)
        streams = []
        for out in self.sbs:
            s = []
            for t in out:
                if isinstance(t, tuple):
                    k = t[1]
                    s.extend(int(v) for v in toks[offs[k]:offs[k + 1]])
                else:
                    s.append(t)
            streams.append(np.array(s, np.uint32))
        fp = ct.FrameHeaderParams()
        fp.w8, fp.h8, fp.base_q_idx = self.w, self.h, self.qidx
        fp.qm_y, fp.qm_u, fp.qm_v = self.qm_level, self.qm_uv, self.qm_uv
        fp.updating_cdf = 1
        fp.cdef_bits, fp.cdef_damping = -1, 3
        self.out = [p.copy() for p in self.rec]
        if not self.filters:
            tile = en.pack_tile(self.qidx, streams)
        else:
            self.out, fp = self.loop_filters(fp)
            # every superblock's first block is coded (skip = 0): its read_cdef()
            # point follows that block's skip flag, the fifth token of the SB
            points = [5] * len(streams) if fp.cdef_bits >= 0 else None
            _, trace = en.pack_tile(self.qidx, streams, points, want_trace=True)
            if fp.cdef_bits > 0:
                tile = en.replay_tile_with_filters(trace, (0, 0, self.w, self.h), self.cdef["grid"],
                                                   unit_cols=self.w // 64, cdef_bits=fp.cdef_bits)
            else:
                tile = en.replay_tile_with_filters(trace, (0, 0, self.w, self.h))
        sp = ct.SequenceHeaderParams()
        sp.width, sp.height, sp.profile, sp.bit_depth = self.w, self.h, 1, 8
        sp.color_present, sp.primaries, sp.transfer, sp.matrix, sp.full_range = 1, 1, 13, 0, 1
        sp.enable_filter_intra = sp.enable_intra_edge_filter = 1
        obu = ct.av1_stream(sp, fp, [tile])
        item = ct.srgb_item(self.w, self.h, "444")
        item.matrix = 0
        return ct.wrap_av1_image(obu, item)


def _loop_filters(self, fp):
    """Deblocking with the shipped levels (uniform 8x8 blocks and transforms)
    and the oracle's CDEF decision over the deblocked planes."""
    n4r, n4c = self.h // 4, self.w // 4
    two = np.full((n4r, n4c), 2, np.uint8)
    tv = np.zeros((n4r, n4c), np.uint8)
    tv[:, ::2] = 1
    tt = np.zeros((n4r, n4c), np.uint8)
    tt[::2, :] = 1
    ly, luv, sharp = self.mt.loop_filter_levels(self.qidx, 0, 0)
    fp.lf_y, fp.lf_u, fp.lf_v, fp.lf_sharpness = ly, luv, luv, sharp
    planes = self.po.deblock_frame(self.rec, self.w, self.h, 0, 0, (two, two, tv, tt), (two, two), ly, luv, luv)
    prm = self.mt.cdef_params(self.w, self.h, 0, 0, self.qidx)
    skip8 = np.zeros((self.h // 8, self.w // 8), np.uint8)
    out, dec, _ = self.po.cdef_frame(planes, self.src, skip8, prm)
    self.cdef = dec
    if dec["bits"] >= 0:
        fp.cdef_bits, fp.cdef_damping = dec["bits"], dec["damping"]
        for e, st in enumerate(dec["strengths"]):
            for k in range(4):
                fp.cdef_strengths[e][k] = st[k]
    return out, fp


Coder.loop_filters = _loop_filters


def decode_rgb(avif):
    from PIL import Image

    im = Image.open(io.BytesIO(avif))
    im.load()
    return np.asarray(im.convert("RGB"))


def encode_and_decode(mt, po, w, h, seed, qidx, qm_level, gpu, filters=False, pick="random", sigma=4.0):
    rgb = synth.generate_rgb(w, h, seed, sigma=sigma)
    c = Coder(mt, po, rgb, qidx, qm_level, gpu, seed, filters, pick)
    avif = c.encode()
    return c, decode_rgb(avif), avif
