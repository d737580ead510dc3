"""The default decision snapshot ``Cdfs::new(qctx)`` (src/coder/cdfs.rs:401-629)
assembled in Python from the arrays of tests/golden/cdfs_default.json, which
gen_default_cdfs.py parses out of the reference's sources.  The tests compare
this assembly with the library's ``mt_coef_cdfs_default`` and use the
library's slices as the CDF input of every parity case at the real configs."""
import json
import os

import numpy as np

from maroontree_b200 import abi

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cdfs_default.json")
_G = None


def golden():
    global _G
    if _G is None:
        _G = json.load(open(GOLDEN))
    return _G


def icdf(vals, width):
    """src/tables.rs:31-35 icdf: 32768 - v per entry, then the terminal 0."""
    out = np.zeros(width, np.uint16)
    out[:len(vals)] = [32768 - v for v in vals]
    return out


def slice_from_golden(qctx, w, h, plane):
    """One (class, plane) slice following Cdfs::new's field sources: class by
    the AV1 txSzCtx of w x h, eob_pt CDF by coefficient count (capped at 1024),
    1-D eob_pt for luma 16 / 64 / 128, tx-type CDFs for luma without a
    32-point side (INTRA1 at square sizes 4 / 8, INTRA2 at 16)."""
    g = golden()
    lg = {4: 0, 8: 1, 16: 2, 32: 3, 64: 4}
    sqr, up = min(lg[w], lg[h]), max(lg[w], lg[h])
    cls = (sqr + up + 1) >> 1
    n = (4, 8, 16, 32, 64)[cls]
    p = "CHROMA" if plane else "LUMA"
    c = abi.CoefCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    arr("txb_skip")[...] = np.stack([icdf([v], 2) for v in g[f"SKIP_TX{n}"][qctx]])
    bt = arr("base_tok")
    for k, row in enumerate(g[f"BASE_TOK_TX{n}_{p}_Q"][qctx]):
        bt[k] = icdf(row, 4)
    br = arr("br_tok")
    for k, row in enumerate(g[f"BR_TOK_TX{min(n, 32)}_{p}_Q"][qctx]):
        br[k] = icdf(row, 4)
    arr("eob_base")[...] = np.stack([icdf(r, 3) for r in g[f"EOB_BASE_TX{n}_{p}_Q"][qctx]])
    arr("eob_hi")[...] = np.stack([icdf([v], 2) for v in g[f"EOB_HI_TX{n}_{p}"][qctx]])
    arr("dc_sign")[...] = np.stack([icdf([v], 2) for v in g["DC_SIGN_Q"][qctx][plane]])
    area = min(w * h, 1024)
    arr("eob_bin")[...] = icdf(g[f"EOB_BIN_{area}_{p}"][qctx], 11)
    if plane == 0 and area in (16, 64, 128):
        arr("eob_bin_1d")[...] = icdf(g[f"EOB_BIN_{area}_LUMA_1D"][qctx], 11)
    if plane == 0 and up <= 2 and sqr <= 2:
        tab = g[("TXTP_INTRA1_TX4", "TXTP_INTRA1_TX8", "TXTP_INTRA2_TX16")[sqr]]
        tx = arr("txtp")
        for m, row in enumerate(tab):
            tx[m] = icdf(row, 16)
    return c


def default_cdfs(mt, qidx, n, plane=0, h=None):
    """The library's default slice for base qindex `qidx` and an n x h transform."""
    return mt.coef_cdfs_default(mt.qcat(qidx), n, n if h is None else h, plane)
