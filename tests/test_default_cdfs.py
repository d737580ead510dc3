"""The default decision snapshot of the library (mt_coef_cdfs_default, the
coefficient slices of Cdfs::new(qctx), src/coder/cdfs.rs:401-629, and qcat,
src/coef_q.rs:31-41) against the reference's own arrays parsed from its
sources (tests/golden/cdfs_default.json, assembled by the oracle's
default_cdfs), and against the qctx-0 luma slices
the leaf-trial parity tests were first pinned with.  No device call."""
import json
import os

import numpy as np
import pytest


SIZES = [(w, h) for w in (4, 8, 16, 32, 64) for h in (4, 8, 16, 32, 64) if max(w, h) <= 4 * min(w, h)]


@pytest.mark.parametrize("qctx", range(4))
@pytest.mark.parametrize("plane", (0, 1))
def test_default_slices_match_reference_arrays(mt_lib, oracle_lib, qctx, plane):
    for w, h in SIZES:
        cls = ({4: 0, 8: 1, 16: 2, 32: 3, 64: 4}[min(w, h)] + {4: 0, 8: 1, 16: 2, 32: 3, 64: 4}[max(w, h)] + 1) >> 1
        if plane == 1 and cls == 4:
            from maroontree_b200 import MtError

            with pytest.raises(MtError):
                mt_lib.coef_cdfs_default(qctx, w, h, plane)
            continue
        got = mt_lib.coef_cdfs_default(qctx, w, h, plane)
        want = oracle_lib.default_cdfs(qctx, w, h, plane)
        assert bytes(got) == bytes(want), (qctx, w, h, plane)


def test_qcat_matches_reference_law(mt_lib, oracle_lib):
    want = [oracle_lib.qcat(q) for q in range(256)]
    assert [mt_lib.qcat(q) for q in range(256)] == want
    # the configs' qindices: q40 -> 116, q60 -> 70, q80 -> 35
    assert (mt_lib.qcat(116), mt_lib.qcat(70), mt_lib.qcat(35)) == (2, 2, 1)


@pytest.mark.parametrize("n,name", [(8, "cdfs_luma_tx8_qctx0.json"), (4, "cdfs_luma_tx4_qctx0.json")])
def test_default_slice_matches_first_fixtures(mt_lib, n, name):
    from test_split16 import luma_tx8_cdfs
    from test_split16_depth2 import luma_tx4_cdfs

    want = luma_tx8_cdfs() if n == 8 else luma_tx4_cdfs()
    assert bytes(mt_lib.coef_cdfs_default(0, n, n, 0)) == bytes(want)


def test_rejects_bad_shapes(mt_lib):
    from maroontree_b200 import MtError

    for args in [(4, 8, 8, 0), (0, 8, 64, 0), (0, 12, 12, 0), (0, 8, 8, 2)]:
        with pytest.raises(MtError):
            mt_lib.coef_cdfs_default(*args)
