"""The rate walk pinned to the reference's own golden values: the test
`rectangular_orientations_use_their_own_contexts` (src/rate.rs:371-401) prices
the same four coefficients in a 4x8 and an 8x4 chroma block against the default
CDFs of `Cdfs::new(0)`; the expected rates 38.532284 and 38.2208 exercise the
eob, eob-base, base-token, base-range ladder, DC-sign and bypass-sign terms and
both rectangular context tables.  The CDF data, scans and expected values are
in tests/golden/rate_default_qctx0.json, made by gen_rate_golden.py beside it
from the reference's sources."""
import json
import os

import numpy as np
import pytest

from maroontree_b200 import abi

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rate_default_qctx0.json")


def _icdf(vals, width):
    """src/tables.rs:31-35 icdf: 32768 - v per entry, then the terminal 0."""
    out = np.zeros(width, np.uint16)
    out[:len(vals)] = [32768 - v for v in vals]
    return out


def _cdfs(g):
    c = abi.CoefCdfs()
    arr = lambda name: np.ctypeslib.as_array(getattr(c, name))
    arr("txb_skip")[...] = np.stack([_icdf([v], 2) for v in g["skip"]])
    bt = arr("base_tok")
    for k, row in enumerate(g["base_tok"]):
        bt[k] = _icdf(row, 4)
    br = arr("br_tok")
    for k, row in enumerate(g["br_tok"]):
        br[k] = _icdf(row, 4)
    arr("eob_base")[...] = np.stack([_icdf(r, 3) for r in g["eob_base"]])
    arr("eob_hi")[...] = np.stack([_icdf([v], 2) for v in g["eob_hi"]])
    arr("dc_sign")[...] = np.stack([_icdf([v], 2) for v in g["dc_sign"]])
    arr("eob_bin")[...] = _icdf(g["eob_bin_32"], 11)
    return c


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _block(g, scan):
    cf = np.zeros(32, np.int32)
    for i, level in g["coeffs"]:
        cf[scan[i]] = level
    return cf


def test_rate_4x8_matches_reference_golden(oracle_lib, golden):
    scan = golden["scan_4x8"]
    got = oracle_lib.real_block_bits_wh(_block(golden, scan), scan, 4, 8, _cdfs(golden), golden["skip_ctx"],
                                        golden["dcs_ctx"])
    assert abs(got - golden["rate_4x8"]) < golden["tolerance"], got


def test_rate_8x4_matches_reference_golden(oracle_lib, golden):
    scan = golden["scan_8x4"]
    got = oracle_lib.real_block_bits_wh(_block(golden, scan), scan, 8, 4, _cdfs(golden), golden["skip_ctx"],
                                        golden["dcs_ctx"])
    assert abs(got - golden["rate_8x4"]) < golden["tolerance"], got


def test_rate_orientations_differ(oracle_lib, golden):
    a = oracle_lib.real_block_bits_wh(_block(golden, golden["scan_4x8"]), golden["scan_4x8"], 4, 8, _cdfs(golden),
                                      golden["skip_ctx"], golden["dcs_ctx"])
    b = oracle_lib.real_block_bits_wh(_block(golden, golden["scan_8x4"]), golden["scan_8x4"], 8, 4, _cdfs(golden),
                                      golden["skip_ctx"], golden["dcs_ctx"])
    assert a != b
