"""Writes rate_default_qctx0.json: the default coefficient CDFs of the
reference's `Cdfs::new(0)` for the (TX_8X8 class, chroma) slice, the 4x8 / 8x4
scans and lo-context offsets, and the golden rates of the reference's test
`rectangular_orientations_use_their_own_contexts` (src/rate.rs:371-401); and
cdfs_luma_tx8_qctx0.json / cdfs_luma_tx4_qctx0.json: the (TX_8X8 / TX_4X4
class, luma) slices of the same snapshot with the 1-D eob_pt CDF and the intra
tx-type CDFs.

Run in a checkout that has the reference next to it:
    python tests/golden/gen_rate_golden.py /path/to/maroontree
The arrays and the test's inputs and expected values are parsed verbatim from
the reference's Rust sources (AV1 default CDF data, scan/context tables, the
test body); nothing is computed.
"""
import json
import os
import re
import sys


def rust_array(path, name):
    src = open(path).read()
    m = re.search(r"static\s+" + re.escape(name) + r"\s*:\s*([^=]+)=\s*\[", src)
    if not m:
        raise KeyError(name)
    ty = m.group(1)
    dims = [int(d) for d in re.findall(r";\s*(\d+)\s*\]", ty)][::-1]
    i = m.end() - 1
    depth, j = 0, i
    while True:
        if src[j] == "[":
            depth += 1
        elif src[j] == "]":
            depth -= 1
            if depth == 0:
                break
        j += 1
    body = re.sub(r"//[^\n]*", "", src[i:j + 1])
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    n = 1
    for d in dims:
        n *= d
    assert len(vals) == n, (name, dims, len(vals))

    def shape(v, ds):
        if len(ds) == 1:
            return v
        step = len(v) // ds[0]
        return [shape(v[k * step:(k + 1) * step], ds[1:]) for k in range(ds[0])]

    return shape(vals, dims)


def golden_test(path):
    """Coefficients and expected rates of rectangular_orientations_use_their_own_contexts."""
    src = open(path).read()
    body = src[src.index("fn rectangular_orientations_use_their_own_contexts"):]
    body = body[:body.index("assert_ne!")]
    pairs = re.search(r"for &\(i, level\) in &\[(.*?)\]\s*\{", body, re.S).group(1)
    coeffs = [[int(a), int(b)] for a, b in re.findall(r"\((\d+)(?:usize)?,\s*(-?\d+)\)", pairs)]
    rates = [float(v.replace("_", "")) for v in re.findall(r"\(\w+ - ([\d_.]+)\)\.abs\(\) < ", body)]
    tol = float(re.search(r"\.abs\(\) < ([\d.e-]+)", body).group(1))
    skip_ctx = int(re.search(r"skip_ctx:\s*(\d+)", body).group(1))
    dcs_ctx = int(re.search(r"dcs_ctx:\s*(\d+)", body).group(1))
    return coeffs, rates, tol, skip_ctx, dcs_ctx


def main(ref):
    q = os.path.join(ref, "src", "coef_q.rs")
    t = os.path.join(ref, "src", "tables.rs")
    coeffs, rates, tol, skip_ctx, dcs_ctx = golden_test(os.path.join(ref, "src", "rate.rs"))
    out = {
        "source": "src/coef_q.rs, src/tables.rs (qctx 0, class 1 = TX_8X8, plane 1 = chroma); "
                  "golden rates src/rate.rs:371-401",
        "skip": rust_array(q, "SKIP_TX8")[0],
        "base_tok": rust_array(q, "BASE_TOK_TX8_CHROMA_Q")[0],
        "br_tok": rust_array(q, "BR_TOK_TX8_CHROMA_Q")[0],
        "eob_base": rust_array(q, "EOB_BASE_TX8_CHROMA_Q")[0],
        "eob_hi": rust_array(q, "EOB_HI_TX8_CHROMA")[0],
        "dc_sign": rust_array(q, "DC_SIGN_Q")[0][1],
        "eob_bin_32": rust_array(q, "EOB_BIN_32_CHROMA")[0],
        "scan_4x8": rust_array(t, "SCAN_4X8"),
        "scan_8x4": rust_array(t, "SCAN_8X4"),
        "lo_ctx_off_wlh": rust_array(t, "LO_CTX_OFF_WLH"),
        "lo_ctx_off_wgh": rust_array(t, "LO_CTX_OFF_WGH"),
        # The test's coefficients: (scan index, level), its contexts and rates.
        "coeffs": coeffs,
        "skip_ctx": skip_ctx,
        "dcs_ctx": dcs_ctx,
        "rate_4x8": rates[0],
        "rate_8x4": rates[1],
        "tolerance": tol,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rate_default_qctx0.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print(dst)
    # The luma TX_8X8 slice of the same snapshot (plane 0), with the 1-D eob_pt
    # CDF of V_DCT / H_DCT and the intra tx-type CDFs (set INTRA_1) per y mode.
    luma = {
        "source": "src/coef_q.rs, src/tables.rs (qctx 0, class 1 = TX_8X8, plane 0 = luma), "
                  "src/coder/cdfs.rs:591-610 Cdfs::new field sources",
        "skip": rust_array(q, "SKIP_TX8")[0],
        "base_tok": rust_array(q, "BASE_TOK_TX8_LUMA_Q")[0],
        "br_tok": rust_array(q, "BR_TOK_TX8_LUMA_Q")[0],
        "eob_base": rust_array(q, "EOB_BASE_TX8_LUMA_Q")[0],
        "eob_hi": rust_array(q, "EOB_HI_TX8_LUMA")[0],
        "dc_sign": rust_array(q, "DC_SIGN_Q")[0][0],
        "eob_bin_64": rust_array(q, "EOB_BIN_64_LUMA")[0],
        "eob_bin_64_1d": rust_array(q, "EOB_BIN_64_LUMA_1D")[0],
        "txtp": rust_array(t, "TXTP_INTRA1_TX8"),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cdfs_luma_tx8_qctx0.json")
    with open(dst, "w") as f:
        json.dump(luma, f, indent=1)
    print(dst)
    # The luma TX_4X4 slice (class 0, plane 0) with its 1-D eob_pt CDF and the
    # 4x4 intra tx-type CDFs.
    luma4 = {
        "source": "src/coef_q.rs, src/tables.rs (qctx 0, class 0 = TX_4X4, plane 0 = luma), "
                  "src/coder/cdfs.rs:593-609 Cdfs::new field sources",
        "skip": rust_array(q, "SKIP_TX4")[0],
        "base_tok": rust_array(q, "BASE_TOK_TX4_LUMA_Q")[0],
        "br_tok": rust_array(q, "BR_TOK_TX4_LUMA_Q")[0],
        "eob_base": rust_array(q, "EOB_BASE_TX4_LUMA_Q")[0],
        "eob_hi": rust_array(q, "EOB_HI_TX4_LUMA")[0],
        "dc_sign": rust_array(q, "DC_SIGN_Q")[0][0],
        "eob_bin": rust_array(q, "EOB_BIN_16_LUMA")[0],
        "eob_bin_1d": rust_array(q, "EOB_BIN_16_LUMA_1D")[0],
        "txtp": rust_array(t, "TXTP_INTRA1_TX4"),
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cdfs_luma_tx4_qctx0.json")
    with open(dst, "w") as f:
        json.dump(luma4, f, indent=1)
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: gen_rate_golden.py <reference-root>")
    main(sys.argv[1])
