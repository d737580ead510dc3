"""Writes cdfs_default.json: every array the coefficient part of the
reference's ``Cdfs::new(qctx)`` reads (src/coder/cdfs.rs:401-629), for all four
coefficient q contexts, plus the intra tx-type CDF tables, parsed verbatim from
the reference's Rust sources (src/coef_q.rs, src/tables.rs).  Nothing is
computed; the tests assemble the per-(class, plane) slices from these arrays
following Cdfs::new's field sources and compare them with the library's
``mt_coef_cdfs_default``.

Run in a checkout that has the reference next to it:
    python tests/golden/gen_default_cdfs.py /path/to/maroontree
"""
import json
import os
import sys

from gen_rate_golden import rust_array

NAMES_COEF_Q = (
    [f"SKIP_TX{n}" for n in (4, 8, 16, 32, 64)]
    + [f"{k}_TX{n}_{p}_Q" for k in ("BASE_TOK", "BR_TOK", "EOB_BASE") for n in (4, 8, 16, 32)
       for p in ("LUMA", "CHROMA")]
    + ["BASE_TOK_TX64_LUMA_Q", "EOB_BASE_TX64_LUMA_Q"]
    + [f"EOB_HI_TX{n}_{p}" for n in (4, 8, 16, 32) for p in ("LUMA", "CHROMA")]
    + ["EOB_HI_TX64_LUMA", "DC_SIGN_Q"]
    + [f"EOB_BIN_{a}_{p}" for a in (16, 32, 64, 128, 256, 512, 1024) for p in ("LUMA", "CHROMA")]
    + [f"EOB_BIN_{a}_LUMA_1D" for a in (16, 64, 128)]
)
NAMES_TABLES = ["TXTP_INTRA1_TX4", "TXTP_INTRA1_TX8", "TXTP_INTRA2_TX16", "SKIP_CDF", "FILTER_INTRA_MODE_CDF",
                "FILTER_INTRA_CDF", "KF_Y_MODE_CDF", "UV_MODE_NOCFL_CDF", "UV_MODE_CFL_CDF", "ANGLE_DELTA_CDF",
                "PART_SPLIT_CDF", "PART_BL8_CDF", "TXSZ_CAT0_CDF", "TXSZ_CAT1_CDF", "TXSZ_CAT2_CDF", "TXSZ_CAT3_CDF"]
NAMES_INTRAPRED = ["CFL_SIGN_CDF", "CFL_ALPHA_CDF"]


def palette_tables(path):
    """The palette CDFs of src/coder/palette.rs: the function-local RAW tables of
    palette_y_mode_cdfs / palette_y_size_cdfs / palette_uv_size_cdfs, the
    (size, ctx) arms of palette_y_color_raw and palette_uv_color_raw's S2..S8."""
    import re

    src = open(path).read()

    def fn_body(name):
        i = src.index("fn " + name + "(")
        return src[i:src.index("\n}\n", i)]

    def nums(text):
        return [int(v) for v in re.findall(r"\d+", re.sub(r"//[^\n]*", "", text))]

    def table(name, static):
        b = fn_body(name)
        i = b.index(static + ":")
        j = b.index("= [", i) + 2
        depth, k = 0, j
        while True:
            depth += {"[": 1, "]": -1}.get(b[k], 0)
            if depth == 0:
                break
            k += 1
        return nums(b[j:k + 1])

    yc = {}
    for a, c, body in re.findall(r"\((\d+),\s*(\d+)\)\s*=>\s*&\[([^\]]*)\]", fn_body("palette_y_color_raw")):
        yc[f"{a},{c}"] = nums(body)
    uvc = {str(n): table("palette_uv_color_raw", f"S{n}") for n in range(2, 9)}
    return {"PALETTE_Y_MODE": table("palette_y_mode_cdfs", "RAW"),
            "PALETTE_Y_SIZE": table("palette_y_size_cdfs", "RAW"),
            "PALETTE_UV_SIZE": table("palette_uv_size_cdfs", "RAW"),
            "PALETTE_Y_COLOR": yc, "PALETTE_UV_COLOR": uvc}


def main(ref):
    q = os.path.join(ref, "src", "coef_q.rs")
    t = os.path.join(ref, "src", "tables.rs")
    out = {"source": "src/coef_q.rs, src/tables.rs; assembled as src/coder/cdfs.rs:401-629 Cdfs::new"}
    for n in NAMES_COEF_Q:
        out[n] = rust_array(q, n)
    for n in NAMES_TABLES:
        out[n] = rust_array(t, n)
    for n in NAMES_INTRAPRED:
        out[n] = rust_array(os.path.join(ref, "src", "intrapred.rs"), n)
    out.update(palette_tables(os.path.join(ref, "src", "coder", "palette.rs")))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cdfs_default.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: gen_default_cdfs.py <reference-root>")
    main(sys.argv[1])
