"""Generate ``av1_tables.h``: the normative AV1 data tables the intra RD path needs.

The tables are AV1 specification data (the dav1d runtime forms the reference
vendors), not algorithm: dequantiser lookups (``Dc_Qlookup``/``Ac_Qlookup``),
inverse quantisation-matrix weights, default coefficient scans and the
coefficient-base context offsets.  They must be identical to the reference's
for byte parity, so this script reads them out of the reference's Rust sources
once and writes a C header that is committed; nothing at run time reads the
reference.

Usage (from the repository root, with the reference checkout available; the
reference root is a required argument)::

    python maroontree_b200/csrc/gen_av1_tables.py <reference-root>

It also writes ``av1_cdfs.h``: the AV1 default coefficient CDFs of every
coefficient q context (the arrays ``Cdfs::new(qctx)`` reads, src/coder/cdfs.rs:401-629)
and the intra transform-type CDFs, in the AV1 cumulative form the reference
stores (the inverse form is 32768 - v, src/tables.rs:31-35).

Source locations (reference paths):
  src/coef_q.rs     DC_QLOOKUP_8, AC_QLOOKUP_8/10/12, SCAN_16X16, SCAN_32X32
  src/tables.rs     SCAN_8X8, SCAN_4X4, LO_CTX_OFF, LO_CTX_OFF_WLH, LO_CTX_OFF_WGH
  src/qm_tables.rs  AV1_IQM  ([15][2][3344] u8)
  src/dct.rs        ADST16_FWD_Q12 ([16][16] i16, the forward 16-point ADST in Q12)
  src/tables.rs     INTRA_FILTER_TAPS ([5][8][7] i8, the recursive filter-intra taps)
  src/coef_q.rs     SKIP_TX*, BASE_TOK_TX*_Q, BR_TOK_TX*_Q, EOB_BASE_TX*_Q, EOB_HI_TX*,
                    DC_SIGN_Q, EOB_BIN_*  (av1_cdfs.h)
  src/tables.rs     TXTP_INTRA1_TX4, TXTP_INTRA1_TX8, TXTP_INTRA2_TX16 (av1_cdfs.h)
"""
import os
import re
import sys

TABLES = [
    # (file, rust name, C name, C type)
    ("src/coef_q.rs", "DC_QLOOKUP_8", "MT_DC_QLOOKUP_8", "uint16_t"),
    ("src/coef_q.rs", "AC_QLOOKUP_8", "MT_AC_QLOOKUP_8", "uint16_t"),
    ("src/coef_q.rs", "AC_QLOOKUP_10", "MT_AC_QLOOKUP_10", "uint16_t"),
    ("src/coef_q.rs", "AC_QLOOKUP_12", "MT_AC_QLOOKUP_12", "uint16_t"),
    ("src/skip_tables.rs", "SCAN_4X4", "MT_SCAN_4X4", "uint16_t"),
    ("src/tables.rs", "SCAN_8X8", "MT_SCAN_8X8", "uint16_t"),
    ("src/coef_q.rs", "SCAN_16X16", "MT_SCAN_16X16", "uint16_t"),
    ("src/coef_q.rs", "SCAN_32X32", "MT_SCAN_32X32", "uint16_t"),
    ("src/tables.rs", "LO_CTX_OFF", "MT_LO_CTX_OFF", "uint8_t"),
    ("src/tables.rs", "LO_CTX_OFF_WLH", "MT_LO_CTX_OFF_WLH", "uint8_t"),
    ("src/tables.rs", "LO_CTX_OFF_WGH", "MT_LO_CTX_OFF_WGH", "uint8_t"),
    ("src/qm_tables.rs", "AV1_IQM", "MT_AV1_IQM", "uint8_t"),
    ("src/dct.rs", "ADST16_FWD_Q12", "MT_ADST16_FWD_Q12", "int16_t"),
    ("src/tables.rs", "INTRA_FILTER_TAPS", "MT_INTRA_FILTER_TAPS", "int8_t"),
]


def extract(path, name):
    text = open(path, encoding="utf-8").read()
    m = re.search(r"static\s+" + re.escape(name) + r"\s*:\s*([^=]+)=\s*\[", text)
    if not m:
        raise SystemExit(f"{name} not found in {path}")
    i = m.end() - 1
    depth = 0
    j = i
    while True:
        c = text[j]
        if c == "[":
            depth += 1
        elif c == "]":
            depth -= 1
            if depth == 0:
                break
        j += 1
    body = re.sub(r"//[^\n]*", "", text[i : j + 1])
    nums = [int(v) for v in re.findall(r"-?\d+", body)]
    dims = [int(d) for d in re.findall(r";\s*([A-Z_0-9]+|\d+)\s*\]", m.group(1)) if d.isdigit()]
    return nums, m.group(1).strip()


CDF_TABLES = (
    [("src/coef_q.rs", f"SKIP_TX{n}") for n in (4, 8, 16, 32, 64)]
    + [("src/coef_q.rs", f"{k}_TX{n}_{p}_Q") for k in ("BASE_TOK", "BR_TOK", "EOB_BASE")
       for n in (4, 8, 16, 32) for p in ("LUMA", "CHROMA")]
    + [("src/coef_q.rs", "BASE_TOK_TX64_LUMA_Q"), ("src/coef_q.rs", "EOB_BASE_TX64_LUMA_Q")]
    + [("src/coef_q.rs", f"EOB_HI_TX{n}_{p}") for n in (4, 8, 16, 32) for p in ("LUMA", "CHROMA")]
    + [("src/coef_q.rs", "EOB_HI_TX64_LUMA"), ("src/coef_q.rs", "DC_SIGN_Q")]
    + [("src/coef_q.rs", f"EOB_BIN_{a}_{p}") for a in (16, 32, 64, 128, 256, 512, 1024)
       for p in ("LUMA", "CHROMA")]
    + [("src/coef_q.rs", f"EOB_BIN_{a}_LUMA_1D") for a in (16, 64, 128)]
    + [("src/tables.rs", "TXTP_INTRA1_TX4"), ("src/tables.rs", "TXTP_INTRA1_TX8"),
       ("src/tables.rs", "TXTP_INTRA2_TX16")]
    # the mode / partition / tool CDFs of Cdfs::new (src/coder/cdfs.rs:506-627)
    + [("src/tables.rs", n) for n in ("SKIP_CDF", "FILTER_INTRA_MODE_CDF", "FILTER_INTRA_CDF", "KF_Y_MODE_CDF",
                                      "UV_MODE_NOCFL_CDF", "UV_MODE_CFL_CDF", "ANGLE_DELTA_CDF", "PART_SPLIT_CDF",
                                      "PART_BL8_CDF", "TXSZ_CAT0_CDF", "TXSZ_CAT1_CDF", "TXSZ_CAT2_CDF",
                                      "TXSZ_CAT3_CDF")]
    + [("src/intrapred.rs", "CFL_SIGN_CDF"), ("src/intrapred.rs", "CFL_ALPHA_CDF")]
)


def extract_fn_static(path, fn_name, static_name):
    """The values of `static static_name` (or `const`) declared inside fn_name."""
    text = open(path, encoding="utf-8").read()
    i = text.index("fn " + fn_name + "(")
    j = text.index("\n}\n", i)
    body = text[i:j]
    m = re.search(r"(?:static|const)\s+" + re.escape(static_name) + r"\s*:\s*([^=]+)=\s*\[", body)
    k = m.end() - 1
    depth, e = 0, k
    while True:
        if body[e] == "[":
            depth += 1
        elif body[e] == "]":
            depth -= 1
            if depth == 0:
                break
        e += 1
    vals = re.sub(r"//[^\n]*", "", body[k:e + 1])
    return [int(v) for v in re.findall(r"-?\d+", vals)], m.group(1).strip()


def extract_palette_y_color(path):
    """palette_y_color_raw's (size, ctx) => &[..] arms, sizes 2..8 x 5 contexts,
    concatenated in (size, ctx) order (size - 1 values each)."""
    text = open(path, encoding="utf-8").read()
    i = text.index("fn palette_y_color_raw(")
    j = text.index("\n}\n", i)
    arms = re.findall(r"\((\d+),\s*(\d+)\)\s*=>\s*&\[([^\]]*)\]", text[i:j])
    got = {(int(a), int(b)): [int(v) for v in re.findall(r"\d+", c)] for a, b, c in arms}
    out = []
    for n in range(2, 9):
        for ctx in range(5):
            assert len(got[(n, ctx)]) == n - 1
            out += got[(n, ctx)]
    return out


def extract_palette_uv_color(path):
    """palette_uv_color_raw's S2..S8 tables ([5][size - 1]) in size order."""
    out = []
    for n in range(2, 9):
        vals, _ = extract_fn_static(path, "palette_uv_color_raw", f"S{n}")
        assert len(vals) == 5 * (n - 1)
        out += vals
    return out


def write_cdfs(ref):
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "av1_cdfs.h")
    lines = [
        "/* Generated by gen_av1_tables.py: the AV1 default coefficient CDFs of every",
        " * coefficient q context and the intra transform-type CDFs, in the cumulative",
        " * form the reference stores (inverse form: 32768 - v).  Do not edit. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
    ]
    for rel, rname in CDF_TABLES:
        nums, decl = extract(os.path.join(ref, rel), rname)
        cname = "MT_CDF_" + rname
        lines.append(f"/* {rel} {rname}: {decl} ({len(nums)} values) */")
        lines.append(f"static const uint16_t {cname}[{len(nums)}] = {{")
        for k in range(0, len(nums), 24):
            lines.append("  " + ",".join(str(v) for v in nums[k : k + 24]) + ",")
        lines.append("};")
        lines.append("")
    pal = os.path.join(ref, "src/coder/palette.rs")
    extra = [
        ("MT_CDF_PALETTE_Y_MODE", extract_fn_static(pal, "palette_y_mode_cdfs", "RAW")[0],
         "src/coder/palette.rs palette_y_mode_cdfs RAW [7][3]"),
        ("MT_CDF_PALETTE_Y_SIZE", extract_fn_static(pal, "palette_y_size_cdfs", "RAW")[0],
         "src/coder/palette.rs palette_y_size_cdfs RAW [7][6]"),
        ("MT_CDF_PALETTE_UV_SIZE", extract_fn_static(pal, "palette_uv_size_cdfs", "RAW")[0],
         "src/coder/palette.rs palette_uv_size_cdfs RAW [7][6]"),
        ("MT_CDF_PALETTE_Y_COLOR", extract_palette_y_color(pal),
         "src/coder/palette.rs palette_y_color_raw, sizes 2..8 x 5 contexts, size-1 values each"),
        ("MT_CDF_PALETTE_UV_COLOR", extract_palette_uv_color(pal),
         "src/coder/palette.rs palette_uv_color_raw S2..S8, sizes 2..8 x 5 contexts, size-1 values each"),
    ]
    for cname, nums, what in extra:
        lines.append(f"/* {what} ({len(nums)} values) */")
        lines.append(f"static const uint16_t {cname}[{len(nums)}] = {{")
        for k in range(0, len(nums), 24):
            lines.append("  " + ",".join(str(v) for v in nums[k : k + 24]) + ",")
        lines.append("};")
        lines.append("")
    open(out, "w").write("\n".join(lines))
    print("wrote", out)


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: gen_av1_tables.py <reference-root>")
    ref = sys.argv[1]
    write_cdfs(ref)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "av1_tables.h")
    lines = [
        "/* Generated by gen_av1_tables.py: normative AV1 tables (dequantiser lookups,",
        " * inverse quantisation matrices, default scans, coefficient-base context",
        " * offsets).  Do not edit. */",
        "#pragma once",
        "#include <stdint.h>",
        "",
    ]
    for rel, rname, cname, ctype in TABLES:
        nums, decl = extract(os.path.join(ref, rel), rname)
        lines.append(f"/* {rel} {rname}: {decl} ({len(nums)} values) */")
        lines.append(f"#define {cname}_LEN {len(nums)}")
        lines.append(f"static const {ctype} {cname}[{len(nums)}] = {{")
        for k in range(0, len(nums), 24):
            lines.append("  " + ",".join(str(v) for v in nums[k : k + 24]) + ",")
        lines.append("};")
        if "QLOOKUP" in cname or cname in ("MT_SCAN_16X16", "MT_SCAN_32X32", "MT_ADST16_FWD_Q12",
                                           "MT_INTRA_FILTER_TAPS"):  # initialiser lists for device copies
            lines.append(f"#define {cname}_LIST " + ",".join(str(v) for v in nums))
        lines.append("")
    open(out, "w").write("\n".join(lines))
    print("wrote", out)


if __name__ == "__main__":
    main()
