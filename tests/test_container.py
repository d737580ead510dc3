"""Headers and container: the reference's own known answers (leb128,
src/bitwriter.rs:105-128; OBU framing and the temporal delimiter,
src/obu.rs:832-846; av1C header bytes, ftyp brand, av01 item, av1C box,
colr boxes and the iloc offset into mdat, src/isobmff.rs:1286-1618; the clli
payload, src/metadata.rs:190-193), the increment bits of the spec-minimum
tiling, and a whole AVIF built from the library's sequence header, frame
header, tile packer and container that a real AV1 decoder (dav1d through
Pillow's libavif) decodes.  No device call."""
import io

import numpy as np
import pytest

from maroontree_b200 import container as ct
from maroontree_b200 import entropy as en


def test_leb128_known_answers(mt_lib):
    assert ct.leb128(0) == b"\x00"
    assert ct.leb128(127) == b"\x7f"
    assert ct.leb128(128) == b"\x80\x01"
    assert ct.leb128(200) == b"\xc8\x01"
    assert ct.leb128(16384) == b"\x80\x80\x01"


def test_obu_wrapping_and_temporal_delimiter(mt_lib):
    obu = ct.wrap_obu(6, b"\xaa" * 200)
    assert (obu[0] >> 3) & 0xF == 6 and obu[1:3] == ct.leb128(200) and len(obu) == 203
    td = ct.wrap_obu(2, b"")
    assert len(td) == 2 and (td[0] >> 3) & 0xF == 2


def _boxes(b, start, end):
    out = []
    while start + 8 <= end:
        sz = int.from_bytes(b[start:start + 4], "big")
        out.append((b[start + 4:start + 8], start, start + sz))
        start += sz
    return out


def _item(**kw):
    p = ct.srgb_item(16, 16)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def test_ftyp_meta_av01_av1c(mt_lib):
    b = ct.wrap_av1_image(b"\xab\xcd", _item())
    assert b[4:8] == b"ftyp" and b[8:12] == b"avif"
    ftyp = int.from_bytes(b[:4], "big")
    assert b[ftyp + 4:ftyp + 8] == b"meta"
    assert b"av01" in b and b"av1C" in b and b"hvc1" not in b and b"hvcC" not in b


def test_av1c_header_bytes(mt_lib):
    p = _item(seq_profile=1, seq_level_idx=12, bit_depth=10, chroma_sub_x=0, chroma_sub_y=0)
    b = ct.wrap_av1_image(b"\x00", p)
    i = b.index(b"av1C") + 4
    assert b[i] == 0x81 and (b[i + 1] >> 5) & 7 == 1 and b[i + 1] & 0x1F == 12
    assert b[i + 2] & 0x40 and not b[i + 2] & 0x20


def test_iloc_offset_points_into_mdat(mt_lib):
    payload = b"hello av1"
    b = ct.wrap_av1_image(payload, _item())
    mdat = [s for c, s, e in _boxes(b, 0, len(b)) if c == b"mdat"][0] + 8
    iloc = b.index(b"iloc") - 4
    off = int.from_bytes(b[iloc + 16 + 6:iloc + 16 + 10], "big")
    assert off == mdat and b[off:off + len(payload)] == payload


@pytest.mark.parametrize("cicp,icc,n", [(True, False, 1), (False, True, 1), (True, True, 2), (False, False, 0)])
def test_colr_boxes(mt_lib, cicp, icc, n):
    b = ct.wrap_av1_image(b"\x00", _item(color_present=int(cicp)), icc=b"ICCDATA" if icc else None)
    assert b.count(b"colr") == n
    assert (b"nclx" in b) == cicp and (b"prof" in b) == icc


def test_exif_item_and_transforms(mt_lib):
    b = ct.wrap_av1_image(b"\x01\x02", _item(irot_steps=3, imir_axis=1, clli_present=1, max_content_light_level=1000,
                                              max_pic_average_light_level=400), exif=b"II*\x00")
    assert b"Exif" in b and b"cdsc" in b and b"irot" in b and b"imir" in b
    i = b.index(b"clli") + 4
    assert b[i:i + 4] == bytes([0x03, 0xE8, 0x01, 0x90])


def test_tiling_increments(mt_lib):
    # one tile per frame below 4096 wide and 2304 superblocks: no increments
    # beyond the terminating zero; 4096 x 4096 needs two tile rows
    assert ct.tiling_increments(1920, 1080, 0, 0) == ([False], [False])
    cols, rows = ct.tiling_increments(4096, 4096, 0, 1)
    assert cols == [False] and rows == [False]
    assert mt_lib.load().mt_tiling_spec_min is not None


def _seq(w, h):
    p = ct.SequenceHeaderParams()
    p.width, p.height, p.profile, p.bit_depth = w, h, 0, 8
    p.color_present, p.primaries, p.transfer, p.matrix, p.full_range = 1, 1, 13, 6, 1
    p.ss_x, p.ss_y = 1, 1
    p.enable_filter_intra = p.enable_intra_edge_filter = 1
    return p


def _frame(w, h, qidx=70):
    p = ct.FrameHeaderParams()
    p.w8, p.h8, p.base_q_idx = w, h, qidx
    p.qm_y = p.qm_u = p.qm_v = 15
    p.updating_cdf = 1
    p.lf_y, p.lf_u, p.lf_v, p.lf_sharpness = 8, 5, 5, 0
    p.cdef_bits, p.cdef_damping = -1, 3
    return p


def _all_skip_tile(oracle_lib, w, h, qidx):
    """Token streams of a frame of 64x64 DC_PRED blocks coded as skip: per
    superblock the partition NONE, skip, the y / uv modes, the palette flags and
    tx_depth 0, with the AV1 contexts of all-skip 64x64 neighbours."""
    sec = {}
    slots = oracle_lib.cdfs_new_slots(oracle_lib.qcat(qidx), sec)
    sbs = []
    for r in range(h // 64):
        for c in range(w // 64):
            nb = int(r > 0) + int(c > 0)
            tok = lambda slot, s: (slot << 8) | s
            sbs.append(np.array([
                tok(sec["part_split"] + 0 * 4 + 0, 0),       # PARTITION_NONE at 64x64, ctx 0
                tok(sec["skip"] + nb, 1),                      # skip, ctx = above + left skip
                tok(sec["kf_y"] + 0, 0),                       # DC_PRED, mode ctx (0, 0)
                tok(sec["uv_mode"] + 0, 0),                    # UV DC_PRED, no CfL at 64x64
                tok(sec["palette_y_mode"] + 6 * 3 + 0, 0),     # has_palette_y, bsize ctx 6
                tok(sec["palette_uv_mode"] + 0, 0),            # has_palette_uv
                tok(sec["txsz"] + 3 * 3 + nb, 0),              # tx_depth 0, TX_64X64 category 3, ctx = nb
            ], np.uint32))
    return sbs


def test_decodable_avif(mt_lib, oracle_lib):
    """A whole file through the library's packer, headers and container,
    decoded by dav1d (Pillow's libavif): a frame of skip blocks predicts the
    mid-grey DC everywhere."""
    from PIL import Image

    w, h, qidx = 128, 64, 70
    tile = en.pack_tile(qidx, _all_skip_tile(oracle_lib, w, h, qidx))
    obu = ct.av1_stream(_seq(w, h), _frame(w, h, qidx), [tile])
    avif = ct.wrap_av1_image(obu, ct.srgb_item(w, h))
    im = Image.open(io.BytesIO(avif))
    im.load()
    a = np.asarray(im.convert("RGB"))
    assert a.shape == (h, w, 3)
    assert (np.abs(a.astype(int) - 128) <= 2).all()
