"""The oracle's whole-frame encode (oracle/oracle_avif.py: the library's 8x8
decision rule, frame filters, block syntax, range coder, headers and
container, all on the CPU without the product library), checked without a
GPU:

  * identity-matrix 4:4:4 files decode under dav1d (Pillow's libavif) to the
    oracle's own deblocked and CDEF-filtered planes, sample for sample, at
    sizes that are and are not multiples of 64;
  * 4:2:0 through the colour conversion decodes to the oracle's luma within
    the YUV -> RGB -> Y rounding;
  * the oracle's sequence header, frame header and container equal the
    library's host writers for the same parameters;
  * serial and threaded decisions give the same file."""
import io

import numpy as np
import pytest

from maroontree_b200 import synth


def _decode(avif):
    from PIL import Image

    im = Image.open(io.BytesIO(avif))
    im.load()
    return np.asarray(im.convert("RGB"))


IDENTITY = (1, 13, 0, 1, 0)


# 4160x64 is the smallest kind of frame in two tiles (65 superblock columns:
# over the 64-column maximum tile width)
@pytest.mark.parametrize("w,h,quality", [(128, 64, 60), (200, 136, 40), (72, 200, 80), (4160, 64, 60)])
def test_identity_444_oracle_encode_decodes_exactly(oracle_lib, w, h, quality):
    from oracle import oracle_avif as oa

    rgb = synth.generate_rgb(w, h, w + quality)
    avif, rec = oa.encode_yuv8(rgb[..., 1], rgb[..., 2], rgb[..., 0], quality, 2, IDENTITY, want_recon=True)
    dec = _decode(avif)
    assert dec.shape == (h, w, 3)
    assert np.array_equal(dec[..., 1], rec[0][:h, :w])
    assert np.array_equal(dec[..., 2], rec[1][:h, :w])
    assert np.array_equal(dec[..., 0], rec[2][:h, :w])


@pytest.mark.parametrize("w,h,quality", [(203, 117, 80), (128, 128, 40), (4163, 72, 80)])
def test_420_oracle_encode_decodes_to_its_luma(oracle_lib, w, h, quality):
    from oracle import oracle_avif as oa

    rgb = synth.generate_rgb(w, h, 7)
    avif, rec = oa.encode_rgb8(rgb, quality, 0, want_recon=True)
    dec = _decode(avif)
    diff = np.abs(synth.rgb_to_luma(dec).astype(np.int32) - rec[0][:h, :w].astype(np.int32))
    assert np.mean(diff > 6) < 0.01 and diff.mean() < 1.0


def test_threaded_decisions_equal_serial(oracle_lib):
    from oracle import oracle_avif as oa

    rgb = synth.generate_rgb(320, 192, 9)
    assert oa.encode_rgb8(rgb, 60, 0, threads=1) == oa.encode_rgb8(rgb, 60, 0, threads=4)


@pytest.mark.parametrize("w,h,sub", [(1920, 1080, 2), (512, 512, 0), (203, 117, 2)])
def test_oracle_headers_and_container_equal_the_library_writers(mt_lib, oracle_lib, w, h, sub):
    from maroontree_b200 import abi
    from maroontree_b200 import container as ct
    from oracle import oracle_avif as oa

    cicp = oa.SRGB_YCBCR
    sp = abi.SequenceHeaderParams()
    sp.width, sp.height, sp.profile, sp.bit_depth = w, h, 0 if sub else 1, 8
    sp.color_present, sp.primaries, sp.transfer, sp.matrix, sp.full_range = 1, *cicp[:4]
    sp.ss_x = sp.ss_y = 1 if sub else 0
    sp.enable_filter_intra = sp.enable_intra_edge_filter = 1
    assert oa.sequence_header(w, h, sp.profile, bool(sub), cicp) == ct.sequence_header(sp)
    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    for cdef in (None, (4, 2, [(3, 1, 2, 4), (0, 0, 1, 2), (7, 2, 0, 0), (15, 4, 15, 4)]), (3, 0, [(5, 2, 1, 1)])):
        fp = abi.FrameHeaderParams()
        fp.w8, fp.h8, fp.base_q_idx, fp.qm_y, fp.qm_u, fp.qm_v = pw, ph, 70, 6, 6, 6
        fp.updating_cdf, fp.lf_y, fp.lf_u, fp.lf_v, fp.lf_sharpness = 1, 8, 3, 3, 0
        fp.cdef_bits = -1 if cdef is None else cdef[1]
        fp.cdef_damping = 3 if cdef is None else cdef[0]
        if cdef is not None:
            for e, st in enumerate(cdef[2]):
                for k in range(4):
                    fp.cdef_strengths[e][k] = st[k]
        assert oa.frame_header(pw, ph, 70, (6, 6), (8, 3), 0, cdef) == ct.frame_header(fp)
    payload = bytes(range(200)) * 3
    ip = ct.srgb_item(w, h, "420" if sub else "444")
    ip.seq_profile = 0 if sub else 1
    ip.seq_level_idx = ct.level_for(w, h)
    assert oa.wrap_av1_image(payload, w, h, ip.seq_profile, bool(sub), cicp) == ct.wrap_av1_image(payload, ip)


@pytest.mark.parametrize("w,h", [(1920, 1080), (4096, 4096), (4160, 64), (4104, 2400), (8200, 64), (4096, 2368)])
def test_oracle_tiling_and_frame_obus_equal_the_library(mt_lib, oracle_lib, w, h):
    """The spec-minimum tiling, the frame header with its tile info and the
    frame OBUs (one OBU_FRAME, or OBU_FRAME_HEADER + OBU_TILE_GROUP) against
    the library's writers."""
    from maroontree_b200 import abi
    from maroontree_b200 import container as ct
    from oracle import oracle_avif as oa

    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    tcl, trl, _, tsw, tsh = oa.tiling(pw, ph)
    assert (tcl, trl) == mt_lib.tiling_spec_min(pw, ph)
    sbc, sbr = (pw + 63) // 64, (ph + 63) // 64
    assert tsw <= 64 and tsw * tsh <= 2304  # the AV1 tile limits
    ntiles = -(-sbc // tsw) * -(-sbr // tsh)
    fp = abi.FrameHeaderParams()
    fp.w8, fp.h8, fp.base_q_idx, fp.qm_y, fp.qm_u, fp.qm_v = pw, ph, 70, 6, 6, 6
    fp.updating_cdf, fp.lf_y, fp.lf_u, fp.lf_v, fp.lf_sharpness = 1, 8, 3, 3, 0
    fp.cdef_bits, fp.cdef_damping = 1, 4
    fp.tile_cols_log2, fp.tile_rows_log2 = tcl, trl
    cdef = (4, 1, [(3, 1, 2, 4), (0, 0, 1, 2)])
    for e, st in enumerate(cdef[2]):
        for k in range(4):
            fp.cdef_strengths[e][k] = st[k]
    fh = oa.frame_header(pw, ph, 70, (6, 6), (8, 3), 0, cdef)
    assert fh == ct.frame_header(fp, trailing=ntiles > 1)
    tiles = [bytes([(7 * t + k) & 0xFF for k in range(50 + 13 * t)]) for t in range(ntiles)]
    assert oa.frame_obus(fh, tiles) == ct.assemble_frame_obus(fp, tiles)
