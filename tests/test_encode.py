"""mt_encode_rgb8 / mt_encode_yuv8 on the device: a whole AVIF per call.

  * identity matrix 4:4:4 (the picture's G, B, R as the coded planes): dav1d's
    output through Pillow equals the encoder's reconstruction after deblocking
    and CDEF, sample for sample;
  * the same picture coded by the oracle-side coder of tests/stream_harness.py
    under the same decision rule (lowest RD cost of 13 modes x 7 types per 8x8
    block, UV DC) and the same frame laws gives the same bytes;
  * 4:2:0 through the colour conversion decodes to the encoder's own luma
    (within the YUV -> RGB -> Y rounding), with a real encode's PSNR at the
    benchmark sizes.
"""
import io

import numpy as np
import pytest

from maroontree_b200 import synth

pytestmark = pytest.mark.gpu


def _decode(avif):
    from PIL import Image

    im = Image.open(io.BytesIO(avif))
    im.load()
    return np.asarray(im.convert("RGB"))


def _identity_cfg(enc, quality):
    return enc.config(quality=quality, chroma=2, matrix=0)


@pytest.mark.parametrize("w,h,quality", [(256, 192, 60), (200, 136, 40), (128, 128, 80)])
def test_identity_444_decodes_to_the_encoders_reconstruction(mt_lib, cuda, w, h, quality):
    from maroontree_b200 import encoder as enc

    rgb = synth.generate_rgb(w, h, w + quality)
    avif, rec = enc.encode_yuv8(rgb[..., 1], rgb[..., 2], rgb[..., 0], _identity_cfg(enc, quality), want_recon=True)
    dec = _decode(avif)
    assert dec.shape == (h, w, 3)
    assert np.array_equal(dec[..., 1], rec[0][:h, :w])
    assert np.array_equal(dec[..., 2], rec[1][:h, :w])
    assert np.array_equal(dec[..., 0], rec[2][:h, :w])


@pytest.mark.parametrize("quality,seed", [(60, 11), (40, 12)])
def test_encoder_bytes_match_the_oracle_coder(mt_lib, oracle_lib, cuda, quality, seed):
    """The same decisions and syntax restated on the oracle side give the same file."""
    import stream_harness as sh
    from maroontree_b200 import encoder as enc

    w, h = 192, 128
    rgb = synth.generate_rgb(w, h, seed)
    qidx = mt_lib.quality_to_q(quality)
    qy, quv = mt_lib.qm_levels(qidx, 0)
    coder = sh.Coder(mt_lib, oracle_lib, rgb, qidx, qy, False, seed, filters=True, pick="best", qm_uv=quv)
    want = coder.encode()
    got = enc.encode_yuv8(rgb[..., 1], rgb[..., 2], rgb[..., 0], _identity_cfg(enc, quality))
    assert got == want


@pytest.mark.parametrize("w,h,quality,seed", [(1920, 1080, 60, 3), (512, 512, 60, 1), (203, 117, 80, 5),
                                               (200, 136, 40, 6)])
def test_420_rgb_encode_decodes(mt_lib, cuda, w, h, quality, seed):
    """4:2:0 through the colour conversion: the decoder's RGB, taken back to
    luma with the same Q13 weights, equals the encoder's filtered luma within
    the rounding of the YUV -> RGB -> Y round trip (8-bit RGB, chroma
    upsampling, clamping): no 8x8 block is off on average by more than 4 and
    under 1% of samples by more than 6; on the large pictures the PSNR
    against the source is that of a real encode."""
    from maroontree_b200 import encoder as enc

    rgb = synth.generate_rgb(w, h, seed, variant="1080p" if w == 1920 else "plain")
    avif, rec = enc.encode_rgb8(rgb, enc.config(quality=quality), want_recon=True)
    dec = _decode(avif)
    assert dec.shape == (h, w, 3)
    yd = synth.rgb_to_luma(dec).astype(np.int32)
    diff = np.abs(yd - rec[0][:h, :w].astype(np.int32))
    assert np.mean(diff > 6) < 0.01
    hb, wb = h // 8, w // 8
    assert diff[:hb * 8, :wb * 8].reshape(hb, 8, wb, 8).mean(axis=(1, 3)).max() <= 4.0
    assert len(avif) < w * h * 3 // 4
    if w >= 512:
        mse = np.mean((dec.astype(np.float64) - rgb.astype(np.float64)) ** 2)
        assert 10 * np.log10(255.0 ** 2 / mse) > 28.0


@pytest.mark.parametrize("name", ["C1", "C2q40", "C2q60", "C2q80", "C3"])
def test_encoder_bytes_equal_the_oracle_encode_at_the_benchmark_configs(mt_lib, oracle_lib, cuda, name):
    """mt_encode_rgb8 on the benchmark configurations (512x512 4:4:4 quality
    60; 1920x1080 4:2:0 at quality 40 / 60 / 80; 4096x4096 4:4:4 quality 60 in
    two tiles) gives the oracle encode's file byte for byte: the same
    decisions, reconstruction, filters, syntax, range coding, headers and
    container."""
    import configs
    from maroontree_b200 import encoder as enc
    from oracle import oracle_avif as oa

    c = configs.CONFIGS[name]
    rgb = synth.generate_rgb(c["w"], c["h"], c["seed"], sigma=c.get("sigma", 4.0), variant=c["variant"])
    chroma = 2 if c["sub"] == 0 else 0
    got = enc.encode_rgb8(rgb, enc.config(quality=c["quality"], chroma=chroma))
    assert got == oa.encode_rgb8(rgb, c["quality"], chroma, threads=configs.THREADS)


# 4160x64, 4163x72 and 4100x131: two tile columns (65 superblock columns;
# the C3 frame has two tile rows)
@pytest.mark.parametrize("w,h,quality,chroma", [(203, 117, 80, 0), (200, 136, 40, 2), (72, 520, 60, 0),
                                                (4160, 64, 60, 2), (4163, 72, 80, 0), (4100, 131, 50, 0)])
def test_encoder_bytes_equal_the_oracle_encode_at_ragged_sizes(mt_lib, oracle_lib, cuda, w, h, quality, chroma):
    from maroontree_b200 import encoder as enc
    from oracle import oracle_avif as oa

    rgb = synth.generate_rgb(w, h, w * 3 + h)
    got = enc.encode_rgb8(rgb, enc.config(quality=quality, chroma=chroma))
    assert got == oa.encode_rgb8(rgb, quality, chroma)


def test_reused_device_buffers_give_the_same_bytes(mt_lib, cuda):
    """Calls of one device share a set of device buffers, grown to the largest
    frame: a small frame after a large one, the large one again, and a call
    after the set is released all give the bytes of the first calls."""
    from maroontree_b200 import encoder as enc

    big, small = synth.generate_rgb(640, 360, 21), synth.generate_rgb(136, 72, 22)
    cfg = enc.config(quality=55)
    a, b = enc.encode_rgb8(big, cfg), enc.encode_rgb8(small, cfg)
    assert enc.encode_rgb8(big, cfg) == a and enc.encode_rgb8(small, cfg) == b
    mt_lib.load().mt_encode_release_buffers()
    assert enc.encode_rgb8(small, cfg) == b and enc.encode_rgb8(big, cfg) == a


def test_batch_encode_equals_each_image_alone(mt_lib, cuda):
    """mt_encode_rgb8_batch: images of different sizes, chroma formats and
    qualities decided in one persistent launch give, each, the bytes of
    encoding it alone (and a batch of one is the single call)."""
    from maroontree_b200 import encoder as enc

    shapes = [(640, 360, 60, 0), (203, 117, 80, 0), (512, 512, 40, 2), (136, 72, 55, 2), (64, 64, 90, 0)]
    imgs = [synth.generate_rgb(w, h, 30 + k) for k, (w, h, _, _) in enumerate(shapes)]
    cfgs = [enc.config(quality=q, chroma=c) for (_, _, q, c) in shapes]
    batch = enc.encode_rgb8_batch(imgs, cfgs)
    alone = [enc.encode_rgb8(im, c) for im, c in zip(imgs, cfgs)]
    assert batch == alone
    assert enc.encode_rgb8_batch(imgs[:1], cfgs[0]) == alone[:1]
