"""Conformance against a real AV1 decoder.  A 4:4:4 picture of 8x8 blocks in
every intra mode (with angle deltas) and every 8x8 intra transform type is
coded block by block by the candidate chain, its coefficients by the token
emitter, and packed, wrapped and decoded by dav1d (Pillow's libavif); the
decoded picture must equal the coder's reconstruction sample for sample.  With
the oracle as the coder this pins the oracle's prediction, forward and inverse
transforms, quantisation matrices and coefficient coder to the AV1 decoding
process; with the CUDA kernels (-m gpu) it checks the library's candidate
chain and token emitter the same way."""
import numpy as np
import pytest

from stream_harness import encode_and_decode


@pytest.mark.parametrize("qidx,qm", [(70, 6), (116, 15), (35, 8)])
def test_oracle_stream_decodes_to_its_reconstruction(mt_lib, oracle_lib, qidx, qm):
    c, rgb, _ = encode_and_decode(mt_lib, oracle_lib, 128, 64, 5 + qidx, qidx, qm, gpu=False)
    dec = [rgb[..., 1], rgb[..., 2], rgb[..., 0]]  # identity matrix: G, B, R = Y, U, V
    for p in range(3):
        bad = np.argwhere(dec[p] != c.rec[p])
        assert len(bad) == 0, (p, bad[:4], dec[p][tuple(bad[0])], c.rec[p][tuple(bad[0])])


@pytest.mark.parametrize("qidx,qm", [(70, 6), (160, 15), (116, 2)])
def test_oracle_filters_match_decoder(mt_lib, oracle_lib, qidx, qm):
    """The same stream with the loop filter and CDEF on: dav1d's output equals
    the oracle's deblocked, CDEF-filtered planes, which pins the oracle's
    deblocking and CDEF (and the library's cdef_idx replay) to the decoder."""
    c, rgb, _ = encode_and_decode(mt_lib, oracle_lib, 192, 128, 3 + qidx, qidx, qm, gpu=False, filters=True)
    dec = [rgb[..., 1], rgb[..., 2], rgb[..., 0]]
    for p in range(3):
        bad = np.argwhere(dec[p] != c.out[p])
        assert len(bad) == 0, (p, c.cdef["bits"], bad[:4])


@pytest.mark.gpu
@pytest.mark.parametrize("qidx,qm", [(70, 6), (116, 15)])
def test_gpu_stream_decodes_to_its_reconstruction(mt_lib, oracle_lib, cuda, qidx, qm):
    c, rgb, avif = encode_and_decode(mt_lib, oracle_lib, 128, 128, 9 + qidx, qidx, qm, gpu=True)
    dec = [rgb[..., 1], rgb[..., 2], rgb[..., 0]]
    for p in range(3):
        assert np.array_equal(dec[p], c.rec[p]), p
    # and the oracle codes the same picture to the same bytes
    c2, _, avif2 = encode_and_decode(mt_lib, oracle_lib, 128, 128, 9 + qidx, qidx, qm, gpu=False)
    assert avif2 == avif


@pytest.mark.parametrize("sigma", [0.0, 1.0])
def test_oracle_cdef_on_matches_decoder(mt_lib, oracle_lib, sigma):
    """A smooth 256x256 picture coded with each block's cheapest (mode, type):
    the oracle's CDEF search turns CDEF on (cdef_bits 1), and dav1d applies the
    signalled strengths per 64x64 unit exactly as the oracle's CDEF did."""
    c, rgb, _ = encode_and_decode(mt_lib, oracle_lib, 256, 256, 7, 120, 15, gpu=False, filters=True, pick="best",
                                  sigma=sigma)
    assert c.cdef["bits"] >= 1 and any(any(s) for s in c.cdef["strengths"])
    dec = [rgb[..., 1], rgb[..., 2], rgb[..., 0]]
    for p in range(3):
        assert np.array_equal(dec[p], c.out[p]), p
