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
