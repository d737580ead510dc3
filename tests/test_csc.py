"""Colour conversion + padding: oracle known answers (CPU) and GPU parity,
including sizes that are not multiples of 8 and 1-pixel images."""
import numpy as np
import pytest

from maroontree_b200 import synth


def test_oracle_csc_matches_numpy_restatement(oracle_lib):
    """The oracle's luma equals the Q13 formula of src/encoder.rs:403-409."""
    rgb = synth.generate_rgb(37, 21, 5)
    y, cb, cr = oracle_lib.csc_rgb8(rgb, 0)
    ref = synth.rgb_to_luma(rgb)
    assert np.array_equal(y[:21, :37], ref)
    assert np.all(y[:21, 37:] == y[:21, 36:37]) and np.all(y[21:, :] == y[20:21, :])


def test_oracle_csc_known_colours(oracle_lib):
    """White -> (255, 128, 128), black -> (0, 128, 128), pure red -> (76, 85, 255) in Q13 BT.601."""
    rgb = np.array([[[255, 255, 255], [0, 0, 0], [255, 0, 0]]], np.uint8)
    y, cb, cr = oracle_lib.csc_rgb8(rgb, 0)
    assert list(y[0, :3]) == [255, 0, 76]
    assert list(cb[0, :3]) == [128, 128, 85]
    assert list(cr[0, :3]) == [128, 128, 255]


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(64, 48), (1001, 777), (1, 1), (9, 3), (1920, 1080)])
@pytest.mark.parametrize("sub", [0, 2])
def test_csc_matches_oracle(mt_lib, oracle_lib, cuda, w, h, sub):
    rgb = synth.generate_rgb(w, h, w * 7 + h)
    a = mt_lib.csc_rgb8(rgb, sub)
    b = oracle_lib.csc_rgb8(rgb, sub)
    for pa, pb in zip(a, b):
        assert pa.shape == pb.shape and np.array_equal(pa, pb)


def test_csc_rejects_bad_sizes(mt_lib):
    from maroontree_b200 import MtError

    with pytest.raises(MtError):
        mt_lib.padded_plane_dims(0, 10, 2)
    with pytest.raises(MtError):
        mt_lib.padded_plane_dims(16384, 10, 0)
    with pytest.raises(MtError):
        mt_lib.padded_plane_dims(16, 16, 1)
