"""The oracle of the blur channel pinned to OpenCV.

The fixture tests/golden/blur_cv.npz holds OpenCV's own outputs
(tests/golden/make_blur_golden.py): cv2.Laplacian with ksize 1 over images with
one-pixel rows and columns, saturating edges and values near the threshold, and
windows of the saturated score and counts of the thresholded map.  Where OpenCV
is importable, a larger seeded frame is compared directly too.
"""
import os

import numpy as np
import pytest

from oracle import pfd_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    return np.load(os.path.join(HERE, "golden", "blur_cv.npz"))


def test_laplacian_matches_opencv_fixture():
    d = _golden()
    for i in range(int(d["n"])):
        got = orc.laplacian(d[f"gray_{i}"])
        np.testing.assert_array_equal(got, d[f"score_{i}"], err_msg=f"image {i} {d[f'gray_{i}'].shape}")


def test_blur_tiles_match_opencv_fixture():
    d = _golden()
    mw, mh = (int(v) for v in d["win"])
    seen = 0
    for i in range(int(d["n"])):
        if f"tiles_{i}" not in d:
            continue
        tiles, counts = orc.blur_tiles(d[f"gray_{i}"], d[f"origins_{i}"], mw, mh)
        np.testing.assert_array_equal(tiles, d[f"tiles_{i}"])
        np.testing.assert_array_equal(counts, d[f"counts_{i}"])
        seen += 1
    assert seen >= 2


def test_blur_tiles_reject_windows_outside():
    g = np.zeros((8, 8), np.uint8)
    with pytest.raises(AssertionError):
        orc.blur_tiles(g, np.array([[5, 0]], np.int32), 4, 4)


def test_window_origins_follow_the_frame_convention():
    # centre minus (mi - 1) / 2, truncated: (10.9 - 2.5) -> 8, (3.0 - 2.0) -> 1
    o = orc.window_origins(np.array([[10.9, 3.0]], np.float32), 6, 5)
    assert o.tolist() == [[8, 1]]


def test_laplacian_matches_opencv_directly():
    cv2 = pytest.importorskip("cv2")
    rs = np.random.RandomState(5)
    g = rs.randint(0, 256, (97, 131)).astype(np.uint8)
    g[40:60, 50:90] = 128                      # flat patch: zeros inside
    np.testing.assert_array_equal(orc.laplacian(g), cv2.Laplacian(g, cv2.CV_32F, ksize=1))
