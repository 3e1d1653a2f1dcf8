"""The oracle of the richness channel pinned to OpenCV.

The fixture tests/golden/richness_cv.npz (tests/golden/make_richness_golden.py)
holds the GLCM contrast map of ImageQualityEstimate::QuantizeRichnessByGLCM
built by counting every window's co-occurrence matrix, OpenCV's
cv2.normalize(NORM_MINMAX) of it, windows of the normalised map and counts of
the thresholded 8-bit windows, over frames too small for any window, flat frames
and textures near the threshold.  The box-sum identity the device kernel relies
on is checked against the oracle's literal GLCM here as well.
"""
import os

import numpy as np
import pytest

from oracle import pfd_oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    return np.load(os.path.join(HERE, "golden", "richness_cv.npz"))


def test_glcm_contrast_matches_fixture():
    d = _golden()
    for i in range(int(d["n"])):
        got = orc.glcm_contrast(d[f"gray_{i}"])
        np.testing.assert_array_equal(got, d[f"contrast_{i}"], err_msg=f"image {i}")


def test_normalize_matches_opencv_fixture():
    d = _golden()
    nonzero = 0
    for i in range(int(d["n"])):
        got = orc.normalize_minmax(d[f"contrast_{i}"])
        np.testing.assert_array_equal(got, d[f"norm_{i}"], err_msg=f"image {i}")
        nonzero += int(got.max() > 0)
    assert nonzero >= 3


def test_richness_tiles_match_opencv_fixture():
    d = _golden()
    mw, mh = (int(v) for v in d["win"])
    hits = 0
    for i in range(int(d["n"])):
        score, binary, counts = orc.richness_tiles(d[f"gray_{i}"], d[f"origins_{i}"], mw, mh)
        np.testing.assert_array_equal(score, d[f"tiles_{i}"])
        np.testing.assert_array_equal(counts, d[f"counts_{i}"])
        assert np.array_equal(binary == 255, score > 10) and set(np.unique(binary)) <= {0, 255}
        hits += int(counts.sum())
    assert hits > 0


def _box_sum_contrast(g):
    """The device's form: 7 x 7 box sums of squared diagonal 3-bit differences."""
    q = (g >> 5).astype(np.int64)
    h, w = g.shape
    out = np.zeros((h, w), np.int64)
    if h <= 8 or w <= 8:
        return out
    d = (q[:-1, :-1] - q[1:, 1:]) ** 2
    c = np.cumsum(np.cumsum(np.pad(d, ((1, 0), (1, 0))), 0), 1)
    for row in range(4, h - 4):
        y0, y1 = row - 4, row + 3
        x0 = np.arange(0, w - 8)
        x1 = x0 + 7
        out[row, 4:w - 4] = c[y1, x1] - c[y0, x1] - c[y1, x0] + c[y0, x0]
    return out


@pytest.mark.parametrize("shape,seed", [((37, 53), 1), ((9, 64), 2), ((70, 9), 3)])
def test_glcm_contrast_is_an_integer_box_sum(shape, seed):
    rs = np.random.RandomState(seed)
    g = rs.randint(0, 256, shape).astype(np.uint8)
    g[: shape[0] // 3] = np.clip(rs.normal(100, 25, (shape[0] // 3, shape[1])), 0, 255).astype(np.uint8)
    got = orc.glcm_contrast(g)
    ref = _box_sum_contrast(g)
    assert np.array_equal(got, ref.astype(np.float32))
    assert got.max() <= 49 * 49


def test_richness_tiles_reject_windows_outside():
    g = np.zeros((12, 12), np.uint8)
    with pytest.raises(AssertionError):
        orc.richness_tiles(g, np.array([[9, 0]], np.int32), 4, 4)


def test_normalize_matches_opencv_directly():
    cv2 = pytest.importorskip("cv2")
    rs = np.random.RandomState(8)
    g = rs.randint(0, 256, (83, 121)).astype(np.uint8)
    g[20:50, 30:80] = 200                      # flat patch: zero contrast inside
    c = orc.glcm_contrast(g)
    np.testing.assert_array_equal(orc.normalize_minmax(c), cv2.normalize(c, None, 0, 255, cv2.NORM_MINMAX))
    for mx in (1, 7, 49, 255, 1000, 2401):
        m = np.zeros((5, 7), np.float32)
        m[2, 3] = mx
        m[1, 1] = mx // 3
        np.testing.assert_array_equal(orc.normalize_minmax(m), cv2.normalize(m, None, 0, 255, cv2.NORM_MINMAX))
