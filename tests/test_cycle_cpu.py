"""The cycle-check oracle (MICycleCheckerCPU, CheckModule/MICycleCheck.cpp):
OpenCV arithmetic pinned against OpenCV itself (cv2, run here), and known
answers on the hand-built micro-image row of test_filter_cpu."""
import numpy as np
import pytest

import pfd_oracle
from conftest import load_pfd
from test_filter_cpu import N, SPACING, line_scene, view

cv2 = pytest.importorskip("cv2")


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def ycfg(**kw):
    return load_pfd().CycleCfg(**kw)


@pytest.mark.parametrize("seed,size", [(1, 16), (2, 16), (3, 21), (4, 10)])
def test_texture_mask_matches_opencv(orc_lib, seed, size):
    """BuildTextureMaskAndViz (MICycleCheck.cpp:186-213): Sobel magnitude and 7x7
    variance with OpenCV's default reflect-101 border, bit for bit."""
    rs = np.random.RandomState(seed)
    g = rs.randint(0, 256, size=(size, size)).astype(np.float32)
    if seed == 2:
        g = np.clip(g * 0.05 + 100, 0, 255).round().astype(np.float32)   # low texture: mask mostly off
    gx = cv2.Sobel(g, cv2.CV_32F, 1, 0, ksize=3)
    gy = cv2.Sobel(g, cv2.CV_32F, 0, 1, ksize=3)
    mag = cv2.magnitude(gx, gy)
    mean = cv2.boxFilter(g, cv2.CV_32F, (7, 7))
    mean2 = cv2.boxFilter(g * g, cv2.CV_32F, (7, 7))
    var = mean2 - mean * mean
    mask = ((mag > 8.0) & (var > 60.0)).astype(np.uint8) * 255
    grad_o, var_o, mask_o = pfd_oracle.texture_mask(g, ycfg())
    # The oracle takes the IEEE square root, as OpenCV 4.2's SIMD magnitude does
    # (v_sqrt of v_muladd); the 4.13 wheel here is up to 2 ulp off, so the
    # magnitude is compared in ulps and the mask away from the 8.0 threshold.
    ulp = np.abs(grad_o.view(np.int32).astype(np.int64) - mag.view(np.int32).astype(np.int64))
    assert ulp.max() <= 2
    assert np.array_equal(grad_o, np.sqrt(gx.astype(np.float64) ** 2 + gy.astype(np.float64) ** 2).astype(np.float32))
    assert np.array_equal(var_o, var)
    near = np.abs(mag - 8.0) < 1e-5
    assert np.array_equal(mask_o[~near], mask[~near])


def test_mean_std_3x3_matches_opencv(orc_lib):
    """cv::meanStdDev of a 3x3 window (MIDisparityFilter.cpp:120-136,
    MICycleCheck.cpp:327-339)."""
    rs = np.random.RandomState(9)
    img = rs.randint(0, 256, size=(16, 16)).astype(np.float32)
    img[4:8, 4:8] = 77                                      # zero-variance windows too
    for y0 in range(14):
        for x0 in range(14):
            m, s = cv2.meanStdDev(img[y0:y0 + 3, x0:x0 + 3])
            om, os_ = pfd_oracle.mean_std_3x3(img, x0, y0)
            assert om == np.float32(m[0, 0]) and os_ == np.float32(s[0, 0]), (x0, y0)


def test_cycle_check_consistent_row(orc_lib):
    orc, st = line_scene()
    stats, geo, pho, tm = pfd_oracle.cycle_check(orc, ycfg(), SPACING, st)
    assert np.all(geo == 0.0)
    # views 0 and 2 see one neighbour at x - 2 / x + 2; view 1 sees one or both
    assert stats["num_samples"] == 120 + 144 + 120
    assert stats["mean_geo_err_px"] == 0.0 and stats["rmse_geo_err_px"] == 0.0
    # reference windows (top-left round(p) - 2) fit for 2 <= x, y <= 9: 64 pixels per view
    assert stats["completeness_masked_pixels"] == 3 * 64
    # two neighbours pass the geometric gate wherever both project inside: view 1, 2 <= x <= 9
    assert stats["completeness_good_pixels_geo"] == 64
    # the photometric gate also needs both neighbour windows: 4 <= x <= 7
    assert stats["completeness_good_pixels_photo"] == 32
    assert stats["completeness_good_pixels"] == 32
    assert stats["completeness"] == 32 / 192
    # z-scores agree on the ramp (0), raw differences are 20 and clamp to 3
    p1 = view(pho, 1)
    assert np.all(p1[2:10, 4:8] == 0.0)
    assert np.all(p1[:, :2] == 3.0)
    assert 0.0 < stats["mean_photo_err"] < 3.0
    # a steep ramp is textured everywhere except the corners, where reflect-101
    # borders zero both Sobel derivatives
    t1 = view(tm, 1).copy()
    assert t1[0, 0] == t1[0, -1] == t1[-1, 0] == t1[-1, -1] == 0
    t1[0, 0] = t1[0, -1] = t1[-1, 0] = t1[-1, -1] = 255
    assert np.all(t1 == 255)


def test_cycle_check_inconsistent_neighbour(orc_lib):
    orc, st = line_scene()
    st["plane"][2 * N * N:, 3] = 3.0
    stats, geo, _, _ = pfd_oracle.cycle_check(orc, ycfg(), SPACING, st)
    g1 = view(geo, 1)
    x = np.arange(N)[None, :].repeat(N, 0)
    # view 1 -> view 2 at x - 2, back with d = 3: off by 1 px; view 1 -> view 0 closes exactly
    assert np.all(g1[x >= 2] == 1.0)
    assert np.all(g1[x < 2] == 0.0)
    # view 2 -> view 1 at x + 3 (d = 3), back with d = 2: off by 1 px
    assert np.all(view(geo, 2)[x <= 8] == 1.0)
    # clamping at 2 px: a 3 px error is reported as 2
    orc, st = line_scene()
    st["plane"][2 * N * N:, 3] = 5.0
    _, geo, _, _ = pfd_oracle.cycle_check(orc, ycfg(), SPACING, st)
    assert np.all(view(geo, 2)[x <= 6] == 2.0)
    _, geo, _, _ = pfd_oracle.cycle_check(orc, ycfg(clamp_geo=False), SPACING, st)
    assert np.all(view(geo, 2)[x <= 6] == 3.0)
