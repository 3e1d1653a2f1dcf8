"""Micro-lens centre detection oracle (DepthSolver::ComputeMLACentersFromWhiteImage,
DepthSolver.cpp:710-870) pinned against OpenCV: the contour centroids and
areas of orc_mla_contours must equal cv2.findContours(RETR_EXTERNAL,
CHAIN_APPROX_SIMPLE) + cv2.moments / cv2.contourArea on the same thresholded
image, in cv2's order, bit for bit (the Python cv2 here is 4.13; the reference
pins 4.2.0, whose contour and moment code is the same algorithm).  Then the
row/column bookkeeping on hexagonal white images."""
import numpy as np
import pytest

import pfd_oracle

cv2 = pytest.importorskip("cv2")


def white_image(W, H, pitch, seed, radius_frac=0.46, noise=3.0, x0=None, y0=None):
    """Hexagonal lens array (rows horizontal, odd rows shifted by pitch / 2)
    seen through a uniform white target: bright disks with soft edges."""
    rs = np.random.RandomState(seed)
    x0 = pitch * 0.5 + 1.3 if x0 is None else x0
    y0 = pitch * 0.5 + 0.7 if y0 is None else y0
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float64)
    img = np.zeros((H, W))
    dy = pitch * np.sqrt(3) / 2
    centers = []
    r = 0
    while y0 + r * dy < H + pitch:
        cy = y0 + r * dy
        c = 0
        while x0 + c * pitch + (pitch / 2 if r % 2 else 0) < W + pitch:
            cx = x0 + c * pitch + (pitch / 2 if r % 2 else 0)
            centers.append((cx, cy))
            c += 1
        r += 1
    rad = int(np.ceil(radius_frac * pitch)) + 1
    for cx, cy in centers:
        x0b, x1b = max(0, int(cx) - rad), min(W, int(cx) + rad + 2)
        y0b, y1b = max(0, int(cy) - rad), min(H, int(cy) + rad + 2)
        if x0b >= x1b or y0b >= y1b:
            continue
        d = np.hypot(xs[y0b:y1b, x0b:x1b] - cx, ys[y0b:y1b, x0b:x1b] - cy) / (radius_frac * pitch)
        img[y0b:y1b, x0b:x1b] = np.maximum(img[y0b:y1b, x0b:x1b], 230.0 * np.clip(1.0 - d ** 4, 0, 1))
    img += rs.normal(0, noise, size=img.shape) + 12
    gray = np.clip(np.rint(img), 0, 255).astype(np.uint8)
    return np.ascontiguousarray(np.repeat(gray[:, :, None], 3, axis=2)), np.array(centers)


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def test_gray_and_threshold_match_opencv(orc_lib):
    rs = np.random.RandomState(0)
    bgr = rs.randint(0, 256, size=(137, 253, 3)).astype(np.uint8)
    g = cv2.cvtColor(bgr, cv2.COLOR_BGR2GRAY)
    b = bgr.astype(np.int64)
    assert np.array_equal(g, ((b[..., 0] * 3735 + b[..., 1] * 19235 + b[..., 2] * 9798 + 16384) >> 15).astype(np.uint8))
    _, th = cv2.threshold(g, 117, 255, cv2.THRESH_BINARY)
    assert np.array_equal(th, np.where(g > 117, 255, 0).astype(np.uint8))


@pytest.mark.parametrize("seed,pitch", [(1, 23.0), (2, 17.3), (3, 30.1)])
def test_contours_match_opencv(orc_lib, seed, pitch):
    bgr, _ = white_image(320, 240, pitch, seed)
    t = orc_lib.mla_otsu(bgr)
    assert 20 < t < 230
    cx, cy, area = orc_lib.mla_contours(bgr, t)
    g = cv2.cvtColor(bgr, cv2.COLOR_BGR2GRAY)
    _, th = cv2.threshold(g, t, 255, cv2.THRESH_BINARY)
    contours, _ = cv2.findContours(th, cv2.RETR_EXTERNAL, cv2.CHAIN_APPROX_SIMPLE)
    assert len(contours) == len(cx) > 50
    for k, c in enumerate(contours):
        m = cv2.moments(c)
        ex, ey = (np.float32(m["m10"] / m["m00"]), np.float32(m["m01"] / m["m00"])) if m["m00"] != 0 else (-1, -1)
        assert cx[k] == ex and cy[k] == ey, (k, cx[k], ex, cy[k], ey)
        assert area[k] == cv2.contourArea(c)


def test_odd_shapes_match_opencv(orc_lib):
    """Spurs, single pixels, diagonal chains, a ring with a hole, shapes at
    the image border."""
    img = np.zeros((40, 60), np.uint8)
    img[5, 5] = 200                                  # single pixel
    img[10:13, 3:12] = 200
    img[13:20, 7] = 200                              # spur
    for i in range(8):
        img[25 + i, 20 + i] = 200                    # diagonal chain
    cv2.circle(img, (45, 15), 9, 200, -1)
    cv2.circle(img, (45, 15), 4, 0, -1)              # hole
    img[0:6, 55:60] = 200                            # touches two borders
    img[35:40, 0:3] = 200
    bgr = np.ascontiguousarray(np.repeat(img[:, :, None], 3, axis=2))
    cx, cy, area = orc_lib.mla_contours(bgr, 100)
    contours, _ = cv2.findContours(np.where(img > 100, 255, 0).astype(np.uint8), cv2.RETR_EXTERNAL,
                                   cv2.CHAIN_APPROX_SIMPLE)
    assert len(contours) == len(cx)
    for k, c in enumerate(contours):
        m = cv2.moments(c)
        ex, ey = (np.float32(m["m10"] / m["m00"]), np.float32(m["m01"] / m["m00"])) if m["m00"] != 0 else (-1, -1)
        assert (cx[k], cy[k]) == (ex, ey), k
        assert area[k] == cv2.contourArea(c), k


def test_otsu_restates_the_reference(orc_lib):
    """DepthSolver::Otsu reads the first W bytes of each row of the 3-channel
    image: for a gray image, the left third of the pixels, each three times."""
    bgr, _ = white_image(300, 200, 23.0, 5)
    left = bgr.reshape(200, -1)[:, :300]
    hist = np.bincount(left.ravel(), minlength=256).astype(np.float32)
    pro = hist / np.float32(300 * 200)
    best, t = np.float32(0), 0
    for i in range(256):
        w0 = w1 = u0t = u1t = np.float32(0)
        for j in range(256):
            if j <= i:
                w0 = np.float32(w0 + pro[j]); u0t = np.float32(u0t + np.float32(j) * pro[j])
            else:
                w1 = np.float32(w1 + pro[j]); u1t = np.float32(u1t + np.float32(j) * pro[j])
        with np.errstate(divide="ignore", invalid="ignore"):
            u0, u1 = np.float32(u0t / w0), np.float32(u1t / w1)
            u = np.float32(u0t + u1t)
            d = np.float32(np.float32(np.float32(w0 * np.float32(u0 - u)) * np.float32(u0 - u)) +
                           np.float32(np.float32(w1 * np.float32(u1 - u)) * np.float32(u1 - u)))
        if d > best:
            best, t = d, i
    assert orc_lib.mla_otsu(bgr) == t


def test_rows_and_columns(orc_lib):
    pitch = 23.0
    bgr, centers = white_image(400, 300, pitch, 7)
    u_size, v_size = int(400 / pitch) + 1, int(300 / (pitch * np.sqrt(3) / 2)) + 1
    m, t = orc_lib.mla_centers(bgr, pitch, u_size, v_size)
    assert len(m["col"]) > 150
    # key order and a plausible grid: every row's columns run 0..n-1 with x increasing
    keys = list(zip(m["row"], m["col"]))
    assert keys == sorted(keys)
    for r in np.unique(m["row"]):
        sel = m["row"] == r
        assert np.array_equal(m["col"][sel], np.arange(sel.sum()))
        assert np.all(np.diff(m["cx"][sel]) > 0)
        assert np.ptp(m["cy"][sel]) < pitch * 0.5
    # detected centres sit on the generated lenses
    full = ~m["abandon"].astype(bool)
    d = np.min(np.hypot(m["cx"][full, None] - centers[None, :, 0], m["cy"][full, None] - centers[None, :, 1]), axis=1)
    assert np.median(d) < 0.2 and np.max(d) < 0.75
    # lenses cut by the image border are flagged
    assert np.any(m["abandon"])
