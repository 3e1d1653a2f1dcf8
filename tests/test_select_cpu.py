"""Matching-neighbour selection oracle (SelectNeighbors::CollectMIANeighImagesForMatch,
MINeighbor/SelectNeighbors.cpp:113-193, with MISimilarityMeasure::MeasureSimilarity,
Util/MISimilarityMeasure.cpp:173-284).

The similarity is pinned against OpenCV: a Python restatement of
MeasureSimilarity that calls cv2.threshold, cv2.warpAffine(INTER_NEAREST),
cv2.compare, cv2.bitwise_and and cv2.countNonZero exactly as the reference does
must give the oracle's count.  The lists are checked against the reference's
rules on hexagonal arrays."""
import math

import numpy as np
import pytest

import pfd_oracle

cv2 = pytest.importorskip("cv2")


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def measure_similarity_cv2(src_gray, nb_gray, dx, dy):
    """MeasureSimilarity with OpenCV's own operations; the shift loop runs in
    order on one thread (the nested OpenMP region is inactive)."""
    _, src = cv2.threshold(src_gray, 128, 255, cv2.THRESH_BINARY)
    _, nb = cv2.threshold(nb_gray, 128, 255, cv2.THRESH_BINARY)
    dx, dy = np.float32(dx), np.float32(dy)
    if abs(dx) < 5:
        dx = np.float32(0)
    if abs(dy) < 5:
        dy = np.float32(0)
    norm = np.float32(math.sqrt(np.float32(dx * dx + dy * dy)))
    dxs = np.float32(np.float32(dx / norm) * np.float32(2))
    dys = np.float32(np.float32(dy / norm) * np.float32(2))
    H, W = src.shape
    with np.errstate(divide="ignore"):
        fx, fy = np.float32(W) / np.float32(abs(dxs)), np.float32(H) / np.float32(abs(dys))
    dxc = int(fx) if abs(fx) < 2 ** 31 else -2 ** 31
    dyc = int(fy) if abs(fy) < 2 ** 31 else -2 ** 31
    if dxs == 0:
        dxc = 0
    elif dys == 0:
        dyc = 0
    steps = int(math.ceil(max(dxc, dyc)))
    counts = [0] * max(steps, 0)
    sx = sy = np.float32(0)
    for step in range(steps):
        if abs(sx) >= W or abs(sy) >= H:
            continue
        M = np.array([[1, 0, float(sx)], [0, 1, float(sy)]], np.float64)
        shifted = cv2.warpAffine(nb, M, (W, H), flags=cv2.INTER_NEAREST, borderMode=cv2.BORDER_CONSTANT, borderValue=0)
        overlap = np.zeros_like(src)
        x1, y1 = int(max(np.float32(0), sx)), int(max(np.float32(0), sy))
        x2 = int(math.floor(min(np.float32(W - 1), np.float32(np.float32(sx + W) - 1))))
        y2 = int(math.floor(min(np.float32(H - 1), np.float32(np.float32(sy + H) - 1))))
        if x2 >= x1 and y2 >= y1:
            overlap[y1:y2 + 1, x1:x2 + 1] = 255
        eq = cv2.compare(src, shifted, cv2.CMP_EQ)
        counts[step] = cv2.countNonZero(cv2.bitwise_and(eq, overlap))
        sx = np.float32(np.float32(step) * dxs)
        sy = np.float32(np.float32(step) * dys)
    return max(counts) if counts else 0


@pytest.mark.parametrize("seed", range(6))
def test_similarity_matches_opencv(orc_lib, seed):
    rs = np.random.RandomState(seed)
    m = 16
    base = (rs.rand(m + 12, m + 12) * 255).astype(np.uint8)
    base = cv2.GaussianBlur(base, (5, 5), 1.5)
    src = np.ascontiguousarray(base[6:6 + m, 6:6 + m])
    for ang in np.linspace(0, 2 * np.pi, 13)[:-1]:
        for r in (23.2, 40.18, 46.4):
            dx, dy = np.float32(r * np.cos(ang + 0.01 * seed)), np.float32(r * np.sin(ang + 0.01 * seed))
            sh = (int(rs.randint(-3, 4)), int(rs.randint(-3, 4)))
            nb = np.ascontiguousarray(base[6 + sh[1]:6 + sh[1] + m, 6 + sh[0]:6 + sh[0] + m])
            _, sb = cv2.threshold(src, 128, 255, cv2.THRESH_BINARY)
            _, nbb = cv2.threshold(nb, 128, 255, cv2.THRESH_BINARY)
            got = orc_lib.similarity(sb, nbb, float(dx), float(dy))
            assert got == measure_similarity_cv2(src, nb, dx, dy), (ang, r)


def test_warp_nearest_fixed_point(orc_lib):
    """Sub-pixel shifts near the rounding boundary of OpenCV's 10-bit fixed
    point, where a float rounding would pick the other source pixel."""
    rs = np.random.RandomState(3)
    img = (rs.rand(16, 16) > 0.5).astype(np.uint8) * 255
    for s in (0.4995, 0.5, 0.5004, 0.50049, 1.4990, 1.5, -0.5, -0.50049, 2.00048, 3.4996):
        M = np.array([[1, 0, s], [0, 1, -s]], np.float64)
        w = cv2.warpAffine(img, M, (16, 16), flags=cv2.INTER_NEAREST, borderMode=cv2.BORDER_CONSTANT, borderValue=0)
        x0 = int(np.rint(-np.float32(s) * 1024.0)) + 512
        ref = np.zeros_like(img)
        for y in range(16):
            Y = (int(np.rint((y + float(np.float32(s))) * 1024.0)) + 512) >> 10
            for x in range(16):
                X = (x0 + x * 1024) >> 10
                ref[y, x] = img[Y, X] if 0 <= X < 16 and 0 <= Y < 16 else 0
        assert np.array_equal(w, ref), s


def hex_array(cols, rows, pitch, jitter=0.0, seed=0):
    rs = np.random.RandomState(seed)
    c, k = [], []
    for r in range(rows):
        for q in range(cols):
            c.append((30 + q * pitch + (pitch / 2 if r % 2 else 0) + rs.uniform(-jitter, jitter),
                      30 + r * pitch * math.sqrt(3) / 2 + rs.uniform(-jitter, jitter)))
            k.append((q, r))
    return np.array(c, np.float32), np.array(k, np.int32)


def test_geometric_lists(orc_lib):
    """No images: no candidate is rejected, so every lens collects five rings
    (6, 12, 18, 24, 30 lenses in the interior), best first by baseline."""
    pitch = 23.2
    c, k = hex_array(24, 22, pitch, jitter=0.05)
    ids, cnt, _ = orc_lib.select_neighbors(c, k, 24, 22, pitch)
    interior = [v for v in range(len(c)) if 6 <= k[v, 0] < 18 and 6 <= k[v, 1] < 16]
    assert len(interior) > 50
    for v in interior:
        assert cnt[v] == 90
        b = np.linalg.norm(c[ids[v, :90]].astype(np.float64) - c[v], axis=1)
        assert np.all(np.diff(b) > -0.5)          # best first = nearest first (up to the jitter)
        assert np.all(np.abs(b[:6] - pitch) < 0.2)
    assert np.all(cnt <= 90) and np.all(cnt >= 6)


def test_ransac_rejects_dissimilar_outer_lenses(orc_lib):
    """Micro-images that all look alike except beyond the second ring: the
    line fitted on the first two rings predicts a high similarity, so the
    dissimilar outer lenses are outliers; two or more outliers in a ring stop
    the search there."""
    pitch = 23.2
    c, k = hex_array(20, 18, pitch)
    V, m = len(c), 16
    rs = np.random.RandomState(5)
    pattern = np.where(rs.rand(m, m) > 0.5, 200, 40).astype(np.uint8)
    imgs = np.repeat(pattern[None], V, 0).copy()
    centre = int(np.argmin(np.linalg.norm(c - c.mean(0), axis=1)))
    far = np.linalg.norm(c - c[centre], axis=1) > 2.5 * pitch
    imgs[far] = 255 - imgs[far]
    ids, cnt, sim = orc_lib.select_neighbors(c, k, 20, 18, pitch, images=imgs)
    got = set(ids[centre, :cnt[centre]].tolist())
    near = {v for v in range(V) if v != centre and not far[v]}
    # the first two rings (6 + 12 lenses, within 2 pitches) are kept; the third
    # ring (from sqrt(7) pitches) is all outliers and ends the search
    assert len(near) == 18 and got == near and cnt[centre] == 18
    assert np.all(sim[centre, :18] > 0.8 * m * m)


def test_geometry_only_lists_match_the_engine_host_code(orc_lib):
    """pfd_neighbors_by_baseline (the engine's host code, no device) is the
    selection with every similarity 0: equal to the oracle's lists."""
    from conftest import load_pfd
    pfd = load_pfd()
    for seed, jitter in ((0, 0.0), (1, 0.3), (2, 1.5)):
        c, k = hex_array(22, 19, 23.2, jitter=jitter, seed=seed)
        ids, cnt = pfd.neighbors_by_baseline(c, k, 23.2, 128, rings=5)
        oids, ocnt, _ = orc_lib.select_neighbors(c, k, 22, 19, 23.2)
        assert np.array_equal(cnt, ocnt)
        assert np.array_equal(ids, oids)
