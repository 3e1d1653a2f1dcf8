"""Records OpenCV's blur-channel arithmetic into tests/golden/blur_cv.npz.

Run from the repository root where OpenCV's Python package is importable:
    python tests/golden/make_blur_golden.py
For seeded gray images of several shapes (edges, single rows and columns
included) it stores cv2.Laplacian(gray, CV_32F) with ksize 1 (what
ImageQualityEstimate::QuantizeBlurByLaplacian computes), and for windows cut at
seeded corners the window converted to 8 bits with OpenCV's saturating
conversion and the count of 255s in the window of cv2.threshold(score, 10, 255,
THRESH_BINARY) converted the same way (DepthSolver::SliceAndIndicatlizeForMI
and MLA_Problem::ComputeBlurenessValue).  The CPU test
tests/test_blur_cpu.py compares the oracle with these values.
"""
import os

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPES = [(1, 1), (1, 7), (6, 1), (2, 2), (3, 5), (17, 23), (48, 64)]
WIN = (5, 4)      # mi_w, mi_h of the windows cut from the larger images


def to_u8(a):
    """OpenCV's saturating conversion to 8 bits (saturate_cast<uchar>)."""
    return cv2.add(a, np.zeros_like(a), dtype=cv2.CV_8U)


def main():
    rs = np.random.RandomState(11)
    res = {}
    for i, (h, w) in enumerate(SHAPES):
        kind = i % 3
        if kind == 0:
            g = rs.randint(0, 256, (h, w)).astype(np.uint8)
        elif kind == 1:
            g = (rs.rand(h, w) < 0.3).astype(np.uint8) * 255      # saturating edges both ways
        else:
            g = np.clip(rs.normal(128, 6, (h, w)), 0, 255).astype(np.uint8)    # near the threshold of 10
        score = cv2.Laplacian(g, cv2.CV_32F, ksize=1)
        res[f"gray_{i}"] = g
        res[f"score_{i}"] = score
        mw, mh = WIN
        if w >= mw and h >= mh:
            n = 6
            ox = rs.randint(0, w - mw + 1, n)
            oy = rs.randint(0, h - mh + 1, n)
            origins = np.stack([ox, oy], 1).astype(np.int32)
            u8 = to_u8(score)
            _, binary = cv2.threshold(score, 10, 255, cv2.THRESH_BINARY)
            b8 = to_u8(binary)
            tiles = np.stack([u8[y:y + mh, x:x + mw] for x, y in origins])
            counts = np.array([int((b8[y:y + mh, x:x + mw] == 255).sum()) for x, y in origins], np.uint32)
            res[f"origins_{i}"] = origins
            res[f"tiles_{i}"] = tiles
            res[f"counts_{i}"] = counts
    np.savez_compressed(os.path.join(HERE, "blur_cv.npz"), n=len(SHAPES), win=np.array(WIN), **res)


if __name__ == "__main__":
    main()
