"""Records OpenCV's richness-channel arithmetic into tests/golden/richness_cv.npz.

Run from the repository root where OpenCV's Python package is importable:
    python tests/golden/make_richness_golden.py
For seeded gray images of several shapes (frames too small for any 8x8 window,
flat frames and frames with a single window included) it stores the GLCM
contrast map of ImageQualityEstimate::QuantizeRichnessByGLCM
(Util/ImageQualityEstimate.cpp:310-340, calculate_matrix :659-682), built here
by counting the 8x8 co-occurrence matrix of every window with numpy, and
OpenCV's cv2.normalize(map, 0, 255, NORM_MINMAX) of it.  For windows cut at
seeded corners it stores the normalised window (DepthSolver::GetRichnessScoreMI)
and the count of 255s of the window of cv2.threshold(normalised, 10, 255,
THRESH_BINARY) converted to 8 bits (DepthSolver::SliceAndIndicatlizeForMI and
MLA_Problem::ComputeRichnessValue).  tests/test_richness_cpu.py compares the
oracle with these values.
"""
import os

import cv2
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPES = [(8, 8), (9, 9), (9, 30), (5, 40), (12, 12), (23, 17), (40, 56), (64, 48)]
WIN = (6, 5)      # mi_w, mi_h of the windows cut from the images


def contrast_map(g):
    """calculate_matrix over every window that fits, zero elsewhere."""
    h, w = g.shape
    out = np.zeros((h, w), np.float32)
    q = (g // 32).astype(np.int64)
    for row in range(4, h - 4):
        for col in range(4, w - 4):
            m = q[row - 4:row + 4, col - 4:col + 4]
            glcm = np.zeros((8, 8), np.float32)
            np.add.at(glcm, (m[:-1, :-1].ravel(), m[1:, 1:].ravel()), 1.0)
            ij = np.subtract.outer(np.arange(8), np.arange(8)) ** 2
            out[row, col] = np.float32((glcm * ij.astype(np.float32)).sum(dtype=np.float64))
    return out


def to_u8(a):
    """OpenCV's saturating conversion to 8 bits (saturate_cast<uchar>)."""
    return cv2.add(a, np.zeros_like(a), dtype=cv2.CV_8U)


def main():
    rs = np.random.RandomState(23)
    res = {}
    for i, (h, w) in enumerate(SHAPES):
        kind = i % 4
        if kind == 0:
            g = rs.randint(0, 256, (h, w)).astype(np.uint8)
        elif kind == 1:
            g = np.full((h, w), 77, np.uint8)                                   # flat: max - min is 0
        elif kind == 2:
            g = np.clip(rs.normal(128, 20, (h, w)), 0, 255).astype(np.uint8)   # few levels apart
        else:
            g = np.where(rs.rand(h, w) < 0.08, 255, 20).astype(np.uint8)       # sparse texture, values near 10
        score = contrast_map(g)
        norm = cv2.normalize(score, None, 0, 255, cv2.NORM_MINMAX)
        _, binary = cv2.threshold(norm, 10, 255, cv2.THRESH_BINARY)
        b8 = to_u8(binary)
        res[f"gray_{i}"] = g
        res[f"contrast_{i}"] = score
        res[f"norm_{i}"] = norm
        mw, mh = WIN
        n = 5
        ox = rs.randint(0, w - mw + 1, n)
        oy = rs.randint(0, h - mh + 1, n)
        origins = np.stack([ox, oy], 1).astype(np.int32)
        res[f"origins_{i}"] = origins
        res[f"tiles_{i}"] = np.stack([norm[y:y + mh, x:x + mw] for x, y in origins])
        res[f"counts_{i}"] = np.array([int((b8[y:y + mh, x:x + mw] == 255).sum()) for x, y in origins], np.uint32)
    np.savez_compressed(os.path.join(HERE, "richness_cv.npz"), n=len(SHAPES), win=np.array(WIN), **res)


if __name__ == "__main__":
    main()
