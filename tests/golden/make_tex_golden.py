"""Records tex2D samples on a CUDA device into tests/golden/tex2d_samples.npz.

Run on a GPU machine from the repository root after building the test helpers
(python plenoptic-for-depth_b200/build.py):
    python tests/golden/make_tex_golden.py
The texture is configured like the reference's micro-image textures
(float32 cudaArray, linear filtering, unnormalised coordinates, wrap mode;
AdaptMIPMFrame.cpp:224-249) and fetched at (x + 0.5, y + 0.5).  The CPU test
test_tex_fetch_matches_recorded_hardware compares the oracle's emulation with
these recorded values.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(os.path.dirname(HERE), "_build", "libtexprobe.so")


def probe(L, img, xs, ys, mode):
    img = np.ascontiguousarray(img, np.float32)
    xs = np.ascontiguousarray(xs, np.float32)
    ys = np.ascontiguousarray(ys, np.float32)
    out = np.zeros(len(xs), np.float32)
    rc = L.tex_probe(img.ctypes.data, img.shape[1], img.shape[0], xs.ctypes.data, ys.ctypes.data, len(xs), mode,
                     out.ctypes.data)
    if rc != 0:
        sys.exit(f"tex_probe failed: {rc}")
    return out


def main():
    L = ctypes.CDLL(PROBE)
    L.tex_probe.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    rs = np.random.RandomState(4)
    res = {}
    for (h, w) in [(16, 16), (21, 21)]:
        img = rs.randint(0, 256, size=(h, w)).astype(np.float32)
        n = 4000
        xs = rs.uniform(0, w, n).astype(np.float32)
        ys = rs.uniform(0, h, n).astype(np.float32)
        xs[:400] = np.float32(w) - rs.uniform(0, 2, 400).astype(np.float32)       # right edge (clamp)
        ys[400:800] = np.float32(h) - rs.uniform(0, 2, 400).astype(np.float32)    # bottom edge
        k = rs.randint(0, w * 256, 800)
        xs[800:1600] = ((k + 0.5) / 256.0).astype(np.float32)                     # rounding ties in x
        ys[1600:2400] = ((rs.randint(0, h * 256, 800) + 0.5) / 256.0).astype(np.float32)
        xs = np.clip(xs, 0, np.nextafter(np.float32(w), np.float32(0)))
        ys = np.clip(ys, 0, np.nextafter(np.float32(h), np.float32(0)))
        res[f"img{h}"] = img
        res[f"xs{h}"] = xs
        res[f"ys{h}"] = ys
        res[f"out{h}"] = probe(L, img, xs, ys, 0)
    np.savez_compressed(os.path.join(HERE, "tex2d_samples.npz"), **res)
    print("wrote", os.path.join(HERE, "tex2d_samples.npz"))


if __name__ == "__main__":
    main()
