"""The two single-frame workloads the parity tests run at full size.

small: 1024x768 8-bit raw, hexagonal MLA of pitch 23.0 px, 4 slanted planes
       (virtual depth 2-12), 6 neighbours, 11x11 bilateral NCC (sigma_s 3,
       sigma_c 12), 3 red-black iterations.
full:  4080x3068 raw, pitch 23.2 px, three interleaved lens types blurred with
       sigma 0.6 / 1.0 / 1.4 px, 12 planes, 12 neighbours, 15x15 NCC,
       8 iterations, then the cycle check, the disparity filter and a 64-slice
       focal stack of 2040x1534 (virtual depth 2-12).
"""
import numpy as np

SMALL = dict(width=1024, height=768, pitch=23.0, n_planes=4, max_nb=6, patch=11, iters=3, seed=2026, kw={})
FULL = dict(width=4080, height=3068, pitch=23.2, n_planes=12, max_nb=12, patch=15, iters=8, seed=2026,
            kw=dict(n_lens_types=3, blur_sigma=(0.6, 1.0, 1.4)))

_cache = {}


def workload(pfd, cfg):
    key = (cfg["width"], cfg["height"], cfg["pitch"], cfg["seed"])
    if key not in _cache:
        _cache[key] = pfd.make_workload(cfg["width"], cfg["height"], cfg["pitch"], cfg["n_planes"], seed=cfg["seed"],
                                        max_nb=cfg["max_nb"], **cfg["kw"])
    return _cache[key]


def params(pfd, cfg, iters=None):
    return pfd.PmParams(base=cfg["pitch"], patch_size=cfg["patch"],
                        max_iterations=cfg["iters"] if iters is None else iters, sigma_spatial=3.0,
                        sigma_color=12.0)


def slice_vds(n=64, lo=2.0, hi=12.0):
    return np.linspace(lo, hi, n).astype(np.float32)


def virtual_depth(plane, pitch):
    """Virtual depth of each pixel, pitch / disparity (disparity = plane.w)."""
    return pitch / np.maximum(plane[:, 3], 1e-6)
