"""The focal-stack render of the oracle (orc_refocus), checked against a
brute-force numpy restatement of the same definition (every view tested for
every output pixel, no culling) and against known answers."""
import numpy as np
import pytest

import pfd_oracle
from conftest import load_pfd


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def brute_force(gray, centers, raw_w, raw_h, vds, out_w, out_h):
    """Direct numpy form of the render with the same float32 operation order;
    fma(a, b, c) is exact here as round32(a*b + c) in float64 because |a| < 1,
    |b| <= 255 and c is an integer <= 255 (49 significant bits at most)."""
    V, mh, m = gray.shape
    f32 = np.float32
    cmx, cmy = f32(m - 1) * f32(0.5) + f32(1), f32(mh - 1) * f32(0.5) + f32(1)
    sx, sy = f32(raw_w) / f32(out_w), f32(raw_h) / f32(out_h)
    X = (np.arange(out_w, dtype=f32) + f32(0.5)) * sx - f32(0.5)
    Y = (np.arange(out_h, dtype=f32) + f32(0.5)) * sy - f32(0.5)
    out = np.zeros((len(vds), out_h, out_w), f32)

    def fma(a, b, c):
        return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(f32)

    for s, v in enumerate(np.asarray(vds, f32)):
        acc = np.zeros((out_h, out_w), f32)
        cnt = np.zeros((out_h, out_w), np.int32)
        for i in range(V):
            u = (X - f32(centers[i, 0])) / v + cmx
            w = (Y - f32(centers[i, 1])) / v + cmy
            uu, ww = np.meshgrid(u, w)
            ok = (uu >= 0) & (uu <= f32(m - 1)) & (ww >= 0) & (ww <= f32(mh - 1))
            if not ok.any():
                continue
            uu, ww = uu[ok], ww[ok]
            x0, y0 = np.floor(uu).astype(int), np.floor(ww).astype(int)
            x1, y1 = np.minimum(x0 + 1, m - 1), np.minimum(y0 + 1, mh - 1)
            ax, ay = (uu - x0.astype(f32)).astype(f32), (ww - y0.astype(f32)).astype(f32)
            T = gray[i]
            t00, t01, t10, t11 = T[y0, x0], T[y0, x1], T[y1, x0], T[y1, x1]
            top = fma(ax, (t01 - t00).astype(f32), t00)
            bot = fma(ax, (t11 - t10).astype(f32), t10)
            acc[ok] = (acc[ok] + fma(ay, (bot - top).astype(f32), top)).astype(f32)
            cnt[ok] += 1
        out[s] = np.where(cnt > 0, acc / np.maximum(cnt, 1).astype(f32), f32(0))
    return out


def test_refocus_matches_brute_force(orc_lib):
    pfd = load_pfd()
    w = pfd.make_workload(200, 150, 23.0, 3, seed=4, max_nb=6)
    vds = [1.5, 2.0, 3.3, 7.0, 12.0]
    orc = pfd_oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    for (ow, oh) in [(100, 75), (67, 41)]:
        got = pfd_oracle.refocus(orc, 200, 150, vds, ow, oh)
        ref = brute_force(w.gray.astype(np.float32), w.centers, 200, 150, vds, ow, oh)
        assert np.array_equal(got, ref), f"{np.count_nonzero(got != ref)} pixels differ at {ow}x{oh}"


def test_refocus_constant_micro_images(orc_lib):
    """Constant micro-images render to that constant wherever a lens reaches,
    0 elsewhere; contributions grow with the slice's virtual depth."""
    pfd = load_pfd()
    w = pfd.make_workload(200, 150, 23.0, 3, seed=4, max_nb=6)
    g = np.full_like(w.gray, 100.0, dtype=np.float32)
    orc = pfd_oracle.Oracle(g, w.centers, w.nb_ids, w.nb_counts)
    out = pfd_oracle.refocus(orc, 200, 150, [2.0, 8.0], 100, 75)
    assert set(np.unique(out)) <= {0.0, 100.0}
    assert np.mean(out[1] == 100.0) > np.mean(out[0] == 100.0) > 0.5
    n2 = pfd_oracle.refocus_samples(orc, 200, 150, [2.0], 100, 75)
    n8 = pfd_oracle.refocus_samples(orc, 200, 150, [8.0], 100, 75)
    # about ((m-1) v)^2 / (p^2 sqrt(3)/2) lenses per pixel: 16x from v = 2 to 8 away from the borders
    assert 8 * n2 < n8
