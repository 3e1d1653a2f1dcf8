"""The virtual-depth fusion oracle (LFRefocus::FuseVirtualDepth_BackProject,
FocalStack/LFRefocus.cpp:1553-1794) against an independent pure-Python
restatement of the same lines on small scenes, and known answers on a row of
lenses seeing a fronto-parallel plane, where every consistent point is the
same virtual point and the masks decide which micro-image pixels fuse."""
import math

import numpy as np
import pytest

import pfd_oracle

F = np.float32
INVALID = F(-9999.0)


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def _i_trunc(x):
    x = float(x)
    return int(x) if abs(x) < 2147483648.0 else -2147483648


def _i_round(x):
    x = float(x)
    if not abs(x) < 2147483648.0:
        return -2147483648
    return int(np.rint(x))              # round half to even, as cvRound


def _vd(mla_base, d):
    if float(d) <= 0:
        return INVALID
    return F(float(mla_base) / float(d))   # float base over a double disparity


def _v3(vd, c, r, mi, cen):
    cm = F(F(mi - 1) * F(0.5)) + F(1)
    return [F(F(F(c) - cm) * vd) + cen[0], F(F(F(r) - cm) * vd) + cen[1], vd]


def _bp(P, cen, mi):
    cm = F(F(mi - 1) * F(0.5)) + F(1)
    return [F((P[0] - cen[0]) / P[2]) + cm, F((P[1] - cen[1]) / P[2]) + cm]


def brute_fuse(gray, centers, plane, lists, is_ref, W, H, mla_base):
    """Lines 1610-1789, statement by statement, in float32."""
    V, mi = gray.shape[0], gray.shape[1]
    ppv = mi * mi
    mask = np.zeros((V, ppv), np.uint8)
    vd_map = np.zeros((H, W), F)
    conf = np.zeros((H, W), np.uint8)
    aif = np.zeros((H, W, 3), np.uint8)
    pts = []
    pl = plane.reshape(V, ppv, 4)
    for v in range(V):
        if not is_ref[v]:
            continue
        cen = centers[v]
        for r in range(mi):
            for c in range(mi):
                idx = r * mi + c
                if mask[v, idx] == 1:
                    continue
                d_ref = pl[v, idx, 3]
                if d_ref < F(1.0):
                    continue
                vd_ref = _vd(mla_base, d_ref)
                if abs(vd_ref - INVALID) < F(1e-6) or not np.isfinite(vd_ref):
                    continue
                normal = [pl[v, idx, 0], pl[v, idx, 1], pl[v, idx, 2]]
                P = _v3(vd_ref, c, r, mi, cen)
                point = list(P)
                color = [F(gray[v, r, c])] * 3
                used = {}
                for j, u in enumerate(lists[v]):
                    if u < 0:
                        continue
                    q = _bp(P, centers[u], mi)
                    sr, sc = _i_trunc(q[1] + F(0.5)), _i_trunc(q[0] + F(0.5))
                    if sc < 0 or sc >= mi or sr < 0 or sr >= mi:
                        continue
                    si = sr * mi + sc
                    if mask[u, si] == 1:
                        continue
                    d_src = pl[u, si, 3]
                    if d_src <= F(0):
                        continue
                    vd_src = _vd(mla_base, d_src)
                    if abs(vd_src - INVALID) < F(1e-6) or not np.isfinite(vd_src):
                        continue
                    Ps = _v3(vd_src, sc, sr, mi, centers[u])
                    rq = _bp(Ps, cen, mi)
                    ex, ey = F(F(c) - rq[0]), F(F(r) - rq[1])
                    err = F(math.sqrt(float(F(F(ex * ex) + F(ey * ey)))))
                    rel = F(abs(vd_src - vd_ref) / max(vd_ref, F(1e-6)))
                    if err < F(1.0) and rel < F(0.05):
                        point = [F(a + b) for a, b in zip(point, Ps)]
                        normal = [F(a + b) for a, b in zip(normal, pl[u, si, :3])]
                        color = [F(a + F(gray[u, sr, sc])) for a in color]
                        used[j] = (u, si)
                if len(used) < 2:
                    continue
                ia = F(F(1.0) / F(F(len(used)) + F(1.0)))
                point = [F(a * ia) for a in point]
                normal = [F(a * ia) for a in normal]
                color = [F(a * ia) for a in color]
                vx, vy = _i_round(point[0]), _i_round(point[1])
                if 0 <= vy < H and 0 <= vx < W:
                    vd_map[vy, vx] = point[2]
                    conf[vy, vx] = min(255, (len(used) + 1) * 60)
                    aif[vy, vx] = [min(255, max(0, _i_round(x))) for x in color]
                    pts.append(point + normal + color)
                for u, si in used.values():
                    mask[u, si] = 1
    return vd_map, conf, aif, np.array(pts, F).reshape(-1, 9)


def _line_scene(n=5, mi=8, spacing=20.0, d=2.0):
    gray = np.stack([(np.arange(mi * mi).reshape(mi, mi) * 3 + 17 * v) % 251 for v in range(n)]).astype(np.float32)
    centers = np.array([[100 + spacing * v, 60] for v in range(n)], np.float32)
    lists = np.array([[u for u in range(n) if u != v] for v in range(n)], np.int32)
    plane = np.zeros((n * mi * mi, 4), np.float32)
    plane[:, 2] = 1.0
    plane[:, 3] = d
    return gray, centers, lists, plane


def _run_oracle(orc_lib, gray, centers, lists, plane, is_ref, W, H, mla_base):
    V = gray.shape[0]
    orc = orc_lib.Oracle(gray, centers, np.full((V, 1), -1, np.int32), np.zeros(V, np.int32))
    return orc_lib.fuse_virtual_depth(orc, plane, lists, np.full(V, lists.shape[1], np.int32), is_ref, W, H, mla_base)


def test_line_of_lenses_known_answer(orc_lib):
    """mla_base 20, d 2: virtual depth 10, neighbour k lenses away sees pixel c
    at c - 2k (view order to the right), so every fused point is the pixel's
    own virtual point and lands on an integer raw position."""
    gray, centers, lists, plane = _line_scene()
    n, mi = 5, 8
    vd, cf, aif, pts = _run_oracle(orc_lib, gray, centers, lists, plane, np.ones(n, np.uint8), 240, 120, 20.0)
    assert len(pts) > 0
    assert np.all(pts[:, 2] == 10.0) and np.all(pts[:, 3:6] == [0, 0, 1])
    assert np.all(vd[vd != 0] == 10.0)
    # view 0 is processed first: pixel c needs two neighbours in bounds, c - 2 >= 0 and c - 4 >= 0
    cm = (mi - 1) * 0.5 + 1
    first = [(r, c) for r in range(mi) for c in range(mi) if c >= 4]
    for r, c in first:
        x, y = int((c - cm) * 10 + 100), int((r - cm) * 10 + 60)
        assert vd[y, x] == 10.0
    ref = brute_fuse(gray.reshape(n, mi, mi), centers, plane, lists, np.ones(n, np.uint8), 240, 120, 20.0)
    for a, b in zip((vd, cf, aif, pts), ref):
        assert np.array_equal(a, b)


def test_masks_are_order_dependent(orc_lib):
    """Reversing the view order changes which pixels fuse (masks set by the
    earlier views), so the sequential order is part of the result."""
    gray, centers, lists, plane = _line_scene()
    n = 5
    a = _run_oracle(orc_lib, gray, centers, lists, plane, np.ones(n, np.uint8), 240, 120, 20.0)
    perm = np.arange(n)[::-1]
    inv = np.argsort(perm)
    b = _run_oracle(orc_lib, gray[perm], centers[perm], inv[lists[perm]].astype(np.int32),
                    plane.reshape(n, -1, 4)[perm].reshape(-1, 4), np.ones(n, np.uint8), 240, 120, 20.0)
    assert len(a[3]) != len(b[3]) or not np.array_equal(a[3], b[3])


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_brute_force_on_noisy_scenes(orc_lib, seed):
    """Hex-ish lens grid, disparities around a plane with noise, invalid
    pixels, garbage (non-reference) lenses and foreign list entries."""
    rs = np.random.RandomState(seed)
    mi, cols, rows = 8, 5, 4
    centers, keys = [], []
    for r in range(rows):
        for c in range(cols):
            centers.append((30 + 11.0 * c + (5.5 if r % 2 else 0.0), 30 + 9.5 * r))
    centers = np.array(centers, np.float32)
    V = len(centers)
    gray = rs.randint(0, 256, size=(V, mi, mi)).astype(np.float32)
    d = (np.float32(2.2) + rs.normal(0, 0.03, size=(V, mi * mi))).astype(np.float32)
    d[rs.rand(V, mi * mi) < 0.1] = -1.0
    d[rs.rand(V, mi * mi) < 0.05] = 0.5
    plane = np.zeros((V * mi * mi, 4), np.float32)
    plane[:, 0:3] = rs.normal(0, 0.1, size=(V * mi * mi, 3)).astype(np.float32)
    plane[:, 3] = d.ravel()
    dist = np.linalg.norm(centers[:, None] - centers[None], axis=2)
    L = 10
    lists = np.full((V, L), -1, np.int32)
    for v in range(V):
        order = [u for u in np.argsort(dist[v], kind="stable") if u != v][:L]
        lists[v, :len(order)] = order
        if v % 4 == 1:
            lists[v, 3] = -1                      # a key that has no result map
    is_ref = (rs.rand(V) > 0.15).astype(np.uint8)
    W, H = 110, 80
    mla = 14.0
    got = _run_oracle(orc_lib, gray, centers, lists, plane, is_ref, W, H, mla)
    ref = brute_fuse(gray, centers, plane, lists, is_ref, W, H, mla)
    assert len(ref[3]) > 20, "too few fused points for a meaningful comparison"
    for name, a, b in zip(("vd", "conf", "aif", "points"), got, ref):
        assert np.array_equal(a, b), name
