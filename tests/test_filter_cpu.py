"""Known answers of the disparity-filter oracle (MIDisparityFilterCPU::FilterGlobal
and ComputeTileReprojectionErrorMap, CheckModule/MIDisparityFilter.cpp) on hand-built
micro-image rows whose outcome follows from the reference's rules by hand:

* three views on a horizontal line, spacing = baseline unit = 20 px, so a pixel
  p of view v with disparity d projects to p + (c_v - c_u)/|c_v - c_u| * d in
  view u (MIDisparityFilter.cpp:562-571) and back with u's disparity;
* gray = 10 x + 3 y + 5 in every view: on this ramp the 3x3-normalised photo
  residual is 0 when p and q are integers with 3x3 windows inside the image,
  and |I_q - I_p| = 10 |dx| otherwise (ComputePhotoResidual, :138-156).
"""
import numpy as np
import pytest

import pfd_oracle
from conftest import load_pfd

N = 12                      # micro-image side
SPACING = 20.0
PR_KEEP, PR_COST, PR_NOSUPPORT, PR_CYCLE, PR_SPIKE = 0, 80, 140, 200, 255
TOTAL, VALID_IN, KEPT, REMOVED, BY_COST, BY_NOSUPPORT, BY_CYCLE, BY_SPIKE = range(8)


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def line_scene(d=2.0, V=3):
    xs, ys = np.meshgrid(np.arange(N, dtype=np.float32), np.arange(N, dtype=np.float32))
    gray = np.repeat((10 * xs + 3 * ys + 5)[None], V, 0)
    centers = np.array([[100 + SPACING * v, 100] for v in range(V)], np.float32)
    nb_ids = np.full((V, 2), -1, np.int32)
    nb_counts = np.zeros(V, np.int32)
    for v in range(V):
        lst = [u for u in (v - 1, v + 1) if 0 <= u < V]
        nb_ids[v, :len(lst)] = lst
        nb_counts[v] = len(lst)
    n = V * N * N
    sel = np.zeros(n, np.uint32)
    for v in range(V):
        sel[v * N * N:(v + 1) * N * N] = (1 << nb_counts[v]) - 1
    state = dict(plane=np.zeros((n, 4), np.float32), cost=np.full(n, 0.5, np.float32),
                 disp=np.zeros((n, 4), np.float32), sel=sel)
    state["plane"][:, 2] = 1.0
    state["plane"][:, 3] = d
    state["disp"][:, 0] = d
    return pfd_oracle.Oracle(gray, centers, nb_ids, nb_counts), state


def cfg(**kw):
    return load_pfd().FilterCfg(**kw)


def view(a, v):
    return a.reshape(-1, N, N)[v]


def test_consistent_row_geometry_only(orc_lib):
    """Geometric cycle only, one good neighbour needed: a pixel keeps iff one
    projection lands inside a neighbour whose four bilinear corners are still
    valid when the view is processed (views run in map order, in place)."""
    orc, st = line_scene()
    reason, stats = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_photo_filter=False,
                                                      enable_spike_filter=False), SPACING, st)
    x = np.arange(N)[None, :].repeat(N, 0)
    # view 0 projects to x - 2 in view 1: needs x >= 2
    assert np.array_equal(view(reason, 0), np.where(x >= 2, PR_KEEP, PR_NOSUPPORT))
    # view 1: x + 2 in view 0 (columns 0, 1 of view 0 now invalid -> corners at x+2 >= 2 fine) or x - 2 in view 2
    assert np.all(view(reason, 1) == PR_KEEP)
    # view 2: x + 2 in view 1 (all kept): needs x + 2 <= 11
    assert np.array_equal(view(reason, 2), np.where(x <= 9, PR_KEEP, PR_NOSUPPORT))
    assert stats[TOTAL] == 3 * N * N and stats[VALID_IN] == 3 * N * N
    assert stats[REMOVED] == stats[BY_NOSUPPORT] == 2 * 2 * N
    assert stats[KEPT] + stats[REMOVED] == stats[VALID_IN]


def test_order_dependence_through_invalidated_corners(orc_lib):
    """View 1 reads view 0 after view 0 was filtered: a projection whose
    bilinear footprint touches an invalidated pixel (d = -1) has no support."""
    orc, st = line_scene()
    # view 0 keeps only x >= 2; view 2 is switched off for view 1 (sel bit 1 cleared)
    v1 = slice(N * N, 2 * N * N)
    st["sel"][v1] = 1
    reason, _ = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_photo_filter=False,
                                                  enable_spike_filter=False), SPACING, st)
    x = np.arange(N)[None, :].repeat(N, 0)
    # view 1 pixel x projects to x + 2 of view 0: inside for x <= 9; corners x+2, x+3 (clamped) all >= 2 valid
    assert np.array_equal(view(reason, 1), np.where(x <= 9, PR_KEEP, PR_NOSUPPORT))
    # now run with view 0 fully invalid beforehand except x >= 6
    orc, st = line_scene()
    st["sel"][v1] = 1
    st["plane"][:N * N, 3] = np.where(x.ravel() >= 6, 2.0, -1.0)
    reason, _ = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_photo_filter=False,
                                                  enable_spike_filter=False), SPACING, st)
    # view 0 pixel x >= 6 projects to x - 2 >= 4 of view 1: all kept; x < 6 is not valid input (untouched)
    assert np.all(view(reason, 0)[:, 6:] == PR_KEEP)
    assert np.all(view(reason, 0)[:, :6] == PR_KEEP)          # invalid input keeps the default reason
    assert np.array_equal(view(reason, 1), np.where((x + 2 >= 6) & (x <= 9), PR_KEEP, PR_NOSUPPORT))


def test_cost_nosupport_cycle_and_invalidation(orc_lib):
    orc, st = line_scene()
    i_cost = N * N + 5 * N + 5            # view 1, (5, 5)
    i_nosel = N * N + 6 * N + 5           # view 1, (5, 6)
    st["cost"][i_cost] = 1.9
    st["sel"][i_nosel] = 0
    # view 2 disagrees: disparity 3 -> geometric cycle error |(x-2) + 3 - x| = 1 > 0.5
    st["plane"][2 * N * N:, 3] = 3.0
    # view 0 disagrees too, so view 1 has no good neighbour anywhere
    st["plane"][:N * N, 3] = 3.0
    reason, stats = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_photo_filter=False,
                                                      enable_spike_filter=False), SPACING, st)
    r1 = view(reason, 1)
    assert r1[5, 5] == PR_COST and r1[6, 5] == PR_NOSUPPORT
    # view 0 (processed first) fails its cycle everywhere and is invalidated, so
    # view 1 finds support only in view 2, at x - 2 >= 0.  The neighbour's cost
    # is interpolated (:455-476, :572-580): at the integer projection (x-3, y)
    # only that texel weighs, so only view-0 pixel (8, 5) sees cost 1.9 > 1.8.
    x = np.arange(N)[None, :].repeat(N, 0)
    y = np.arange(N)[:, None].repeat(N, 1)
    touches = (x == 8) & (y == 5)
    exp0 = np.where((x < 3) | touches, PR_NOSUPPORT, PR_CYCLE)
    assert np.array_equal(view(reason, 0), exp0)
    others = np.ones((N, N), bool)
    others[5, 5] = others[6, 5] = False
    assert np.all(r1[others & (x >= 2)] == PR_CYCLE)
    assert np.all(r1[others & (x < 2)] == PR_NOSUPPORT)
    # InvalidatePixel (MIDisparityFilter.cpp:158-174)
    for i in (i_cost, i_nosel, N * N):
        assert np.array_equal(st["plane"][i], [0, 0, 0, -1])
        assert st["cost"][i] == 2.0
        assert np.array_equal(st["disp"][i], [-1, -1, 0, 0])
        assert st["sel"][i] == 0
    assert stats[BY_COST] == 1
    assert stats[REMOVED] == stats[BY_COST] + stats[BY_NOSUPPORT] + stats[BY_CYCLE] + stats[BY_SPIKE]


def test_photo_residual_on_a_ramp(orc_lib):
    """Normalised residual 0 where both 3x3 windows fit, raw |dI| = 20 otherwise."""
    orc, st = line_scene()
    reason, _ = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_geo_filter=False,
                                                  enable_spike_filter=False), SPACING, st)
    x = np.arange(N)[None, :].repeat(N, 0)
    y = np.arange(N)[:, None].repeat(N, 1)
    inner_p = (x >= 1) & (x <= N - 2) & (y >= 1) & (y <= N - 2)
    # view 0: q = x - 2 must be inside and windowed: 3 <= x <= 10
    exp0 = np.where(x < 2, PR_NOSUPPORT, np.where(inner_p & (x >= 3), PR_KEEP, PR_CYCLE))
    assert np.array_equal(view(reason, 0), exp0)


def test_spike(orc_lib):
    orc, st = line_scene()
    i = N * N + 4 * N + 4
    st["plane"][i, 3] = 4.0
    reason, stats = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_geo_filter=False,
                                                      enable_cycle_photo_filter=False), SPACING, st)
    assert view(reason, 1)[4, 4] == PR_SPIKE
    assert stats[BY_SPIKE] >= 1
    assert st["plane"][i, 3] == -1.0
    # a pixel with fewer than spike_min_neighbors kept neighbours is not judged
    orc, st = line_scene()
    st["plane"][i, 3] = 4.0
    reason, _ = pfd_oracle.filter_global(orc, cfg(min_good_neighbors=1, enable_cycle_geo_filter=False,
                                                  enable_cycle_photo_filter=False, spike_min_neighbors=9),
                                         SPACING, st)
    assert view(reason, 1)[4, 4] == PR_KEEP


def test_reprojection_error_map(orc_lib):
    orc, st = line_scene()
    st["plane"][2 * N * N:, 3] = 3.0
    err = pfd_oracle.reprojection_error(orc, cfg(min_good_neighbors=1), SPACING, st)
    e1 = view(err, 1)
    # view 1: neighbour 0 (d 2) closes exactly; neighbour 2 (d 3) misses by 1; median of the two = 0.5
    x = np.arange(N)
    both = (x + 2 <= N - 1) & (x - 2 >= 0)
    assert np.allclose(e1[:, both], 0.5)
    assert np.all(e1[:, (x - 2 < 0)] == 0.0)        # only view 0 reachable
    assert np.all(e1[:, (x + 2 > N - 1)] == 1.0)    # only view 2 reachable
    # min_good_neighbors 2: single-neighbour pixels have no error value
    err2 = pfd_oracle.reprojection_error(orc, cfg(min_good_neighbors=2), SPACING, st)
    assert np.all(view(err2, 0) == -1.0)
