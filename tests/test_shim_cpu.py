"""Bookkeeping of the C++ classes with the reference's interface (include/pfd/),
which needs no device: which micro-images AdaptMIPMFrame matches and with which
neighbour lists (AdaptMIPMFrame::BuildViewIndexMap, AdaptMIPMFrame.cpp:145-222),
and which ones the consistency pass checks against which neighbours
(BuildTileInputsFromMaps, MIDisparityFilter.cpp:362-421).  The selected-view
bit k of a result names entry k of the matcher's list, so these lists must be
exactly the reference's."""
import numpy as np

from shim_scene import GARBAGE, HAS_DN, HAS_GRAY, HAS_INFO, NEED_MATCH, NORMAL, Scene, irregular_scene, load_probe


def _layout(L, fn, scene, width):
    view_of = np.full(scene.n, -7, np.int32)
    nb = np.full((scene.n, width), -7, np.int32)
    cnt = np.full(scene.n, -7, np.int32)
    nv = fn(*scene.args(), view_of.ctypes.data_as(L.shim_run.argtypes[3]),
            nb.ctypes.data_as(L.shim_run.argtypes[3]), cnt.ctypes.data_as(L.shim_run.argtypes[3]))
    return nv, view_of, nb, cnt


def test_match_layout_follows_the_reference(pfd):
    L = load_probe(pfd)
    _, sc = irregular_scene(pfd)
    nv, view_of, nb, cnt = _layout(L, L.shim_match_layout, sc, 16)
    views, lists = sc.expected_match_layout()
    assert nv == len(views)
    assert [i for i in range(sc.n) if view_of[i] >= 0] == views
    assert np.array_equal(view_of[views], np.arange(len(views)))
    long_lists = 0
    for p in views:
        l = lists[p]
        assert cnt[p] == len(l)
        assert list(nb[p, :len(l)]) == l and np.all(nb[p, len(l):] == -1)
        long_lists += len(l) == 16
    assert long_lists > 10, "the scene must exercise the 16-neighbour cap"
    # garbage, no-matching and info-less lenses are not views, and never neighbours
    skipped = [i for i in range(sc.n) if sc.flags[i] & GARBAGE or not sc.flags[i] & NEED_MATCH
               or not sc.flags[i] & HAS_INFO]
    assert len(skipped) >= 8 and not set(skipped) & set(views)
    assert not set(skipped) & set(nb[views].ravel().tolist())


def test_check_layout_follows_the_reference(pfd):
    L = load_probe(pfd)
    _, sc = irregular_scene(pfd)
    nv, view_of, nb, cnt = _layout(L, L.shim_check_layout, sc, 32)
    views, lists = sc.expected_check_layout()
    assert nv == len(views)
    assert [i for i in range(sc.n) if view_of[i] >= 0] == views
    holes = 0
    for p in views:
        l = lists[p]
        assert cnt[p] == len(l)
        assert list(nb[p, :len(l)]) == l and np.all(nb[p, len(l):] == -1)
        holes += l.count(-1)
    assert holes > 5, "some listed neighbours must be unusable"
    # garbage lenses with a result are checked (the checks ignore the flags)
    assert any(sc.flags[p] & GARBAGE for p in views)


def test_check_layout_cuts_lists_at_32_and_drops_self(pfd):
    """Selected-view masks have 32 bits, so entries past 32 can never be
    named; a lens listed as its own neighbour has a zero baseline, which every
    check skips, so it becomes an unusable entry."""
    L = load_probe(pfd)
    mi, n = 16, 40
    keys = np.array([(c, 0) for c in range(n)], np.int32)
    centers = np.array([(20.0 + 23.0 * c, 20.0) for c in range(n)], np.float32)
    gray = np.zeros((n, mi, mi), np.uint8)
    lists = [[(c, 0) for c in range(n) if c != v] for v in range(n)]
    lists[0] = [(0, 0)] + lists[0]
    sc = Scene(keys, centers, gray, np.full(n, NORMAL, np.uint8), lists, mi, 23.0)
    nv, view_of, nb, cnt = _layout(L, L.shim_check_layout, sc, 32)
    assert nv == n and np.all(cnt == 32)
    assert nb[0, 0] == -1 and list(nb[0, 1:]) == list(range(1, 32))
    assert list(nb[5, :]) == [c for c in range(n) if c != 5][:32]


def test_empty_maps(pfd):
    L = load_probe(pfd)
    mi = 16
    sc = Scene(np.array([(0, 0)], np.int32), np.array([(20.0, 20.0)], np.float32), np.zeros((1, mi, mi), np.uint8),
               np.array([GARBAGE | HAS_INFO | HAS_GRAY], np.uint8), [[]], mi, 23.0)
    nv, _, _, _ = _layout(L, L.shim_match_layout, sc, 16)
    assert nv == -1                      # Initialize fails: no valid micro-images
    nv, view_of, _, _ = _layout(L, L.shim_check_layout, sc, 32)
    assert nv == 0 and view_of[0] == -1  # the checks check nothing


def test_acmm_class_refuses_two_level_windows(pfd):
    """AdaptMIPMFrameACMM counts its pyramid levels as BuildBlurAlignedPyramids
    does (AdaptMIPMFrameACMM.cpp:312-321): a 24-pixel window (pitch 34) takes
    two, which is not built, so Initialize fails before any device work."""
    import ctypes
    L = load_probe(pfd)
    w, sc = irregular_scene(pfd, width=420, height=320, pitch=34.0)
    assert sc.mi == 24
    n, ppv = sc.n, sc.mi * sc.mi
    dn = np.zeros((n, ppv, 13), np.float32)
    levels = ctypes.c_int(0)
    msg = ctypes.create_string_buffer(256)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.shim_run_acmm(*sc.args(), p(sc.dn_init), 1, p(dn), ctypes.byref(levels), msg)
    assert rc == -1 and levels.value == 2
    assert b"two-level" in msg.value
