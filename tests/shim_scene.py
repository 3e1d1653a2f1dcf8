"""Reference-style maps for the tests of the C++ classes with the reference's
interface (include/pfd/): a synthetic frame's micro-images as MLA_Problem /
MLA_Info / DisparityAndNormal entries, with the irregularities the reference's
bookkeeping has to handle, and ctypes access to the test driver
tests/csrc/shim_probe.cpp."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROBE = os.path.join(ROOT, "tests", "_build", "libshimprobe.so")

GARBAGE, NEED_MATCH, HAS_INFO, HAS_DN, HAS_GRAY = 1, 2, 4, 8, 16
NORMAL = NEED_MATCH | HAS_INFO | HAS_DN | HAS_GRAY
MATCH_CAP = 16          # AdaptMIPMFrame::m_max_neighbors (AdaptMIPMFrame.cpp:16)

_P = ctypes.c_void_p
_probe = None


def load_probe(pfd):
    """The driver library (built with the engine by build.py)."""
    global _probe
    if _probe is None:
        ctypes.CDLL(pfd.LIB_PATH, mode=ctypes.RTLD_GLOBAL)
        L = ctypes.CDLL(PROBE)
        L.shim_match_layout.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float] + [_P] * 9
        L.shim_check_layout.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float] + [_P] * 9
        L.shim_run.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_float] + [_P] * 7 +
                               [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                ctypes.c_ulonglong] + [_P] * 8)
        L.shim_run_acmm.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_float] + [_P] * 7 +
                                    [ctypes.c_ulonglong] + [_P] * 3)
        for f in (L.shim_match_layout, L.shim_check_layout, L.shim_run, L.shim_run_acmm):
            f.restype = ctypes.c_int
        _probe = L
    return _probe


def _p(a):
    return a.ctypes.data_as(_P)


class Scene:
    """n problems in key order (the maps' order), each with flags, a centre, a
    gray micro-image and a neighbour list of keys (which may name keys that
    are not in the maps)."""

    def __init__(self, keys, centers, gray, flags, nb_lists, mi, pitch, dn_init=None):
        self.keys = np.ascontiguousarray(keys, np.int32)
        self.centers = np.ascontiguousarray(centers, np.float32)
        self.gray = np.ascontiguousarray(gray, np.uint8)
        self.flags = np.ascontiguousarray(flags, np.uint8)
        self.nb_lists = [list(map(tuple, l)) for l in nb_lists]
        self.mi, self.pitch = mi, float(pitch)
        n = self.keys.shape[0]
        self.n = n
        off = [0]
        flat = []
        for l in self.nb_lists:
            flat += l
            off.append(len(flat))
        self.nb_off = np.array(off, np.int32)
        self.nb_keys = np.array(flat if flat else [(0, 0)], np.int32).reshape(-1, 2)
        self.dn_init = (np.zeros((n, mi * mi, 13), np.float32) if dn_init is None
                        else np.ascontiguousarray(dn_init, np.float32))
        order = np.lexsort((self.keys[:, 0], self.keys[:, 1]))
        assert np.array_equal(order, np.arange(n)), "problems must be listed in key order (row, column)"
        self.index = {tuple(k): i for i, k in enumerate(self.keys.tolist())}

    def args(self):
        return [self.n, self.mi, self.pitch, _p(self.keys), _p(self.centers), _p(self.flags), _p(self.gray),
                _p(self.nb_off), _p(self.nb_keys)]

    # ---- the reference's rules, restated -------------------------------------
    def expected_match_layout(self):
        """AdaptMIPMFrame::BuildViewIndexMap (AdaptMIPMFrame.cpp:145-222): views
        are the problems that are not garbage, need matching and have an
        MLA_Info, in map order; a view's neighbours are the first 16 keys of its
        list that are views."""
        views = [i for i in range(self.n)
                 if not self.flags[i] & GARBAGE and self.flags[i] & NEED_MATCH and self.flags[i] & HAS_INFO]
        vset = set(views)
        lists = {}
        for i in views:
            l = []
            for k in self.nb_lists[i]:
                j = self.index.get(k)
                if j is not None and j in vset and len(l) < MATCH_CAP:
                    l.append(j)
            lists[i] = l
        return views, lists

    def expected_check_layout(self):
        """BuildTileInputsFromMaps (MIDisparityFilter.cpp:362-421,
        MICycleCheck.cpp:215-280) as the checks use it: every problem with a
        result, a gray image and an MLA_Info is checked; neighbour k is entry k
        of the full list, usable only when that key has all three itself."""
        ok = [i for i in range(self.n)
              if self.flags[i] & HAS_DN and self.flags[i] & HAS_GRAY and self.flags[i] & HAS_INFO]
        oset = set(ok)
        lists = {}
        for i in ok:
            l = []
            for k in self.nb_lists[i][:32]:
                j = self.index.get(k)
                l.append(j if (j is not None and j in oset and j != i) else -1)
            lists[i] = l
        return ok, lists

    def frame_arrays(self, views, lists, max_nb):
        """Engine-frame arrays (view ids) for a subset of problems."""
        vid = {p: v for v, p in enumerate(views)}
        ids = np.full((len(views), max_nb), -1, np.int32)
        cnt = np.zeros(len(views), np.int32)
        for v, p in enumerate(views):
            l = [vid[j] if j >= 0 else -1 for j in lists[p]]
            ids[v, :len(l)] = l
            cnt[v] = len(l)
        return (np.ascontiguousarray(self.centers[views]), np.ascontiguousarray(self.keys[views]), ids, cnt,
                np.ascontiguousarray(self.gray[views]))


def irregular_scene(pfd, width=300, height=220, pitch=23.0, seed=5, list_len=24):
    """A synthetic frame whose maps carry every case the bookkeeping treats
    specially: garbage lenses, lenses that need no matching (with a result
    from elsewhere), a lens without MLA_Info, one without a gray image, one
    without a result, neighbour keys outside the maps, and lists longer than
    the matcher's 16."""
    w = pfd.make_workload(width, height, pitch, 4, seed=seed, max_nb=6)
    V, mi = w.centers.shape[0], w.mi
    ids, cnt = pfd.neighbors_by_baseline(w.centers, w.tilekeys, pitch, list_len, rings=4)
    keys = [tuple(k) for k in w.tilekeys.tolist()]
    nb_lists = []
    for v in range(V):
        l = [keys[j] for j in ids[v, :cnt[v]]]
        if v % 7 == 3:
            l.insert(2, (-50, -50))           # a key that is not in the maps
        nb_lists.append(l)
    flags = np.full(V, NORMAL, np.uint8)
    rs = np.random.RandomState(seed)
    pick = rs.permutation(V)
    flags[pick[0:4]] = NORMAL | GARBAGE                       # garbage, with a result
    flags[pick[4:6]] = NORMAL & ~NEED_MATCH                   # no matching, with a result
    flags[pick[6]] = NORMAL & ~HAS_INFO                       # no lens information
    flags[pick[7]] = NEED_MATCH | HAS_INFO | HAS_GRAY         # matched, but no result map
    flags[pick[8]] = GARBAGE | HAS_INFO | HAS_DN              # garbage without a gray image
    # results of the lenses nobody matches: invalid, as a fresh map would hold
    dn = np.zeros((V, mi * mi, 13), np.float32)
    dn[:, :, 3] = -1.0
    dn[:, :, 4] = -1.0
    dn[:, :, 5] = 2.0
    return w, Scene(w.tilekeys, w.centers, w.gray, flags, nb_lists, mi, pitch, dn)
