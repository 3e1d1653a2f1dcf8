"""The C ABI library on a machine without a GPU: it loads, exports every
declared entry point, fails cleanly, and its host-side helpers work."""
import ctypes
import os
import re

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pfd_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(pfd):
    L = ctypes.CDLL(pfd.LIB_PATH)
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            names += _declared(h)
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_create_without_device_fails_cleanly(pfd):
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    rc = pfd.lib().pfd_create(ctypes.byref(h), 0, 0)
    assert rc == -6 and not h.value          # PFD_ENODEV, no context
    pfd.lib().pfd_destroy(None)             # safe on NULL


def test_hex_ring_neighbours(pfd):
    """Interior lenses of a hexagonal array: 6 neighbours at one pitch, then 6
    at sqrt(3) pitch, then 6 at two pitches, nearest first."""
    fr = pfd.synth_frame(600, 500, 23.0, 2, seed=1)
    ids, cnt = pfd.neighbors_by_baseline(fr.centers, fr.tilekeys, 23.0, 18)
    c = fr.centers.astype(np.float64)
    interior = [v for v in range(len(c)) if 80 < c[v, 0] < 520 and 80 < c[v, 1] < 420]
    assert len(interior) > 50
    for v in interior:
        assert cnt[v] == 18
        b = np.linalg.norm(c[ids[v]] - c[v], axis=1)
        assert np.all(np.abs(b[:6] - 23.0) < 0.01)
        assert np.all(np.abs(b[6:12] - 23.0 * np.sqrt(3)) < 0.01)
        assert np.all(np.abs(b[12:18] - 46.0) < 0.01)
        assert np.all(np.diff(b) > -1e-3)


def test_synthetic_frame_is_deterministic(pfd):
    a = pfd.synth_frame(320, 240, 23.2, 5, seed=9, n_lens_types=3, blur_sigma=(0.6, 1.0, 1.4))
    b = pfd.synth_frame(320, 240, 23.2, 5, seed=9, n_lens_types=3, blur_sigma=(0.6, 1.0, 1.4))
    assert np.array_equal(a.raw, b.raw) and np.array_equal(a.centers, b.centers)
    assert set(np.unique(a.types)) == {0, 1, 2}
    assert 2.0 <= a.vd_center.min() and a.vd_center.max() <= 12.0
    assert a.raw.mean() > 40
