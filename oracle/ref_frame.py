"""ctypes binding of the reference's own frame PatchMatch kernels, compiled
from the reference tree by oracle/ref/Makefile into oracle/_ref/.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's baseline legs,
never by the product.  Two builds of the same kernels:
  * libref_frame.so        cuRAND XORWOW as the reference uses it (a fixed
                           seed in place of clock64()): the timed plain method
  * libref_frame_philox.so the kernels drawing the engine's Philox streams, so
                           a run follows the same random numbers as the
                           engine and the CPU oracle
  * libref_frame_ieee.so   the Philox build without --use_fast_math: the
                           reference's own sensitivity to its arithmetic

    ref = RefFrame(workload, philox=True)
    costs = ref.ncc_costs(params, vids, pxy, planes)
    ref.patchmatch(params, seed)
    plane, cost, disp, sel = ref.download()
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
LIB_XORWOW = os.path.join(REF_DIR, "libref_frame.so")
LIB_PHILOX = os.path.join(REF_DIR, "libref_frame_philox.so")
LIB_IEEE = os.path.join(REF_DIR, "libref_frame_ieee.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


class RefParams(ctypes.Structure):
    _fields_ = [("max_iterations", _I), ("patch_size", _I), ("radius_increment", _I), ("top_k", _I),
                ("sigma_spatial", _F), ("sigma_color", _F), ("depth_min", _F), ("depth_max", _F), ("base", _F)]


def available() -> bool:
    return all(os.path.exists(p) for p in (LIB_XORWOW, LIB_PHILOX, LIB_IEEE))


def build(reference_tree: str = "/root/reference") -> bool:
    """make -C oracle/ref when the reference tree is present (this container);
    elsewhere the prebuilt libraries are used.  Returns whether all exist."""
    if os.path.isdir(reference_tree):
        r = subprocess.run(["make", "-s", "-C", os.path.join(ORACLE_DIR, "ref"), "REF=" + reference_tree],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference kernel build failed:\n" + r.stdout + r.stderr)
    return available()


_libs: dict = {}


def lib(philox: bool, ieee: bool = False) -> ctypes.CDLL:
    path = LIB_IEEE if ieee else (LIB_PHILOX if philox else LIB_XORWOW)
    if path not in _libs:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with make -C oracle/ref (needs the reference tree)")
        L = ctypes.CDLL(path)
        L.pfdref_last_error.restype = ctypes.c_char_p
        L.pfdref_frame_create.argtypes = [ctypes.POINTER(_P), _I, _I, _P, _P, _P, _P, _P, _P, _I]
        L.pfdref_frame_destroy.argtypes = [_P]
        L.pfdref_ncc_costs.argtypes = [_P, ctypes.POINTER(RefParams), _P, _P, _P, _I, _P]
        L.pfdref_patchmatch.argtypes = [_P, ctypes.POINTER(RefParams), ctypes.c_uint64, _P]
        L.pfdref_patchmatch_sample.argtypes = [_P, ctypes.POINTER(RefParams), ctypes.c_uint64, _I, _P]
        L.pfdref_init.argtypes = [_P, ctypes.POINTER(RefParams), ctypes.c_uint64]
        L.pfdref_sweep.argtypes = [_P, ctypes.POINTER(RefParams), ctypes.c_uint64, _I, _I]
        L.pfdref_download.argtypes = [_P, _P, _P, _P, _P]
        L.pfdref_state_upload.argtypes = [_P, _P, _P, _P, _P]
        _libs[path] = L
    return _libs[path]


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def to_params(p) -> RefParams:
    """From the engine binding's PmParams (same fields, same meaning)."""
    c = p.c()
    return RefParams(c.max_iterations, c.patch_size, c.radius_increment, c.top_k, c.sigma_spatial, c.sigma_color,
                     c.depth_min, c.depth_max, c.base)


class RefFrame:
    """One frame bound to the reference's textures and state buffers."""

    def __init__(self, w, philox: bool = True, blur: np.ndarray | None = None, ieee: bool = False):
        self.L = lib(philox, ieee)
        self.V = int(w.centers.shape[0])
        self.mi = int(w.mi)
        self.max_nb = int(w.nb_ids.shape[1])
        self._keep = [np.ascontiguousarray(w.gray, np.uint8), None if blur is None else np.ascontiguousarray(blur, np.uint8),
                      np.ascontiguousarray(w.centers, np.float32), np.ascontiguousarray(w.tilekeys, np.int32),
                      np.ascontiguousarray(w.nb_ids, np.int32), np.ascontiguousarray(w.nb_counts, np.int32)]
        h = _P()
        g, b, c, k, ids, cnt = self._keep
        self._check(self.L.pfdref_frame_create(ctypes.byref(h), self.V, self.mi, _ptr(g), _ptr(b), _ptr(c), _ptr(k),
                                               _ptr(ids), _ptr(cnt), self.max_nb), "pfdref_frame_create")
        self.h = h

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {rc}: {self.L.pfdref_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.pfdref_frame_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def ncc_costs(self, params, vids, pxy, planes) -> np.ndarray:
        vids = np.ascontiguousarray(vids, np.int32)
        pxy = np.ascontiguousarray(pxy, np.int32)
        planes = np.ascontiguousarray(planes, np.float32)
        n = vids.shape[0]
        out = np.empty((n, self.max_nb), np.float32)
        P = to_params(params)
        self._check(self.L.pfdref_ncc_costs(self.h, ctypes.byref(P), _ptr(vids), _ptr(pxy), _ptr(planes), n, _ptr(out)),
                    "pfdref_ncc_costs")
        return out

    def patchmatch(self, params, seed: int):
        """The reference's RunPatchMatchCUDAForFrame_Impl; returns (init ms, sweeps ms)."""
        ms = np.zeros(2, np.float32)
        P = to_params(params)
        self._check(self.L.pfdref_patchmatch(self.h, ctypes.byref(P), seed, _ptr(ms)), "pfdref_patchmatch")
        return float(ms[0]), float(ms[1])

    def patchmatch_sample(self, params, seed: int, n: int):
        """The reference's run on views [0, n) only (every view initialised
        first, untimed); returns (init ms, sweeps ms) of the sample."""
        ms = np.zeros(2, np.float32)
        P = to_params(params)
        self._check(self.L.pfdref_patchmatch_sample(self.h, ctypes.byref(P), seed, n, _ptr(ms)),
                    "pfdref_patchmatch_sample")
        return float(ms[0]), float(ms[1])

    def init(self, params, seed: int):
        P = to_params(params)
        self._check(self.L.pfdref_init(self.h, ctypes.byref(P), seed), "pfdref_init")

    def sweep(self, params, seed: int, it: int, phase: int):
        P = to_params(params)
        self._check(self.L.pfdref_sweep(self.h, ctypes.byref(P), seed, it, phase), "pfdref_sweep")

    def download(self):
        px = self.V * self.mi * self.mi
        plane = np.empty((px, 4), np.float32)
        cost = np.empty(px, np.float32)
        disp = np.empty((px, 4), np.float32)
        sel = np.empty(px, np.uint32)
        self._check(self.L.pfdref_download(self.h, _ptr(plane), _ptr(cost), _ptr(disp), _ptr(sel)), "pfdref_download")
        return plane, cost, disp, sel

    def state_upload(self, plane, cost, disp, sel):
        arrs = [np.ascontiguousarray(plane, np.float32), np.ascontiguousarray(cost, np.float32),
                np.ascontiguousarray(disp, np.float32), np.ascontiguousarray(sel, np.uint32)]
        self._check(self.L.pfdref_state_upload(self.h, *[_ptr(a) for a in arrs]), "pfdref_state_upload")
