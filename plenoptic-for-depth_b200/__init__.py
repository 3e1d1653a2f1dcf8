"""Python binding of the B200 plenoptic depth engine (libpfd.so).

A thin ctypes layer over include/pfd_abi.h, the way a maintainer of the
reference would bind the C ABI from Python.  Every call goes to the CUDA
library: there is no CPU fallback, and loading fails loudly when the library
has not been built.

    ctx = Context(device=0)
    fid = ctx.frame_upload(raw, centers, tilekeys, mi_w, mi_h, nb_ids, nb_counts)
    ctx.patchmatch(fid, PmParams(...), seed=1)
    plane, cost, disp, sel = ctx.download(fid)
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(PKG_DIR, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libpfd.so")
SYNTH_PATH = os.path.join(BUILD_DIR, "libpfd_synth.so")

PFD_OK = 0
PFD_ETIMEDOUT = -5
SWEEP_SHAPES = 4
SHAPE_AUTOTUNE = -1
FETCH_TEXTURE = 0
FETCH_SHARED = 1
_ERRNAMES = {-1: "PFD_EINVAL", -2: "PFD_ENOMEM", -3: "PFD_ECUDA", -4: "PFD_ENOFRAME",
             -5: "PFD_ETIMEDOUT", -6: "PFD_ENODEV", -7: "PFD_ESTATE"}


class PfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERRNAMES.get(code, code)}: {msg}")
        self.code = code


class PmParamsC(ctypes.Structure):
    _fields_ = [("max_iterations", ctypes.c_int), ("patch_size", ctypes.c_int), ("radius_increment", ctypes.c_int),
                ("top_k", ctypes.c_int), ("sigma_spatial", ctypes.c_float), ("sigma_color", ctypes.c_float),
                ("depth_min", ctypes.c_float), ("depth_max", ctypes.c_float), ("base", ctypes.c_float)]


@dataclass
class PmParams:
    """PatchMatchParamsLF fields of the frame path (LFDepthInfo.h:19-46)."""
    base: float
    max_iterations: int = 3
    patch_size: int = 11
    radius_increment: int = 1
    top_k: int = 5
    sigma_spatial: float = 3.0
    sigma_color: float = 12.0
    depth_min: float = 0.0
    depth_max: float = field(default=-1.0)

    def c(self) -> PmParamsC:
        dmax = self.depth_max if self.depth_max >= 0 else self.base * 0.5
        return PmParamsC(self.max_iterations, self.patch_size, self.radius_increment, self.top_k,
                         self.sigma_spatial, self.sigma_color, self.depth_min, dmax, self.base)


class FilterCfgC(ctypes.Structure):
    _fields_ = [("max_triplet", ctypes.c_int), ("min_valid_disp", ctypes.c_float),
                ("use_selected_views_only", ctypes.c_int), ("clear_selected_views_when_invalid", ctypes.c_int),
                ("enable_cost_filter", ctypes.c_int), ("max_cost", ctypes.c_float),
                ("enable_cycle_geo_filter", ctypes.c_int), ("max_geo_err_px", ctypes.c_float),
                ("enable_cycle_photo_filter", ctypes.c_int), ("max_photo_err_u", ctypes.c_float),
                ("min_good_neighbors", ctypes.c_int), ("enable_spike_filter", ctypes.c_int),
                ("spike_abs_diff", ctypes.c_float), ("spike_min_neighbors", ctypes.c_int)]


@dataclass
class FilterCfg:
    """MIDisparityFilterConfig with the values of MIStereoMatch::FilterAndStatic
    (MIStereoMatch.cpp:759-778)."""
    max_triplet: int = 4
    min_valid_disp: float = 0.0
    use_selected_views_only: bool = True
    clear_selected_views_when_invalid: bool = True
    enable_cost_filter: bool = True
    max_cost: float = 1.8
    enable_cycle_geo_filter: bool = True
    max_geo_err_px: float = 0.5
    enable_cycle_photo_filter: bool = True
    max_photo_err_u: float = 0.5
    min_good_neighbors: int = 2
    enable_spike_filter: bool = True
    spike_abs_diff: float = 1.0
    spike_min_neighbors: int = 3

    def c(self) -> FilterCfgC:
        return FilterCfgC(self.max_triplet, self.min_valid_disp, int(self.use_selected_views_only),
                          int(self.clear_selected_views_when_invalid), int(self.enable_cost_filter), self.max_cost,
                          int(self.enable_cycle_geo_filter), self.max_geo_err_px, int(self.enable_cycle_photo_filter),
                          self.max_photo_err_u, self.min_good_neighbors, int(self.enable_spike_filter),
                          self.spike_abs_diff, self.spike_min_neighbors)


class CycleCfgC(ctypes.Structure):
    _fields_ = [("max_triplet", ctypes.c_int), ("clamp_photo", ctypes.c_int), ("photo_u", ctypes.c_float),
                ("clamp_geo", ctypes.c_int), ("geo_u_px", ctypes.c_float), ("pixel_gate_enabled", ctypes.c_int),
                ("gate_min_good_neighbors", ctypes.c_int), ("gate_geo_px", ctypes.c_float),
                ("gate_photo_u", ctypes.c_float), ("gate_use_clamped", ctypes.c_int),
                ("sobel_thresh", ctypes.c_float), ("var_thresh", ctypes.c_float), ("use_and", ctypes.c_int)]


@dataclass
class CycleCfg:
    """MICycleClampConfig + MICycleMaskParams with the values of the call in
    MIStereoMatch::StereoMatchingForMIA_SoftProxyRepair (MIStereoMatch.cpp:565-583)
    and CheckTile's fixed texture-mask parameters (MICycleCheck.cpp:317-322)."""
    max_triplet: int = 4
    clamp_photo: bool = True
    photo_u: float = 3.0
    clamp_geo: bool = True
    geo_u_px: float = 2.0
    pixel_gate_enabled: bool = False
    gate_min_good_neighbors: int = 2
    gate_geo_px: float = 0.5
    gate_photo_u: float = 0.5
    gate_use_clamped: bool = False
    sobel_thresh: float = 8.0
    var_thresh: float = 60.0
    use_and: bool = True

    def c(self) -> CycleCfgC:
        return CycleCfgC(self.max_triplet, int(self.clamp_photo), self.photo_u, int(self.clamp_geo), self.geo_u_px,
                         int(self.pixel_gate_enabled), self.gate_min_good_neighbors, self.gate_geo_px,
                         self.gate_photo_u, int(self.gate_use_clamped), self.sobel_thresh, self.var_thresh,
                         int(self.use_and))


CYCLE_STATS = ("mean_geo_err_px", "median_geo_err_px", "p90_geo_err_px", "mean_photo_err", "num_samples",
               "rmse_geo_err_px", "rmse_photo_err", "completeness", "completeness_geo", "completeness_photo",
               "completeness_masked_pixels", "completeness_good_pixels", "completeness_good_pixels_geo",
               "completeness_good_pixels_photo", "masked_count", "all_count", "masked_geo_mean",
               "masked_photo_mean", "masked_geo_rmse", "masked_photo_rmse", "coverage",
               "masked_geo_median_approx", "masked_geo_p90_approx", "masked_geo_min", "masked_geo_max")
_CYCLE_INT = {"num_samples", "completeness_masked_pixels", "completeness_good_pixels",
              "completeness_good_pixels_geo", "completeness_good_pixels_photo", "masked_count", "all_count"}


class CycleStatsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong if n in _CYCLE_INT else ctypes.c_double) for n in CYCLE_STATS]


class RequestC(ctypes.Structure):
    _fields_ = [("raw", ctypes.c_void_p), ("W", ctypes.c_int), ("H", ctypes.c_int), ("raw_pitch", ctypes.c_int),
                ("centers", ctypes.c_void_p), ("tilekeys", ctypes.c_void_p), ("n_views", ctypes.c_int),
                ("mi_w", ctypes.c_int), ("mi_h", ctypes.c_int), ("nb_ids", ctypes.c_void_p),
                ("nb_counts", ctypes.c_void_p), ("max_nb", ctypes.c_int), ("params", PmParamsC),
                ("seed", ctypes.c_uint64), ("run_filter", ctypes.c_int), ("filter_cfg", FilterCfgC),
                ("baseline_unit", ctypes.c_float)]


class MlaLensC(ctypes.Structure):
    _fields_ = [("col", ctypes.c_int), ("row", ctypes.c_int), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("area", ctypes.c_float), ("abandon", ctypes.c_int)]


class FuseParamsC(ctypes.Structure):
    _fields_ = [("mla_base", ctypes.c_float), ("min_ref_disp", ctypes.c_float), ("max_reproj_px", ctypes.c_float),
                ("max_rel_vd", ctypes.c_float), ("min_consistent", ctypes.c_int)]


FILTER_STATS = ("total", "valid_in", "kept", "removed", "by_cost", "by_no_support", "by_cycle", "by_spike")

_lib = None
_synth = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


def lib() -> ctypes.CDLL:
    """The engine library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run plenoptic-for-depth_b200/build.py (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "pfd_create": [ctypes.POINTER(_P), _I, ctypes.c_size_t],
            "pfd_destroy": [_P],
            "pfd_last_error": [_P],
            "pfd_stream": [_P],
            "pfd_sync": [_P],
            "pfd_bytes_in_use": [_P],
            "pfd_frame_create": [_P, ctypes.POINTER(_I), _I, _I, _P, _P, _I, _I, _I, _P, _P, _I, _P],
            "pfd_frame_set_raw": [_P, _I, _P, _I],
            "pfd_frame_set_raw_device": [_P, _I, _P, _I],
            "pfd_frame_set_micro_images": [_P, _I, _P],
            "pfd_frame_compute_blur": [_P, _I, _P, _P],
            "pfd_frame_compute_richness": [_P, _I, _P, _P, _P],
            "pfd_set_ncc_moments": [_P, _I],
            "pfd_set_matcher": [_P, _I],
            "pfd_patchmatch_batch": [_P, _P, _I, _P, _P],
            "pfd_read_intrinsics_xml": [ctypes.c_char_p, _P],
            "pfd_read_calib_xml": [ctypes.c_char_p, _P, _I, ctypes.POINTER(_I)],
            "pfd_write_calib_xml": [_P, _P, _I, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)],
            "pfd_acmm_post_refine": [_P, _I, ctypes.POINTER(PmParamsC)],
            "pfd_state_upload": [_P, _I, _P, _P, _P, _P],
            "pfd_frame_upload": [_P, ctypes.POINTER(_I), _P, _I, _I, _I, _P, _P, _I, _I, _I, _P, _P, _I, _P],
            "pfd_frame_free": [_P, _I],
            "pfd_patchmatch": [_P, _I, ctypes.POINTER(PmParamsC), ctypes.c_uint64],
            "pfd_pm_init": [_P, _I, ctypes.POINTER(PmParamsC), ctypes.c_uint64],
            "pfd_pm_sweep": [_P, _I, ctypes.POINTER(PmParamsC), ctypes.c_uint64, _I, _I],
            "pfd_pm_sweep_noalloc": [_P, _I, ctypes.POINTER(PmParamsC), ctypes.c_uint64, _I, _I],
            "pfd_ncc_costs": [_P, _I, ctypes.POINTER(PmParamsC), _P, _P, _P, _I, _P],
            "pfd_download": [_P, _I, _P, _P, _P, _P],
            "pfd_neighbors_by_baseline": [_P, _P, _I, _F, _I, _I, _P, _P],
            "pfd_set_tap_counting": [_P, _I],
            "pfd_read_tap_count": [_P, ctypes.POINTER(ctypes.c_ulonglong)],
            "pfd_filter": [_P, _I, ctypes.POINTER(FilterCfgC), _F, _P, _P],
            "pfd_reprojection_error": [_P, _I, ctypes.POINTER(FilterCfgC), _F, _P],
            "pfd_refocus": [_P, _I, _P, _I, _I, _I, _P],
            "pfd_launch_count": [_P, ctypes.POINTER(ctypes.c_ulonglong)],
            "pfd_vd_to_rd_map": [_P, _P, ctypes.c_size_t, _P, _P],
            "pfd_vd_to_rd_map_device": [_P, _P, ctypes.c_size_t, _P, _P],
            "pfd_vd_to_rd_points": [_P, _P, ctypes.c_size_t, _P, _P],
            "pfd_vd_to_rd_segments": [_P, _P, ctypes.c_size_t, _P, _I, _P],
            "pfd_fit_behavioral_model": [_P, _P, _P, ctypes.c_size_t, _P],
            "pfd_cycle_check": [_P, _I, ctypes.POINTER(CycleCfgC), _F, ctypes.POINTER(CycleStatsC), _P, _P, _P],
            "pfd_cycle_check_stats": [_P, _I, ctypes.POINTER(CycleStatsC)],
            "pfd_mla_lattice_fit": [_P, _P, _I, _I, _P],
            "pfd_download_async": [_P, _I, _P, _P, _P, _P],
            "pfd_server_create": [ctypes.POINTER(_P), _I, ctypes.c_size_t, _I],
            "pfd_server_destroy": [_P],
            "pfd_server_submit": [_P, ctypes.POINTER(RequestC), ctypes.POINTER(ctypes.c_uint64)],
            "pfd_server_wait": [_P, ctypes.c_uint64, _I, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double)],
            "pfd_server_load": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_size_t)],
            "pfd_server_last_error": [_P],
            "pfd_frame_bytes": [_I, _I, _I, _I, _I, _I, _I],
            "pfd_select_neighbors": [_P, _P, _P, _I, _I, _I, _F, _P, _I, _I, _I, _P, _P],
            "pfd_frame_select_neighbors": [_P, _I, _I, _I, _F, _I, _P, _P],
            "pfd_set_sweep_shape": [_P, _I],
            "pfd_set_sweep_fetch": [_P, _I],
            "pfd_set_graphs": [_P, _I],
            "pfd_sweep_shape_info": [_I, _P, _P],
            "pfd_tuned_sweep_shape": [_P, _I, _P, _P],
            "pfd_mla_centers": [_P, _P, _I, _I, _I, _F, _I, _I, _P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)],
            "pfd_fuse_virtual_depth": [_P, _I, ctypes.POINTER(FuseParamsC), _P, _P, _I, _P, _P, _P, _P, _P, _P,
                                       ctypes.POINTER(ctypes.c_longlong)],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _I
        L.pfd_destroy.restype = None
        L.pfd_server_destroy.restype = None
        L.pfd_server_last_error.restype = ctypes.c_char_p
        L.pfd_frame_bytes.restype = ctypes.c_size_t
        L.pfd_last_error.restype = ctypes.c_char_p
        L.pfd_stream.restype = _P
        L.pfd_bytes_in_use.restype = ctypes.c_size_t
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(_P)


def neighbors_by_baseline(centers: np.ndarray, tilekeys: np.ndarray, pitch: float, max_nb: int,
                          rings: int = 5) -> tuple[np.ndarray, np.ndarray]:
    """Ordered matching neighbours per view (see include/pfd_host.h)."""
    c = np.ascontiguousarray(centers, dtype=np.float32)
    k = np.ascontiguousarray(tilekeys, dtype=np.int32)
    n = c.shape[0]
    ids = np.full((n, max_nb), -1, np.int32)
    cnt = np.zeros(n, np.int32)
    rc = lib().pfd_neighbors_by_baseline(_ptr(c), _ptr(k), n, float(pitch), rings, max_nb, _ptr(ids), _ptr(cnt))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_neighbors_by_baseline")
    return ids, cnt


class IntrinsicsC(ctypes.Structure):
    _fields_ = [("D", ctypes.c_float), ("d", ctypes.c_float), ("sensor_rotation", ctypes.c_double * 9),
                ("sensor_translate", ctypes.c_double * 3), ("sensor_pixel_size", ctypes.c_float),
                ("mainlen_focal_length", ctypes.c_float), ("mla_u_size", _I), ("mla_v_size", _I),
                ("baseline", ctypes.c_float), ("distor_depth", ctypes.c_double * 3),
                ("distor_radial", ctypes.c_double * 3), ("distor_tangential", ctypes.c_double * 2),
                ("has_mia", _I)]


MLA_ENTRY = np.dtype([("col", np.int32), ("row", np.int32), ("cx", np.float32), ("cy", np.float32),
                      ("type", np.int32), ("area", np.float32), ("blur_radius", np.float32)])


def read_intrinsics_xml(text: str) -> dict:
    """intrinsics.xml (include/pfd_calib.h) as a dict of its fields."""
    out = IntrinsicsC()
    rc = lib().pfd_read_intrinsics_xml(text.encode(), ctypes.byref(out))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_read_intrinsics_xml")
    d = {}
    for name, _t in IntrinsicsC._fields_:
        v = getattr(out, name)
        d[name] = list(v) if isinstance(v, ctypes.Array) else v
    return d


def read_calib_xml(text: str) -> np.ndarray:
    """CalibInfo.xml lenses in the reference's map order (structured array MLA_ENTRY)."""
    n = _I(0)
    b = text.encode()
    rc = lib().pfd_read_calib_xml(b, None, 0, ctypes.byref(n))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_read_calib_xml")
    out = np.zeros(n.value, MLA_ENTRY)
    rc = lib().pfd_read_calib_xml(b, _ptr(out), n.value, ctypes.byref(n))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_read_calib_xml")
    return out


def write_calib_xml(lenses: np.ndarray, abandon=None) -> str:
    """CalibInfo.xml text of the lenses (structured array MLA_ENTRY)."""
    L = np.ascontiguousarray(lenses, MLA_ENTRY)
    ab = None if abandon is None else np.ascontiguousarray(abandon, np.int32)
    n = ctypes.c_size_t(0)
    rc = lib().pfd_write_calib_xml(_ptr(L), _ptr(ab), len(L), None, 0, ctypes.byref(n))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_write_calib_xml")
    buf = ctypes.create_string_buffer(n.value + 1)
    rc = lib().pfd_write_calib_xml(_ptr(L), _ptr(ab), len(L), buf, n.value + 1, ctypes.byref(n))
    if rc != PFD_OK:
        raise PfdError(rc, "pfd_write_calib_xml")
    return buf.value.decode()


class Context:
    """One engine context (device, stream, frames); see include/pfd_abi.h."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._L = lib()
        h = _P()
        rc = self._L.pfd_create(ctypes.byref(h), device, hbm_budget)
        if rc != PFD_OK:
            raise PfdError(rc, f"pfd_create(device={device})")
        self._h = h
        self._frames: dict[int, dict] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.pfd_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str) -> None:
        if rc != PFD_OK:
            msg = self._L.pfd_last_error(self._h)
            raise PfdError(rc, f"{what}: {msg.decode() if msg else ''}")

    @property
    def stream(self) -> int:
        return self._L.pfd_stream(self._h)

    def sync(self) -> None:
        self._check(self._L.pfd_sync(self._h), "pfd_sync")

    def bytes_in_use(self) -> int:
        return self._L.pfd_bytes_in_use(self._h)

    def frame_create(self, W: int, H: int, centers, tilekeys, mi_w: int, mi_h: int, nb_ids, nb_counts,
                     blur=None) -> int:
        c = np.ascontiguousarray(centers, dtype=np.float32)
        k = np.ascontiguousarray(tilekeys, dtype=np.int32)
        ids = np.ascontiguousarray(nb_ids, dtype=np.int32)
        cnt = np.ascontiguousarray(nb_counts, dtype=np.int32)
        b = None if blur is None else np.ascontiguousarray(blur, dtype=np.uint8)
        fid = _I()
        self._check(self._L.pfd_frame_create(self._h, ctypes.byref(fid), W, H, _ptr(c), _ptr(k), c.shape[0], mi_w,
                                             mi_h, _ptr(ids), _ptr(cnt), ids.shape[1], _ptr(b)), "pfd_frame_create")
        self._frames[fid.value] = dict(V=c.shape[0], mi_w=mi_w, mi_h=mi_h, K=ids.shape[1], W=W, H=H)
        return fid.value

    def frame_set_raw(self, fid: int, raw: np.ndarray) -> None:
        r = np.ascontiguousarray(raw, dtype=np.uint8)
        self._check(self._L.pfd_frame_set_raw(self._h, fid, _ptr(r), r.shape[1]), "pfd_frame_set_raw")

    def frame_set_raw_device(self, fid: int, dev_ptr: int, pitch: int) -> None:
        self._check(self._L.pfd_frame_set_raw_device(self._h, fid, _P(dev_ptr), pitch), "pfd_frame_set_raw_device")

    def frame_set_micro_images(self, fid: int, images: np.ndarray) -> None:
        f = self._frames[fid]
        im = np.ascontiguousarray(images, dtype=np.uint8)
        if im.shape != (f["V"], f["mi_h"], f["mi_w"]):
            raise ValueError(f"micro-images must be {(f['V'], f['mi_h'], f['mi_w'])}, got {im.shape}")
        self._check(self._L.pfd_frame_set_micro_images(self._h, fid, _ptr(im)), "pfd_frame_set_micro_images")

    def frame_compute_blur(self, fid: int, copy_back: bool = True):
        """The blur channel from the frame's raw image, on the device
        (pfd_frame_compute_blur).  Returns (tiles [V][mi_h][mi_w] u8, blureness
        [V] u32) when copy_back, else None without waiting for the device."""
        f = self._frames[fid]
        if not copy_back:
            self._check(self._L.pfd_frame_compute_blur(self._h, fid, None, None), "pfd_frame_compute_blur")
            return None
        tiles = np.zeros((f["V"], f["mi_h"], f["mi_w"]), np.uint8)
        counts = np.zeros(f["V"], np.uint32)
        self._check(self._L.pfd_frame_compute_blur(self._h, fid, _ptr(tiles), _ptr(counts)), "pfd_frame_compute_blur")
        return tiles, counts

    def frame_compute_richness(self, fid: int):
        """The richness channel from the frame's raw image, on the device
        (pfd_frame_compute_richness).  Returns (score [V][mi_h][mi_w] f32, the
        normalised GLCM contrast; binary [V][mi_h][mi_w] u8, 0 or 255; richness
        [V] u32, the 255s of each window)."""
        f = self._frames[fid]
        score = np.zeros((f["V"], f["mi_h"], f["mi_w"]), np.float32)
        binary = np.zeros((f["V"], f["mi_h"], f["mi_w"]), np.uint8)
        counts = np.zeros(f["V"], np.uint32)
        self._check(self._L.pfd_frame_compute_richness(self._h, fid, _ptr(score), _ptr(binary), _ptr(counts)),
                    "pfd_frame_compute_richness")
        return score, binary, counts

    def state_upload(self, fid: int, plane, cost, disp, sel) -> None:
        f = self._frames[fid]
        n = f["V"] * f["mi_w"] * f["mi_h"]
        arrs = [np.ascontiguousarray(plane, np.float32).reshape(n, 4), np.ascontiguousarray(cost, np.float32).reshape(n),
                np.ascontiguousarray(disp, np.float32).reshape(n, 4), np.ascontiguousarray(sel, np.uint32).reshape(n)]
        self._check(self._L.pfd_state_upload(self._h, fid, *[_ptr(a) for a in arrs]), "pfd_state_upload")

    def frame_upload(self, raw, centers, tilekeys, mi_w, mi_h, nb_ids, nb_counts, blur=None) -> int:
        fid = self.frame_create(raw.shape[1], raw.shape[0], centers, tilekeys, mi_w, mi_h, nb_ids, nb_counts, blur)
        try:
            self.frame_set_raw(fid, raw)
        except Exception:
            self.frame_free(fid)
            raise
        return fid

    def frame_free(self, fid: int) -> None:
        self._check(self._L.pfd_frame_free(self._h, fid), "pfd_frame_free")
        self._frames.pop(fid, None)

    def patchmatch(self, fid: int, params: PmParams, seed: int) -> None:
        p = params.c()
        self._check(self._L.pfd_patchmatch(self._h, fid, ctypes.byref(p), seed), "pfd_patchmatch")

    def pm_init(self, fid: int, params: PmParams, seed: int) -> None:
        p = params.c()
        self._check(self._L.pfd_pm_init(self._h, fid, ctypes.byref(p), seed), "pfd_pm_init")

    def pm_sweep(self, fid: int, params: PmParams, seed: int, it: int, phase: int) -> None:
        p = params.c()
        self._check(self._L.pfd_pm_sweep(self._h, fid, ctypes.byref(p), seed, it, phase), "pfd_pm_sweep")

    def pm_sweep_noalloc(self, fid: int, params: PmParams, seed: int, it: int, phase: int) -> None:
        """pfd_pm_sweep on the library's fixed scratch array: for callers that may
        not allocate device memory while frames stream (max_nb <= 30 on B200)."""
        p = params.c()
        self._check(self._L.pfd_pm_sweep_noalloc(self._h, fid, ctypes.byref(p), seed, it, phase),
                    "pfd_pm_sweep_noalloc")

    def ncc_costs(self, fid: int, params: PmParams, vids, pxy, planes) -> np.ndarray:
        v = np.ascontiguousarray(vids, dtype=np.int32)
        xy = np.ascontiguousarray(pxy, dtype=np.int32)
        pl = np.ascontiguousarray(planes, dtype=np.float32)
        K = self._frames[fid]["K"]
        out = np.empty((v.shape[0], K), np.float32)
        p = params.c()
        self._check(self._L.pfd_ncc_costs(self._h, fid, ctypes.byref(p), _ptr(v), _ptr(xy), _ptr(pl), v.shape[0],
                                          _ptr(out)), "pfd_ncc_costs")
        return out

    def set_ncc_moments(self, shifted: bool) -> None:
        """NCC moments of (texel - centre texel) (PFD_NCC_SHIFTED) or the
        reference's raw moments (PFD_NCC_REFERENCE, the default) for the
        context's later initialisations, sweeps and cost queries."""
        self._check(self._L.pfd_set_ncc_moments(self._h, 1 if shifted else 0), "pfd_set_ncc_moments")

    def patchmatch_batch(self, fids, params, seeds) -> None:
        """pfd_patchmatch of several frames, one launch per half-sweep over all of them."""
        ids = np.ascontiguousarray(fids, np.int32)
        arr = (PmParamsC * len(ids))(*[p.c() for p in params])
        sd = np.ascontiguousarray(seeds, np.uint64)
        self._check(self._L.pfd_patchmatch_batch(self._h, _ptr(ids), len(ids), ctypes.cast(arr, _P), _ptr(sd)),
                    "pfd_patchmatch_batch")

    def set_graphs(self, on: bool) -> None:
        """Replay pfd_patchmatch and enqueue-only filter calls from CUDA graphs
        (captured on the second call with the same arguments)."""
        self._check(self._L.pfd_set_graphs(self._h, 1 if on else 0), "pfd_set_graphs")

    def set_sweep_shape(self, shape: int) -> None:
        """Launch shape of later half-sweeps: 0 .. SWEEP_SHAPES - 1, or
        SHAPE_AUTOTUNE (-1) for the engine's autotuner."""
        self._check(self._L.pfd_set_sweep_shape(self._h, int(shape)), "pfd_set_sweep_shape")

    def set_sweep_fetch(self, mode: int) -> None:
        """Where later half-sweeps read neighbour samples: FETCH_SHARED (1,
        the default: tiles staged in shared memory) or FETCH_TEXTURE (0: the
        frame's layered textures, created at its first sweep in this mode).
        Both give the same state bit for bit."""
        self._check(self._L.pfd_set_sweep_fetch(self._h, int(mode)), "pfd_set_sweep_fetch")

    def tuned_sweep_shape(self, fid: int, params: "PmParams") -> int:
        """The autotuner's shape for the frame's key, or -1 if not tuned yet."""
        out = _I(-1)
        p = params.c()
        self._check(self._L.pfd_tuned_sweep_shape(self._h, fid, ctypes.byref(p), ctypes.byref(out)),
                    "pfd_tuned_sweep_shape")
        return out.value

    def set_matcher(self, acmm: bool) -> None:
        """PatchMatch rules of the context's later calls: the ACMM matcher at one
        pyramid level (PFD_MATCHER_ACMM) or the Frame matcher (the default)."""
        self._check(self._L.pfd_set_matcher(self._h, 1 if acmm else 0), "pfd_set_matcher")

    def acmm_post_refine(self, fid: int, params: "PmParams") -> None:
        p = params.c()
        self._check(self._L.pfd_acmm_post_refine(self._h, fid, ctypes.byref(p)), "pfd_acmm_post_refine")

    def set_tap_counting(self, on: bool) -> None:
        self._check(self._L.pfd_set_tap_counting(self._h, 1 if on else 0), "pfd_set_tap_counting")

    def read_tap_count(self) -> int:
        v = ctypes.c_ulonglong()
        self._check(self._L.pfd_read_tap_count(self._h, ctypes.byref(v)), "pfd_read_tap_count")
        return v.value

    def filter(self, fid: int, cfg: FilterCfg, baseline_unit: float, download: bool = True):
        """MIDisparityFilterCPU::FilterGlobal on the frame's state, in place.
        Returns (reason map [V*mi*mi] uint8, stats dict); with download=False
        nothing is copied back (no stream synchronisation) and None is returned."""
        c = cfg.c()
        if not download:
            self._check(self._L.pfd_filter(self._h, fid, ctypes.byref(c), float(baseline_unit), None, None),
                        "pfd_filter")
            return None
        f = self._frames[fid]
        reason = np.empty(f["V"] * f["mi_w"] * f["mi_h"], np.uint8)
        stats = np.zeros(8, np.int64)
        self._check(self._L.pfd_filter(self._h, fid, ctypes.byref(c), float(baseline_unit), _ptr(reason), _ptr(stats)),
                    "pfd_filter")
        return reason, dict(zip(FILTER_STATS, (int(x) for x in stats)))

    def cycle_check(self, fid: int, cfg: CycleCfg, baseline_unit: float, maps: bool = True, stats: bool = True):
        """MICycleCheckerCPU::CheckGlobal on the frame's state (read-only).
        Returns (stats dict, geo_err, pho_err, texture mask); maps are None
        unless maps=True.  With maps and stats False the check is only
        enqueued and None is returned; cycle_check_stats() folds it later."""
        f = self._frames[fid]
        if not maps and not stats:
            c = cfg.c()
            self._check(self._L.pfd_cycle_check(self._h, fid, ctypes.byref(c), float(baseline_unit), None, None, None,
                                                None), "pfd_cycle_check")
            return None
        n = f["V"] * f["mi_w"] * f["mi_h"]
        geo = np.empty(n, np.float32) if maps else None
        pho = np.empty(n, np.float32) if maps else None
        tm = np.empty(n, np.uint8) if maps else None
        out = CycleStatsC()
        c = cfg.c()
        self._check(self._L.pfd_cycle_check(self._h, fid, ctypes.byref(c), float(baseline_unit), ctypes.byref(out),
                                            _ptr(geo) if maps else None, _ptr(pho) if maps else None,
                                            _ptr(tm) if maps else None), "pfd_cycle_check")
        return {k: getattr(out, k) for k in CYCLE_STATS}, geo, pho, tm

    def cycle_check_stats(self, fid: int) -> dict:
        out = CycleStatsC()
        self._check(self._L.pfd_cycle_check_stats(self._h, fid, ctypes.byref(out)), "pfd_cycle_check_stats")
        return {k: getattr(out, k) for k in CYCLE_STATS}

    def vd_to_rd_map(self, vd, c) -> np.ndarray:
        """VirtualToRealDepthFunc::convertVirtualToRealDepth on the device (FP64)."""
        v = np.ascontiguousarray(vd, dtype=np.float32)
        out = np.empty(v.shape, np.float64)
        cc = np.ascontiguousarray(c, dtype=np.float64)
        self._check(self._L.pfd_vd_to_rd_map(self._h, _ptr(v), v.size, _ptr(cc), _ptr(out)), "pfd_vd_to_rd_map")
        return out

    def vd_to_rd_map_device(self, vd_ptr: int, n: int, c, rd_ptr: int) -> None:
        cc = np.ascontiguousarray(c, dtype=np.float64)
        self._check(self._L.pfd_vd_to_rd_map_device(self._h, _P(vd_ptr), n, _ptr(cc), _P(rd_ptr)),
                    "pfd_vd_to_rd_map_device")

    def vd_to_rd_points(self, vd, c) -> np.ndarray:
        """LFRefocus::ConvertVdToRd per value on the device."""
        v = np.ascontiguousarray(vd, dtype=np.float32)
        out = np.empty(v.shape, np.float32)
        cc = np.ascontiguousarray(c, dtype=np.float64)
        self._check(self._L.pfd_vd_to_rd_points(self._h, _ptr(v), v.size, _ptr(cc), _ptr(out)), "pfd_vd_to_rd_points")
        return out

    def vd_to_rd_segments(self, vd, segs) -> np.ndarray:
        """LFRefocus::ConvertVdToRdSegment; segs [n][5] (depth_min, depth_max, c0, c1, c2)."""
        v = np.ascontiguousarray(vd, dtype=np.float32)
        sg = np.ascontiguousarray(segs, dtype=np.float64).reshape(-1, 5)
        out = np.empty(v.shape, np.float32)
        self._check(self._L.pfd_vd_to_rd_segments(self._h, _ptr(v), v.size, _ptr(sg), sg.shape[0], _ptr(out)),
                    "pfd_vd_to_rd_segments")
        return out

    def fit_behavioral_model(self, real_depth, vd) -> np.ndarray:
        """VirtualToRealDepthFunc::BehavioralModel: (c0, c1, c2)."""
        r = np.ascontiguousarray(real_depth, dtype=np.float32)
        v = np.ascontiguousarray(vd, dtype=np.float32)
        c = np.zeros(3, np.float64)
        self._check(self._L.pfd_fit_behavioral_model(self._h, _ptr(r), _ptr(v), r.size, _ptr(c)),
                    "pfd_fit_behavioral_model")
        return c

    def launch_count(self) -> int:
        n = ctypes.c_ulonglong()
        self._check(self._L.pfd_launch_count(self._h, ctypes.byref(n)), "pfd_launch_count")
        return int(n.value)

    def refocus(self, fid: int, slice_vd, out_w: int, out_h: int, download: bool = True):
        """Focal stack [n_slices][out_h][out_w] of the frame (pfd_refocus); with
        download=False the stack stays on the device and None is returned."""
        vd = np.ascontiguousarray(slice_vd, dtype=np.float32)
        out = np.empty((vd.shape[0], out_h, out_w), np.float32) if download else None
        self._check(self._L.pfd_refocus(self._h, fid, _ptr(vd), vd.shape[0], out_w, out_h,
                                        _ptr(out) if download else None), "pfd_refocus")
        return out

    def reprojection_error(self, fid: int, cfg: FilterCfg, baseline_unit: float, download: bool = True):
        c = cfg.c()
        if not download:
            self._check(self._L.pfd_reprojection_error(self._h, fid, ctypes.byref(c), float(baseline_unit), None),
                        "pfd_reprojection_error")
            return None
        f = self._frames[fid]
        err = np.empty(f["V"] * f["mi_w"] * f["mi_h"], np.float32)
        self._check(self._L.pfd_reprojection_error(self._h, fid, ctypes.byref(c), float(baseline_unit), _ptr(err)),
                    "pfd_reprojection_error")
        return err

    def select_neighbors(self, centers, tilekeys, mla_u_size: int, mla_v_size: int, pitch: float, images,
                         max_nb: int = 128):
        """SelectNeighbors::CollectMIANeighImagesForMatch with the device
        similarities: (nb_ids [V][max_nb], nb_counts [V])."""
        c = np.ascontiguousarray(centers, np.float32)
        k = np.ascontiguousarray(tilekeys, np.int32)
        im = np.ascontiguousarray(images, np.uint8)
        V = c.shape[0]
        ids = np.full((V, max_nb), -1, np.int32)
        cnt = np.zeros(V, np.int32)
        self._check(self._L.pfd_select_neighbors(self._h, _ptr(c), _ptr(k), V, mla_u_size, mla_v_size, float(pitch),
                                                 _ptr(im), im.shape[2], im.shape[1], max_nb, _ptr(ids), _ptr(cnt)),
                    "pfd_select_neighbors")
        return ids, cnt

    def frame_select_neighbors(self, fid: int, mla_u_size: int, mla_v_size: int, pitch: float,
                               max_list: int | None = None):
        """The selection on the frame's own micro-images; the first max_nb of
        each list become the frame's matching lists (the PatchMatch state must
        be initialised again).  With max_list, returns the full lists
        (nb_ids [V][max_list], nb_counts [V]); otherwise None."""
        f = self._frames[fid]
        if max_list is None:
            self._check(self._L.pfd_frame_select_neighbors(self._h, fid, mla_u_size, mla_v_size, float(pitch), 0,
                                                           None, None), "pfd_frame_select_neighbors")
            return None
        ids = np.full((f["V"], max_list), -1, np.int32)
        cnt = np.zeros(f["V"], np.int32)
        self._check(self._L.pfd_frame_select_neighbors(self._h, fid, mla_u_size, mla_v_size, float(pitch), max_list,
                                                       _ptr(ids), _ptr(cnt)), "pfd_frame_select_neighbors")
        return ids, cnt

    def mla_centers(self, white, baseline: float, mla_u_size: int, mla_v_size: int):
        """DepthSolver::ComputeMLACentersFromWhiteImage on a white image (H x W x 3
        BGR, or H x W gray).  Returns (dict of col, row, cx, cy, area, abandon
        arrays in key order, Otsu threshold)."""
        img = np.ascontiguousarray(white, np.uint8)
        if img.ndim == 2:
            img = np.ascontiguousarray(np.repeat(img[:, :, None], 3, axis=2))
        H, W = img.shape[:2]
        n = _I(0)
        t = _I(0)
        self._check(self._L.pfd_mla_centers(self._h, _ptr(img), W, H, img.strides[0], float(baseline), mla_u_size,
                                            mla_v_size, None, 0, ctypes.byref(n), ctypes.byref(t)), "pfd_mla_centers")
        out = (MlaLensC * max(1, n.value))()
        self._check(self._L.pfd_mla_centers(self._h, _ptr(img), W, H, img.strides[0], float(baseline), mla_u_size,
                                            mla_v_size, ctypes.cast(out, _P), n.value, ctypes.byref(n),
                                            ctypes.byref(t)), "pfd_mla_centers")
        a = np.ctypeslib.as_array(out)[:n.value]
        return {k: np.array(a[k]) for k in ("col", "row", "cx", "cy", "area", "abandon")}, t.value

    def mla_lattice_fit(self, lenses: dict, skip_abandoned: bool = True) -> dict:
        """Hexagonal lattice through the centres of mla_centers()."""
        n = len(lenses["col"])
        arr = (MlaLensC * n)()
        for i in range(n):
            arr[i] = MlaLensC(int(lenses["col"][i]), int(lenses["row"][i]), float(lenses["cx"][i]),
                              float(lenses["cy"][i]), float(lenses["area"][i]), int(lenses["abandon"][i]))
        fit = np.zeros(6, np.float64)
        self._check(self._L.pfd_mla_lattice_fit(self._h, ctypes.cast(arr, _P), n, int(skip_abandoned), _ptr(fit)),
                    "pfd_mla_lattice_fit")
        return dict(origin=(fit[0], fit[1]), pitch=fit[2], angle=fit[3], rms=fit[4], used=int(fit[5]))

    def fuse_virtual_depth(self, fid: int, lists, list_counts, is_ref, mla_base: float, bgr=None,
                           points: bool = True, download: bool = True, min_ref_disp: float = 1.0,
                           max_reproj_px: float = 1.0, max_rel_vd: float = 0.05, min_consistent: int = 2):
        """LFRefocus::FuseVirtualDepth_BackProject on the frame's state.  Returns
        (vd_map, conf, aif [H][W][3], points [n][9] or None); with download=False
        nothing is copied back and None is returned."""
        f = self._frames[fid]
        ls = np.ascontiguousarray(lists, np.int32)
        lc = np.ascontiguousarray(list_counts, np.int32)
        ir = np.ascontiguousarray(is_ref, np.uint8)
        b = None if bgr is None else np.ascontiguousarray(bgr, np.uint8)
        prm = FuseParamsC(mla_base, min_ref_disp, max_reproj_px, max_rel_vd, min_consistent)
        if not download:
            self._check(self._L.pfd_fuse_virtual_depth(self._h, fid, ctypes.byref(prm), _ptr(ls), _ptr(lc),
                                                       ls.shape[1], _ptr(ir), _ptr(b), None, None, None, None, None),
                        "pfd_fuse_virtual_depth")
            return None
        H, W = f["H"], f["W"]
        vd = np.empty((H, W), np.float32)
        cf = np.empty((H, W), np.uint8)
        aif = np.empty((H, W, 3), np.uint8)
        n = ctypes.c_longlong(0)
        pts = np.empty((f["V"] * f["mi_w"] * f["mi_h"], 9), np.float32) if points else None
        self._check(self._L.pfd_fuse_virtual_depth(self._h, fid, ctypes.byref(prm), _ptr(ls), _ptr(lc), ls.shape[1],
                                                   _ptr(ir), _ptr(b), _ptr(vd), _ptr(cf), _ptr(aif), _ptr(pts),
                                                   ctypes.byref(n)), "pfd_fuse_virtual_depth")
        return vd, cf, aif, (pts[:n.value] if points else None)

    def download(self, fid: int):
        f = self._frames[fid]
        n = f["V"] * f["mi_w"] * f["mi_h"]
        plane = np.empty((n, 4), np.float32)
        cost = np.empty(n, np.float32)
        disp = np.empty((n, 4), np.float32)
        sel = np.empty(n, np.uint32)
        self._check(self._L.pfd_download(self._h, fid, _ptr(plane), _ptr(cost), _ptr(disp), _ptr(sel)), "pfd_download")
        return plane, cost, disp, sel


class Server:
    """The request loop of include/pfd_serve.h: frames of any size and pitch,
    matched concurrently in `slots` slots inside an HBM budget."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, slots: int = 4):
        self._L = lib()
        h = _P()
        rc = self._L.pfd_server_create(ctypes.byref(h), device, hbm_budget, slots)
        if rc != PFD_OK:
            raise PfdError(rc, "pfd_server_create")
        self._h = h
        self._pending = {}

    def close(self) -> None:
        if self._h:
            self._L.pfd_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, w, params: PmParams, seed: int, filter_cfg: FilterCfg | None = None,
               baseline_unit: float = 0.0) -> int:
        """Queues workload w (make_workload) with its own iteration count in params."""
        raw = np.ascontiguousarray(w.frame.raw, np.uint8)
        c = np.ascontiguousarray(w.centers, np.float32)
        k = np.ascontiguousarray(w.tilekeys, np.int32)
        ids = np.ascontiguousarray(w.nb_ids, np.int32)
        cnt = np.ascontiguousarray(w.nb_counts, np.int32)
        fc = (filter_cfg or FilterCfg()).c()
        req = RequestC(_ptr(raw), raw.shape[1], raw.shape[0], raw.shape[1], _ptr(c), _ptr(k), c.shape[0], w.mi, w.mi,
                       _ptr(ids), _ptr(cnt), ids.shape[1], params.c(), seed, 1 if filter_cfg is not None else 0, fc,
                       float(baseline_unit))
        t = ctypes.c_uint64()
        rc = self._L.pfd_server_submit(self._h, ctypes.byref(req), ctypes.byref(t))
        if rc != PFD_OK:
            raise PfdError(rc, "pfd_server_submit: " + self._L.pfd_server_last_error(self._h).decode())
        self._pending[t.value] = c.shape[0] * w.mi * w.mi
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1):
        """(plane, cost, disp, sel, latency_ms), or None on timeout."""
        n = self._pending[ticket]
        plane = np.empty((n, 4), np.float32)
        cost = np.empty(n, np.float32)
        disp = np.empty((n, 4), np.float32)
        sel = np.empty(n, np.uint32)
        lat = ctypes.c_double()
        rc = self._L.pfd_server_wait(self._h, ticket, timeout_ms, _ptr(plane), _ptr(cost), _ptr(disp), _ptr(sel),
                                     ctypes.byref(lat))
        if rc == PFD_ETIMEDOUT:
            return None
        del self._pending[ticket]
        if rc != PFD_OK:
            raise PfdError(rc, "pfd_server_wait: " + self._L.pfd_server_last_error(self._h).decode())
        return plane, cost, disp, sel, lat.value

    def load(self):
        q, r, b = _I(), _I(), ctypes.c_size_t()
        self._L.pfd_server_load(self._h, ctypes.byref(q), ctypes.byref(r), ctypes.byref(b))
        return q.value, r.value, b.value


def frame_bytes(W: int, H: int, n_views: int, mi: int, max_nb: int) -> int:
    return int(lib().pfd_frame_bytes(W, H, n_views, mi, mi, max_nb, 0))


# ---------------------------------------------------------------------------
# synthetic frames
# ---------------------------------------------------------------------------
class SynthConfigC(ctypes.Structure):
    _fields_ = [("width", _I), ("height", _I), ("pitch", _F), ("n_planes", _I), ("vd_min", _F), ("vd_max", _F),
                ("noise_sigma", _F), ("n_lens_types", _I), ("blur_sigma", _F * 3), ("texture_cell", _F),
                ("seed", ctypes.c_uint64)]


def sweep_shape_info(shape: int) -> tuple:
    """(warps per CTA, CTAs per SM) of a sweep launch shape."""
    w, c = _I(), _I()
    if lib().pfd_sweep_shape_info(int(shape), ctypes.byref(w), ctypes.byref(c)) != 0:
        raise ValueError(f"no sweep shape {shape}")
    return w.value, c.value


def synth_lib() -> ctypes.CDLL:
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} is missing: run plenoptic-for-depth_b200/build.py")
        S = ctypes.CDLL(SYNTH_PATH)
        S.pfd_synth_count.argtypes = [ctypes.POINTER(SynthConfigC), ctypes.POINTER(_I), ctypes.POINTER(_I),
                                      ctypes.POINTER(_I)]
        S.pfd_synth_render.argtypes = [ctypes.POINTER(SynthConfigC), _P, _P, _P, _P, _P]
        S.pfd_synth_vd_map.argtypes = [ctypes.POINTER(SynthConfigC), _P]
        _synth = S
    return _synth


@dataclass
class SynthFrame:
    raw: np.ndarray          # [H][W] uint8
    centers: np.ndarray      # [L][2] float32
    tilekeys: np.ndarray     # [L][2] int32 (column, row)
    types: np.ndarray        # [L] int32
    vd_center: np.ndarray    # [L] float32
    pitch: float
    n_cols: int
    n_rows: int
    config: tuple = ()       # the generator's arguments, for synth_vd_map


def synth_frame(width: int, height: int, pitch: float, n_planes: int, seed: int, vd_min: float = 2.0,
                vd_max: float = 12.0, noise_sigma: float = 2.0, n_lens_types: int = 1,
                blur_sigma=(0.0, 0.0, 0.0), texture_cell: float = 0.0) -> SynthFrame:
    """Seeded synthetic plenoptic raw frame (csrc/synth.c)."""
    cfg = SynthConfigC(width, height, pitch, n_planes, vd_min, vd_max, noise_sigma, n_lens_types,
                       (_F * 3)(*blur_sigma), texture_cell, seed)
    S = synth_lib()
    n, nc, nr = _I(), _I(), _I()
    if S.pfd_synth_count(ctypes.byref(cfg), ctypes.byref(n), ctypes.byref(nc), ctypes.byref(nr)) != 0:
        raise ValueError("bad synthetic frame configuration")
    raw = np.empty((height, width), np.uint8)
    cen = np.empty((n.value, 2), np.float32)
    keys = np.empty((n.value, 2), np.int32)
    types = np.empty(n.value, np.int32)
    vd = np.empty(n.value, np.float32)
    if S.pfd_synth_render(ctypes.byref(cfg), _ptr(raw), _ptr(cen), _ptr(keys), _ptr(types), _ptr(vd)) != 0:
        raise ValueError("synthetic rendering failed")
    return SynthFrame(raw, cen, keys, types, vd, pitch, nc.value, nr.value,
                      (width, height, pitch, n_planes, vd_min, vd_max, noise_sigma, n_lens_types, tuple(blur_sigma),
                       texture_cell, seed))


def synth_vd_map(frame: SynthFrame) -> np.ndarray:
    """Ground-truth virtual depth of every raw pixel of a synthetic frame
    ([H][W] float32; 0 outside the lens circles): the depth of the scene point
    the pixel shows."""
    (width, height, pitch, n_planes, vd_min, vd_max, noise_sigma, n_lens_types, blur_sigma, texture_cell,
     seed) = frame.config
    cfg = SynthConfigC(width, height, pitch, n_planes, vd_min, vd_max, noise_sigma, n_lens_types,
                       (_F * 3)(*blur_sigma), texture_cell, seed)
    out = np.empty((height, width), np.float32)
    if synth_lib().pfd_synth_vd_map(ctypes.byref(cfg), _ptr(out)) != 0:
        raise ValueError("bad synthetic frame configuration")
    return out


def depth_error(w: "Workload", plane: np.ndarray, vd_map: np.ndarray | None = None, cost: np.ndarray | None = None):
    """Matched virtual depth (pitch / disparity, disparity = plane.w) of every
    micro-image pixel against the scene's true virtual depth at that raw pixel.
    Pixels count as matched when the disparity is > 0.05 (and the cost < 2 when
    given).  Returns the fraction matched and, over them, the median absolute
    and relative error and the fractions within 0.05, 0.5 and 1 virtual-depth
    units."""
    if vd_map is None:
        vd_map = synth_vd_map(w.frame)
    mi = w.mi
    o = window_origins(w.centers, mi).astype(np.int64)
    ys, xs = np.mgrid[0:mi, 0:mi]
    gt = vd_map[o[:, 1, None, None] + ys[None], o[:, 0, None, None] + xs[None]].reshape(-1)
    d = plane[:, 3].astype(np.float64)
    ok = (d > 0.05) & (gt > 0)
    if cost is not None:
        ok &= cost < 2.0
    est = w.frame.pitch / np.maximum(d, 1e-6)
    err = np.abs(est - gt)[ok]
    rel = err / gt[ok]
    if err.size == 0:
        return {"matched": 0.0}
    return {"matched": float(ok.mean()), "median_abs": float(np.median(err)), "median_rel": float(np.median(rel)),
            "within_0.05": float(np.mean(err <= 0.05)), "within_0.5": float(np.mean(err <= 0.5)),
            "within_1": float(np.mean(err <= 1.0))}


def mi_window(pitch: float) -> int:
    """mi_width_for_match = floor(pitch * 0.707106781186) (Common/Common.cpp:34-38)."""
    return int(pitch * 0.707106781186)


def window_origins(centers: np.ndarray, mi: int) -> np.ndarray:
    """trunc(c - (mi - 1) / 2) as DepthSolver.cpp:1894-1895 and cv::Rect compute it."""
    c = np.asarray(centers, np.float32).astype(np.float64)
    o = (c - (mi - 1) * 0.5).astype(np.float32)
    return np.trunc(o).astype(np.int32)


def valid_views(frame: SynthFrame, mi: int) -> np.ndarray:
    """Indices of lenses whose matching window lies inside the frame
    (the abandon test of DepthSolver::CreateProblemsAndDisNormals_Frame, :1893-1903)."""
    H, W = frame.raw.shape
    c = frame.centers.astype(np.float64)
    lo = (c - (mi - 1) * 0.5).astype(np.float32)
    o = np.trunc(lo).astype(np.int64)
    ok = (lo[:, 0] >= 0) & (lo[:, 1] >= 0) & (o[:, 0] + mi <= W) & (o[:, 1] + mi <= H)
    return np.nonzero(ok)[0]


def slice_views(raw: np.ndarray, centers: np.ndarray, mi: int) -> np.ndarray:
    """Host slicing of the micro-image windows, [V][mi][mi] uint8."""
    o = window_origins(centers, mi)
    out = np.empty((o.shape[0], mi, mi), np.uint8)
    for v, (x, y) in enumerate(o):
        out[v] = raw[y:y + mi, x:x + mi]
    return out


@dataclass
class Workload:
    """A frame ready for matching: valid views, their windows, neighbour lists."""
    frame: SynthFrame
    mi: int
    centers: np.ndarray
    tilekeys: np.ndarray
    nb_ids: np.ndarray
    nb_counts: np.ndarray
    gray: np.ndarray         # [V][mi][mi] uint8 (host slice, for the oracle)


def make_workload(width: int, height: int, pitch: float, n_planes: int, seed: int, max_nb: int, **kw) -> Workload:
    fr = synth_frame(width, height, pitch, n_planes, seed, **kw)
    mi = mi_window(pitch)
    keep = valid_views(fr, mi)
    centers = np.ascontiguousarray(fr.centers[keep])
    keys = np.ascontiguousarray(fr.tilekeys[keep])
    ids, cnt = neighbors_by_baseline(centers, keys, pitch, max_nb)
    return Workload(fr, mi, centers, keys, ids, cnt, slice_views(fr.raw, centers, mi))
