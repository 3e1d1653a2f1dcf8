"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
baseline legs of bench.py, never by the product.  What pins it (the
reference's own kernels for the PatchMatch, OpenCV and known answers for the
host-side stages): see oracle/pfd_oracle.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


class OrcFrame(ctypes.Structure):
    _fields_ = [("n_views", _I), ("mi_w", _I), ("mi_h", _I), ("max_nb", _I), ("gray", _P), ("blur", _P),
                ("centers", _P), ("nb_ids", _P), ("nb_counts", _P)]


class OrcParams(ctypes.Structure):
    _fields_ = [("max_iterations", _I), ("patch_size", _I), ("radius_increment", _I), ("top_k", _I),
                ("sigma_spatial", _F), ("sigma_color", _F), ("depth_min", _F), ("depth_max", _F), ("base", _F),
                ("shifted", _I), ("acmm", _I)]


class OrcFilterCfg(ctypes.Structure):
    _fields_ = [("max_triplet", _I), ("min_valid_disp", _F), ("use_selected_views_only", _I),
                ("clear_selected_views_when_invalid", _I), ("enable_cost_filter", _I), ("max_cost", _F),
                ("enable_cycle_geo_filter", _I), ("max_geo_err_px", _F), ("enable_cycle_photo_filter", _I),
                ("max_photo_err_u", _F), ("min_good_neighbors", _I), ("enable_spike_filter", _I),
                ("spike_abs_diff", _F), ("spike_min_neighbors", _I)]


class OrcCycleCfg(ctypes.Structure):
    _fields_ = [("max_triplet", _I), ("clamp_photo", _I), ("photo_u", _F), ("clamp_geo", _I), ("geo_u_px", _F),
                ("pixel_gate_enabled", _I), ("gate_min_good_neighbors", _I), ("gate_geo_px", _F),
                ("gate_photo_u", _F), ("gate_use_clamped", _I), ("sobel_thresh", _F), ("var_thresh", _F),
                ("use_and", _I)]


CYCLE_STAT_FIELDS = ["mean_geo_err_px", "median_geo_err_px", "p90_geo_err_px", "mean_photo_err", "num_samples",
                     "rmse_geo_err_px", "rmse_photo_err", "completeness", "completeness_geo", "completeness_photo",
                     "completeness_masked_pixels", "completeness_good_pixels", "completeness_good_pixels_geo",
                     "completeness_good_pixels_photo", "masked_count", "all_count", "masked_geo_mean",
                     "masked_photo_mean", "masked_geo_rmse", "masked_photo_rmse", "coverage",
                     "masked_geo_median_approx", "masked_geo_p90_approx", "masked_geo_min", "masked_geo_max"]
_INT_STATS = {"num_samples", "completeness_masked_pixels", "completeness_good_pixels", "completeness_good_pixels_geo",
              "completeness_good_pixels_photo", "masked_count", "all_count"}


class OrcCycleStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_longlong if n in _INT_STATS else ctypes.c_double) for n in CYCLE_STAT_FIELDS]


class OrcFuseParams(ctypes.Structure):
    _fields_ = [("mla_base", _F), ("min_ref_disp", _F), ("max_reproj_px", _F), ("max_rel_vd", _F),
                ("min_consistent", _I)]


class OrcState(ctypes.Structure):
    _fields_ = [("plane", _P), ("cost", _P), ("disp", _P), ("sel", _P)]


def build() -> str:
    """make -C oracle (gcc, -ffp-contract=off)."""
    r = subprocess.run(["make", "-s", "-C", ORACLE_DIR], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        FP, PP, SP = ctypes.POINTER(OrcFrame), ctypes.POINTER(OrcParams), ctypes.POINTER(OrcState)
        L.orc_cost_vectors.argtypes = [FP, PP, _P, _P, _P, _I, _P, _P]
        L.orc_count_taps.argtypes = [FP, PP, _P, _P, _P, _I]
        L.orc_count_taps.restype = ctypes.c_longlong
        L.orc_ncc_fp64.argtypes = [FP, PP, _I, _I, _I, _I, _P]
        L.orc_ncc_fp64.restype = ctypes.c_double
        L.orc_ncc_fp64_batch.argtypes = [FP, PP, _P, _P, _P, _I, _I, _I, _P]
        L.orc_pm_init.argtypes = [FP, PP, ctypes.c_uint64, SP, _I]
        L.orc_pm_init_views.argtypes = [FP, PP, ctypes.c_uint64, SP, _I, _I, _I]
        L.orc_pm_sweep.argtypes = [FP, PP, ctypes.c_uint64, _I, _I, SP, SP, _I]
        L.orc_pm_sweep_views.argtypes = [FP, PP, ctypes.c_uint64, _I, _I, SP, SP, _I, _I, _I]
        L.orc_pm_sweep_views_taps.argtypes = [FP, PP, ctypes.c_uint64, _I, _I, SP, SP, _I, _I, _I]
        L.orc_pm_sweep_views_taps.restype = ctypes.c_longlong
        L.orc_patchmatch.argtypes = [FP, PP, ctypes.c_uint64, SP, _I]
        L.orc_acmm_post_refine.argtypes = [FP, PP, SP, _I]
        L.orc_expf.argtypes = [_F]
        L.orc_expf.restype = _F
        L.orc_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_uniform.restype = _F
        L.orc_tex_fetch.argtypes = [_P, _I, _I, _F, _F]
        L.orc_tex_fetch.restype = _F
        L.orc_philox.argtypes = [_P, _P, _P]
        CP = ctypes.POINTER(OrcFilterCfg)
        L.orc_filter_global.argtypes = [FP, CP, _F, SP, _P, _P]
        L.orc_reprojection_error.argtypes = [FP, CP, _F, SP, _P]
        YP = ctypes.POINTER(OrcCycleCfg)
        L.orc_texture_mask.argtypes = [_P, _I, _I, YP, _P, _P, _P]
        L.orc_cycle_check.argtypes = [FP, YP, _F, SP, ctypes.POINTER(OrcCycleStats), _P, _P, _P]
        L.orc_mean_std_3x3.argtypes = [_P, _I, _I, _I, _P, _P]
        L.orc_refocus.argtypes = [FP, _I, _I, _P, _I, _I, _I, _P]
        L.orc_vd_to_rd.argtypes = [_F, _P]
        L.orc_vd_to_rd.restype = _F
        L.orc_vd_to_rd_segment.argtypes = [_F, _P, _I]
        L.orc_vd_to_rd_segment.restype = _F
        L.orc_vd_to_rd_map.argtypes = [_P, ctypes.c_long, _P, _P]
        L.orc_behavioral_fit.argtypes = [_P, _P, ctypes.c_long, _P]
        L.orc_refocus_samples.argtypes = [FP, _I, _I, _P, _I, _I, _I]
        L.orc_refocus_samples.restype = ctypes.c_longlong
        L.orc_fuse_virtual_depth.argtypes = [FP, _P, _P, _P, _P, _I, _P, ctypes.POINTER(OrcFuseParams), _I, _I,
                                             _P, _P, _P, _P]
        L.orc_fuse_virtual_depth.restype = ctypes.c_longlong
        L.orc_pm_sweep_taps.argtypes = [ctypes.POINTER(OrcFrame), ctypes.POINTER(OrcParams), ctypes.c_uint64, _I, _I,
                                        ctypes.POINTER(OrcState), ctypes.POINTER(OrcState), _I]
        L.orc_pm_sweep_taps.restype = ctypes.c_longlong
        L.orc_similarity.argtypes = [_P, _P, _I, _I, _F, _F]
        L.orc_select_neighbors.argtypes = [_I, _P, _P, _I, _I, _F, _P, _I, _I, _I, _P, _P, _P]
        L.orc_mla_otsu.argtypes = [_P, _I, _I, _I]
        L.orc_mla_contours.argtypes = [_P, _I, _I, _I, _I, _P, _P, _P, _I]
        L.orc_mla_centers.argtypes = [_P, _I, _I, _I, _F, _I, _I, _P, _P, _P, _P, _P, _P, _I, _P]
        L.orc_laplacian.argtypes = [_P, _I, _I, _I, _P]
        L.orc_blur_tiles.argtypes = [_P, _I, _I, _I, _P, _I, _I, _I, _P, _P]
        L.orc_glcm_contrast.argtypes = [_P, _I, _I, _I, _P]
        L.orc_normalize_minmax.argtypes = [_P, ctypes.c_size_t, ctypes.c_double, ctypes.c_double]
        L.orc_richness_tiles.argtypes = [_P, _I, _I, _I, _P, _I, _I, _I, _P, _P, _P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


class Oracle:
    """One frame of views for the oracle.  gray: [V][h][w] uint8/float."""

    def __init__(self, gray, centers, nb_ids, nb_counts, blur=None, shifted=False, acmm=False):
        self.shifted = bool(shifted)     # NCC moments of (texel - centre texel) instead of the reference's
        self.acmm = bool(acmm)           # the ACMM matcher's rules (one pyramid level)
        self.gray = np.ascontiguousarray(gray, dtype=np.float32)
        self.blur = None if blur is None else np.ascontiguousarray(blur, dtype=np.float32)
        self.centers = np.ascontiguousarray(centers, dtype=np.float32)
        self.nb_ids = np.ascontiguousarray(nb_ids, dtype=np.int32)
        self.nb_counts = np.ascontiguousarray(nb_counts, dtype=np.int32)
        V, h, w = self.gray.shape
        self.V, self.h, self.w = V, h, w
        self.K = self.nb_ids.shape[1]
        self.f = OrcFrame(V, w, h, self.K, _p(self.gray), _p(self.blur), _p(self.centers), _p(self.nb_ids),
                          _p(self.nb_counts))

    def params(self, p) -> OrcParams:
        """From the package's PmParams (same fields) and the oracle's moment mode."""
        c = p.c()
        return OrcParams(c.max_iterations, c.patch_size, c.radius_increment, c.top_k, c.sigma_spatial, c.sigma_color,
                         c.depth_min, c.depth_max, c.base, 1 if self.shifted else 0, 1 if self.acmm else 0)

    def new_state(self):
        n = self.V * self.h * self.w
        arr = dict(plane=np.zeros((n, 4), np.float32), cost=np.zeros(n, np.float32),
                   disp=np.zeros((n, 4), np.float32), sel=np.zeros(n, np.uint32))
        st = OrcState(_p(arr["plane"]), _p(arr["cost"]), _p(arr["disp"]), _p(arr["sel"]))
        return arr, st

    def cost_vectors(self, params, vids, pxy, planes):
        v = np.ascontiguousarray(vids, np.int32)
        xy = np.ascontiguousarray(pxy, np.int32)
        pl = np.ascontiguousarray(planes, np.float32)
        costs = np.empty((v.shape[0], self.K), np.float32)
        disps = np.empty((v.shape[0], self.K, 4), np.float32)
        p = self.params(params)
        rc = lib().orc_cost_vectors(ctypes.byref(self.f), ctypes.byref(p), _p(v), _p(xy), _p(pl), v.shape[0],
                                    _p(costs), _p(disps))
        assert rc == 0
        return costs, disps

    def count_taps(self, params, vids, pxy, planes) -> int:
        v = np.ascontiguousarray(vids, np.int32)
        xy = np.ascontiguousarray(pxy, np.int32)
        pl = np.ascontiguousarray(planes, np.float32)
        p = self.params(params)
        return int(lib().orc_count_taps(ctypes.byref(self.f), ctypes.byref(p), _p(v), _p(xy), _p(pl), v.shape[0]))

    def ncc_fp64(self, params, vid, k, px, py, plane) -> float:
        pl = np.ascontiguousarray(plane, np.float32)
        p = self.params(params)
        return float(lib().orc_ncc_fp64(ctypes.byref(self.f), ctypes.byref(p), vid, k, px, py, _p(pl)))

    def ncc_fp64_batch(self, params, vids, pxy, planes, sampling=0, nthreads=0) -> np.ndarray:
        """[n][max_nb] FP64 NCC costs (sampling 0: exact bilinear; 1: the texture's
        quantised sampling)."""
        p = self.params(params)
        v = np.ascontiguousarray(vids, np.int32)
        q = np.ascontiguousarray(pxy, np.int32)
        pl = np.ascontiguousarray(planes, np.float32)
        out = np.zeros((len(v), self.K), np.float64)
        lib().orc_ncc_fp64_batch(ctypes.byref(self.f), ctypes.byref(p), _p(v), _p(q), _p(pl), len(v), sampling,
                                 nthreads, _p(out))
        return out

    def init(self, params, seed, nthreads=0, views=None):
        arr, st = self.new_state()
        p = self.params(params)
        if views is None:
            rc = lib().orc_pm_init(ctypes.byref(self.f), ctypes.byref(p), seed, ctypes.byref(st), nthreads)
        else:
            rc = lib().orc_pm_init_views(ctypes.byref(self.f), ctypes.byref(p), seed, ctypes.byref(st), views[0],
                                         views[1], nthreads)
        assert rc == 0
        return arr

    def sweep(self, params, seed, it, phase, prev, nthreads=0, views=None):
        arr, st = self.new_state()
        ps = OrcState(_p(prev["plane"]), _p(prev["cost"]), _p(prev["disp"]), _p(prev["sel"]))
        p = self.params(params)
        if views is None:
            rc = lib().orc_pm_sweep(ctypes.byref(self.f), ctypes.byref(p), seed, it, phase, ctypes.byref(ps),
                                    ctypes.byref(st), nthreads)
        else:
            rc = lib().orc_pm_sweep_views(ctypes.byref(self.f), ctypes.byref(p), seed, it, phase, ctypes.byref(ps),
                                          ctypes.byref(st), views[0], views[1], nthreads)
        assert rc == 0
        return arr

    def sweep_taps(self, params, seed, it, phase, prev, nthreads=0, views=None):
        """(next state, in-bounds NCC taps of the reference's algorithm in this
        sweep, over the views [views[0], views[1]) when given)."""
        arr, st = self.new_state()
        ps = OrcState(_p(prev["plane"]), _p(prev["cost"]), _p(prev["disp"]), _p(prev["sel"]))
        p = self.params(params)
        if views is None:
            taps = lib().orc_pm_sweep_taps(ctypes.byref(self.f), ctypes.byref(p), seed, it, phase, ctypes.byref(ps),
                                           ctypes.byref(st), nthreads)
        else:
            taps = lib().orc_pm_sweep_views_taps(ctypes.byref(self.f), ctypes.byref(p), seed, it, phase,
                                                 ctypes.byref(ps), ctypes.byref(st), views[0], views[1], nthreads)
        assert taps >= 0
        return arr, int(taps)

    def acmm_post_refine(self, params, state, nthreads=0):
        """PostRefineMetadataFrame over a copy of state (dict of arrays)."""
        arr = {k: np.ascontiguousarray(v).copy() for k, v in state.items()}
        st = OrcState(_p(arr["plane"]), _p(arr["cost"]), _p(arr["disp"]), _p(arr["sel"]))
        p = self.params(params)
        assert lib().orc_acmm_post_refine(ctypes.byref(self.f), ctypes.byref(p), ctypes.byref(st), nthreads) == 0
        return arr

    def patchmatch(self, params, seed, nthreads=0):
        arr, st = self.new_state()
        p = self.params(params)
        assert lib().orc_patchmatch(ctypes.byref(self.f), ctypes.byref(p), seed, ctypes.byref(st), nthreads) == 0
        return arr


def _fcfg(cfg) -> OrcFilterCfg:
    c = cfg.c()
    return OrcFilterCfg(*[getattr(c, n) for n, _ in OrcFilterCfg._fields_])


def _state_struct(arr):
    return OrcState(_p(arr["plane"]), _p(arr["cost"]), _p(arr["disp"]), _p(arr["sel"]))


def filter_global(orc: "Oracle", cfg, baseline_unit: float, state: dict):
    """MIDisparityFilterCPU::FilterGlobal on `state` (modified in place).
    Returns (reason map, stats array of 8 counters)."""
    n = orc.V * orc.h * orc.w
    reason = np.zeros(n, np.uint8)
    stats = np.zeros(8, np.int64)
    st = _state_struct(state)
    c = _fcfg(cfg)
    assert lib().orc_filter_global(ctypes.byref(orc.f), ctypes.byref(c), float(baseline_unit), ctypes.byref(st),
                                   _p(reason), _p(stats)) == 0
    return reason, stats


def reprojection_error(orc: "Oracle", cfg, baseline_unit: float, state: dict) -> np.ndarray:
    err = np.zeros(orc.V * orc.h * orc.w, np.float32)
    st = _state_struct(state)
    c = _fcfg(cfg)
    assert lib().orc_reprojection_error(ctypes.byref(orc.f), ctypes.byref(c), float(baseline_unit), ctypes.byref(st),
                                        _p(err)) == 0
    return err


def _ycfg(cfg) -> OrcCycleCfg:
    c = cfg.c()
    return OrcCycleCfg(*[getattr(c, n) for n, _ in OrcCycleCfg._fields_])


def texture_mask(gray, cfg):
    """BuildTextureMaskAndViz on one float image: (grad magnitude, 7x7 var, mask)."""
    g = np.ascontiguousarray(gray, np.float32)
    H, W = g.shape
    grad = np.zeros_like(g)
    var = np.zeros_like(g)
    mask = np.zeros(g.shape, np.uint8)
    c = _ycfg(cfg)
    assert lib().orc_texture_mask(_p(g), W, H, ctypes.byref(c), _p(grad), _p(var), _p(mask)) == 0
    return grad, var, mask


def cycle_check(orc: "Oracle", cfg, baseline_unit: float, state: dict):
    """MICycleCheckerCPU::CheckGlobal: (stats dict, geo_err, pho_err, texture mask)."""
    n = orc.V * orc.h * orc.w
    geo = np.zeros(n, np.float32)
    pho = np.zeros(n, np.float32)
    tm = np.zeros(n, np.uint8)
    st = _state_struct(state)
    out = OrcCycleStats()
    c = _ycfg(cfg)
    assert lib().orc_cycle_check(ctypes.byref(orc.f), ctypes.byref(c), float(baseline_unit), ctypes.byref(st),
                                 ctypes.byref(out), _p(geo), _p(pho), _p(tm)) == 0
    return {k: getattr(out, k) for k in CYCLE_STAT_FIELDS}, geo, pho, tm


def refocus(orc: "Oracle", raw_w: int, raw_h: int, slice_vd, out_w: int, out_h: int) -> np.ndarray:
    """Focal-stack render [n_slices][out_h][out_w] (see orc_refocus)."""
    vd = np.ascontiguousarray(slice_vd, np.float32)
    out = np.zeros((vd.shape[0], out_h, out_w), np.float32)
    assert lib().orc_refocus(ctypes.byref(orc.f), raw_w, raw_h, _p(vd), vd.shape[0], out_w, out_h, _p(out)) == 0
    return out


def refocus_samples(orc: "Oracle", raw_w: int, raw_h: int, slice_vd, out_w: int, out_h: int) -> int:
    vd = np.ascontiguousarray(slice_vd, np.float32)
    return int(lib().orc_refocus_samples(ctypes.byref(orc.f), raw_w, raw_h, _p(vd), vd.shape[0], out_w, out_h))


def fuse_virtual_depth(orc: "Oracle", plane, lists, list_counts, is_ref, raw_w: int, raw_h: int, mla_base: float,
                       bgr=None, min_ref_disp=1.0, max_reproj_px=1.0, max_rel_vd=0.05, min_consistent=2):
    """LFRefocus::FuseVirtualDepth_BackProject: (vd_map, conf, aif [h][w][3], points [n][9])."""
    pl = np.ascontiguousarray(plane, np.float32).reshape(-1, 4)
    ls = np.ascontiguousarray(lists, np.int32)
    lc = np.ascontiguousarray(list_counts, np.int32)
    ir = np.ascontiguousarray(is_ref, np.uint8)
    b = None if bgr is None else np.ascontiguousarray(bgr, np.uint8)
    vd = np.zeros((raw_h, raw_w), np.float32)
    cf = np.zeros((raw_h, raw_w), np.uint8)
    aif = np.zeros((raw_h, raw_w, 3), np.uint8)
    pts = np.zeros((pl.shape[0], 9), np.float32)
    prm = OrcFuseParams(mla_base, min_ref_disp, max_reproj_px, max_rel_vd, min_consistent)
    n = lib().orc_fuse_virtual_depth(ctypes.byref(orc.f), _p(pl), _p(b), _p(ls), _p(lc), ls.shape[1], _p(ir),
                                     ctypes.byref(prm), raw_w, raw_h, _p(vd), _p(cf), _p(aif), _p(pts))
    assert n >= 0
    return vd, cf, aif, pts[:n]


def similarity(src_bin, nb_bin, dx: float, dy: float) -> int:
    """MISimilarityMeasure::MeasureSimilarity on two binary (0/255) images."""
    a = np.ascontiguousarray(src_bin, np.uint8)
    b = np.ascontiguousarray(nb_bin, np.uint8)
    return int(lib().orc_similarity(_p(a), _p(b), a.shape[1], a.shape[0], dx, dy))


def select_neighbors(centers, tilekeys, u_size: int, v_size: int, pitch: float, images=None, max_out: int = 128):
    """m_NeighsSortVecForMatch per view: (ids [V][max_out], counts [V], similarity [V][max_out])."""
    c = np.ascontiguousarray(centers, np.float32)
    k = np.ascontiguousarray(tilekeys, np.int32)
    V = c.shape[0]
    im = None if images is None else np.ascontiguousarray(images, np.uint8)
    mh, mw = (im.shape[1], im.shape[2]) if im is not None else (0, 0)
    ids = np.full((V, max_out), -1, np.int32)
    cnt = np.zeros(V, np.int32)
    sim = np.zeros((V, max_out), np.float32)
    rc = lib().orc_select_neighbors(V, _p(c), _p(k), u_size, v_size, pitch, _p(im), mw, mh, max_out, _p(ids), _p(cnt),
                                    _p(sim))
    assert rc == 0
    return ids, cnt, sim


def _bgr(img):
    img = np.ascontiguousarray(img, np.uint8)
    if img.ndim == 2:
        img = np.ascontiguousarray(np.repeat(img[:, :, None], 3, axis=2))
    return img


def mla_otsu(img) -> int:
    b = _bgr(img)
    return int(lib().orc_mla_otsu(_p(b), b.shape[1], b.shape[0], b.strides[0]))


def mla_contours(img, threshold: int):
    """(cx, cy, area) of the external contours, in OpenCV's order."""
    b = _bgr(img)
    cap = b.shape[0] * b.shape[1] // 2 + 1
    cx = np.zeros(cap, np.float32)
    cy = np.zeros(cap, np.float32)
    ar = np.zeros(cap, np.float64)
    n = lib().orc_mla_contours(_p(b), b.shape[1], b.shape[0], b.strides[0], threshold, _p(cx), _p(cy), _p(ar), cap)
    assert n >= 0
    return cx[:n], cy[:n], ar[:n]


def mla_centers(img, baseline: float, mla_u_size: int, mla_v_size: int):
    """Map entries in key order: dict of col, row, cx, cy, area, abandon; and the threshold."""
    b = _bgr(img)
    cap = b.shape[0] * b.shape[1] // 2 + 1
    col = np.zeros(cap, np.int32)
    row = np.zeros(cap, np.int32)
    cx = np.zeros(cap, np.float32)
    cy = np.zeros(cap, np.float32)
    ar = np.zeros(cap, np.float32)
    ab = np.zeros(cap, np.int32)
    t = ctypes.c_int(0)
    n = lib().orc_mla_centers(_p(b), b.shape[1], b.shape[0], b.strides[0], baseline, mla_u_size, mla_v_size, _p(col),
                              _p(row), _p(cx), _p(cy), _p(ar), _p(ab), cap, ctypes.byref(t))
    assert n >= 0
    return dict(col=col[:n], row=row[:n], cx=cx[:n], cy=cy[:n], area=ar[:n], abandon=ab[:n]), t.value


def laplacian(gray) -> np.ndarray:
    """cv::Laplacian(gray, CV_32F) with ksize 1 (oracle/blur.c)."""
    g = np.ascontiguousarray(gray, np.uint8)
    out = np.zeros(g.shape, np.float32)
    lib().orc_laplacian(_p(g), g.shape[1], g.shape[0], g.strides[0], _p(out))
    return out


def window_origins(centers, mi_w: int, mi_h: int) -> np.ndarray:
    """Left-down corners of the matching windows: the centre minus (mi - 1) / 2 in
    double, stored as float, truncated to int (DepthSolver.cpp:1894-1895, 1977-1978)."""
    c = np.asarray(centers, np.float32).reshape(-1, 2).astype(np.float64)
    ox = (c[:, 0] - (mi_w - 1) * 0.5).astype(np.float32)
    oy = (c[:, 1] - (mi_h - 1) * 0.5).astype(np.float32)
    return np.ascontiguousarray(np.stack([ox, oy], 1).astype(np.int32))


def blur_tiles(gray, origins, mi_w: int, mi_h: int):
    """Per-view blur channel [V][mi_h][mi_w] (u8) and blureness values [V] (oracle/blur.c)."""
    g = np.ascontiguousarray(gray, np.uint8)
    o = np.ascontiguousarray(origins, np.int32).reshape(-1, 2)
    V = o.shape[0]
    tiles = np.zeros((V, mi_h, mi_w), np.uint8)
    counts = np.zeros(V, np.uint32)
    rc = lib().orc_blur_tiles(_p(g), g.shape[1], g.shape[0], g.strides[0], _p(o), V, mi_w, mi_h, _p(tiles),
                              _p(counts))
    assert rc == 0, "window outside the frame"
    return tiles, counts


def glcm_contrast(gray) -> np.ndarray:
    """GLCM contrast map of QuantizeRichnessByGLCM before normalisation (oracle/blur.c)."""
    g = np.ascontiguousarray(gray, np.uint8)
    out = np.zeros(g.shape, np.float32)
    lib().orc_glcm_contrast(_p(g), g.shape[1], g.shape[0], g.strides[0], _p(out))
    return out


def normalize_minmax(a, lo: float = 0.0, hi: float = 255.0) -> np.ndarray:
    """cv::normalize(a, lo, hi, NORM_MINMAX) of a float map (oracle/blur.c)."""
    out = np.ascontiguousarray(a, np.float32).copy()
    lib().orc_normalize_minmax(_p(out), out.size, lo, hi)
    return out


def richness_tiles(gray, origins, mi_w: int, mi_h: int):
    """Per-view normalised GLCM score [V][mi_h][mi_w] (f32), richness channel (u8,
    0 or 255) and richness values [V] (oracle/blur.c)."""
    g = np.ascontiguousarray(gray, np.uint8)
    o = np.ascontiguousarray(origins, np.int32).reshape(-1, 2)
    V = o.shape[0]
    score = np.zeros((V, mi_h, mi_w), np.float32)
    binary = np.zeros((V, mi_h, mi_w), np.uint8)
    counts = np.zeros(V, np.uint32)
    rc = lib().orc_richness_tiles(_p(g), g.shape[1], g.shape[0], g.strides[0], _p(o), V, mi_w, mi_h, _p(score),
                                  _p(binary), _p(counts))
    assert rc == 0, "window outside the frame"
    return score, binary, counts


def vd_to_rd_points(vd, c):
    """LFRefocus::ConvertVdToRd per value (float results)."""
    cc = np.ascontiguousarray(c, np.float64)
    return np.array([lib().orc_vd_to_rd(float(v), _p(cc)) for v in np.asarray(vd, np.float32)], np.float32)


def vd_to_rd_segments(vd, segs):
    """LFRefocus::ConvertVdToRdSegment per value; segs [n][5] (min, max, c0, c1, c2)."""
    sg = np.ascontiguousarray(segs, np.float64).reshape(-1, 5)
    return np.array([lib().orc_vd_to_rd_segment(float(v), _p(sg), sg.shape[0]) for v in np.asarray(vd, np.float32)],
                    np.float32)


def vd_to_rd_map(vd, c) -> np.ndarray:
    """VirtualToRealDepthFunc::convertVirtualToRealDepth (double results)."""
    v = np.ascontiguousarray(vd, np.float32).ravel()
    out = np.zeros(v.shape[0], np.float64)
    cc = np.ascontiguousarray(c, np.float64)
    lib().orc_vd_to_rd_map(_p(v), v.shape[0], _p(cc), _p(out))
    return out


def behavioral_fit(real_depth, vd):
    """VirtualToRealDepthFunc::BehavioralModel (normal equations, long double)."""
    r = np.ascontiguousarray(real_depth, np.float32)
    v = np.ascontiguousarray(vd, np.float32)
    c = np.zeros(3, np.float64)
    assert lib().orc_behavioral_fit(_p(r), _p(v), r.shape[0], _p(c)) == 0
    return c


def mean_std_3x3(img, x0: int, y0: int):
    a = np.ascontiguousarray(img, np.float32)
    m = np.zeros(1, np.float32)
    s = np.zeros(1, np.float32)
    lib().orc_mean_std_3x3(_p(a), a.shape[1], x0, y0, _p(m), _p(s))
    return float(m[0]), float(s[0])


def expf(x: float) -> float:
    return float(lib().orc_expf(x))


def uniform(seed: int, sweep: int, pixel: int, n: int) -> float:
    return float(lib().orc_uniform(seed, sweep, pixel, n))


def tex_fetch(img: np.ndarray, sx: float, sy: float) -> float:
    a = np.ascontiguousarray(img, np.float32)
    return float(lib().orc_tex_fetch(_p(a), a.shape[1], a.shape[0], sx, sy))


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().orc_philox(_p(c), _p(k), _p(o))
    return [int(x) for x in o]
