"""The C++ classes with the reference's interface (include/pfd/AdaptMIPMFrame.h,
MIDisparityFilter.h, MICycleCheck.h) used as MIStereoMatch uses them, against
the engine's C ABI called directly on the frame the reference's bookkeeping
describes.  Everything is integer, copy or as-written arithmetic on the same
inputs, so every array and every statistic must match bit for bit:

* AdaptMIPMFrame::Initialize / RunPatchMatchCUDAForFrame / WriteBackResults on
  maps with garbage lenses, unmatched lenses, missing lens information, missing
  result maps, foreign neighbour keys and lists past 16 entries, against
  pfd_frame_create + pfd_patchmatch on the views and lists of
  AdaptMIPMFrame.cpp:145-222 (restated in shim_scene.py);
* MICycleCheckerCPU::CheckGlobal and MIDisparityFilterCPU::FilterGlobal
  (with its whole-frame reprojection-error figures, MIDisparityFilter.cpp:
  844-950) on the matched maps, against pfd_cycle_check / pfd_filter /
  pfd_reprojection_error on the views and lists of BuildTileInputsFromMaps,
  and the filter's reasons against the CPU oracle too."""
import ctypes

import numpy as np
import pytest

from shim_scene import HAS_DN, irregular_scene, load_probe

pytestmark = pytest.mark.gpu

SEED = 19


def _f32(x):
    return np.float32(x)


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


def _quantile(sorted_vals, q):
    """QuantileFromSorted (MIDisparityFilter.cpp:36-51) in float32."""
    n = len(sorted_vals)
    if n == 0:
        return 0.0
    if n == 1:
        return float(sorted_vals[0])
    pos = _f32(q) * _f32(n - 1)
    lo, hi = int(np.floor(pos)), int(np.ceil(pos))
    t = _f32(pos - _f32(lo))
    if lo == hi:
        return float(sorted_vals[lo])
    return float(_f32(sorted_vals[lo] * (_f32(1) - t)) + _f32(sorted_vals[hi] * t))


@pytest.fixture(scope="module")
def shim(pfd):
    L = load_probe(pfd)
    w, sc = irregular_scene(pfd)
    P = pfd.PmParams(base=sc.pitch, patch_size=11, max_iterations=2)
    fc = pfd.FilterCfg(min_good_neighbors=1)
    cc = pfd.CycleCfg()
    n, ppv = sc.n, sc.mi * sc.mi
    dn_match = np.full((n, ppv, 13), np.nan, np.float32)
    dn_filter = np.full((n, ppv, 13), np.nan, np.float32)
    fstats = np.zeros(13)
    cstats = np.zeros(14)
    cmasked = np.zeros(11)
    msg = ctypes.create_string_buffer(256)
    fcc, ccc = fc.c(), cc.c()
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.shim_run(*sc.args(), p(sc.dn_init), P.patch_size, P.max_iterations, P.top_k, P.sigma_spatial,
                    P.sigma_color, SEED, ctypes.c_void_p(ctypes.addressof(fcc)),
                    ctypes.c_void_p(ctypes.addressof(ccc)), p(dn_match), p(dn_filter), p(fstats), p(cstats),
                    p(cmasked), msg)
    assert rc == 0, msg.value.decode()
    return dict(w=w, sc=sc, P=P, fc=fc, cc=cc, dn_match=dn_match, dn_filter=dn_filter, fstats=fstats,
                cstats=cstats, cmasked=cmasked)


@pytest.fixture(scope="module")
def direct_match(pfd, shim):
    """pfd_patchmatch on the reference's match views, micro-images sliced on
    the device from the raw frame (the classes upload the problems' images)."""
    sc, w = shim["sc"], shim["w"]
    views, lists = sc.expected_match_layout()
    centers, keys, ids, cnt, _ = sc.frame_arrays(views, lists, 16)
    with pfd.Context(0) as ctx:
        fid = ctx.frame_upload(w.frame.raw, centers, keys, sc.mi, sc.mi, ids, cnt)
        ctx.patchmatch(fid, shim["P"], seed=SEED)
        st = ctx.download(fid)
        ctx.frame_free(fid)
    return views, st


def test_adapt_mipm_frame_matches_the_engine(shim, direct_match):
    sc = shim["sc"]
    views, (plane, cost, disp, sel) = direct_match
    ppv = sc.mi * sc.mi
    dm = shim["dn_match"]
    assert np.mean(cost < 1.0) > 0.3, "too few matched pixels for a meaningful comparison"
    for v, p in enumerate(views):
        s = slice(v * ppv, (v + 1) * ppv)
        if not sc.flags[p] & HAS_DN:
            assert np.all(np.isnan(dm[p])), "a lens without a result map was written"
            continue
        assert _same(dm[p, :, 0:4], plane[s]), f"problem {p}: ph_cuda differs"
        assert _same(dm[p, :, 4], plane[s, 3]), f"problem {p}: d_cuda differs"
        assert _same(dm[p, :, 5], cost[s]), f"problem {p}: c_cuda differs"
        assert _same(dm[p, :, 6:10], disp[s]), f"problem {p}: disp_v_cuda differs"
        assert np.array_equal(dm[p, :, 10].view(np.uint32), sel[s]), f"problem {p}: selected_views differs"
        assert np.all(dm[p, :, 11] == 1.0)                   # eSS_ACMH_Finished
    # results of lenses that are not matched keep their contents
    others = [p for p in range(sc.n) if p not in set(views) and sc.flags[p] & HAS_DN]
    assert others
    for p in others:
        assert _same(dm[p, :, :11], sc.dn_init[p, :, :11])


def _check_frame(pfd, ctx, shim):
    """An engine frame with the consistency pass's views, lists and micro-images,
    holding the matched results."""
    sc = shim["sc"]
    views, lists = sc.expected_check_layout()
    max_nb = max(len(l) for l in lists.values())
    centers, keys, ids, cnt, gray = sc.frame_arrays(views, lists, max_nb)
    W = int(np.max(np.trunc(centers[:, 0] - (sc.mi - 1) * 0.5))) + sc.mi
    H = int(np.max(np.trunc(centers[:, 1] - (sc.mi - 1) * 0.5))) + sc.mi
    fid = ctx.frame_create(W, H, centers, keys, sc.mi, sc.mi, ids, cnt)
    ctx.frame_set_micro_images(fid, gray)
    dm = shim["dn_match"][views]
    plane = dm[:, :, 0:4].reshape(-1, 4).copy()
    bad = ~np.isfinite(plane[:, 3])
    plane[bad, 3] = dm[:, :, 4].reshape(-1)[bad]             # read_disp: ph.w, else d
    ctx.state_upload(fid, plane, dm[:, :, 5], dm[:, :, 6:10].reshape(-1, 4),
                     dm[:, :, 10].reshape(-1).view(np.uint32))
    return fid, views, (gray, centers, ids, cnt)


def test_cycle_checker_matches_the_engine(pfd, shim):
    with pfd.Context(0) as ctx:
        fid, views, _ = _check_frame(pfd, ctx, shim)
        # the checker reads ph.w with no fallback to d; the frame above holds the
        # filter's view of the state, which is the same when every ph.w is finite
        assert np.all(np.isfinite(shim["dn_match"][views, :, 3]))
        st, _, _, _ = ctx.cycle_check(fid, shim["cc"], shim["sc"].pitch, maps=False)
        ctx.frame_free(fid)
    names = ("mean_geo_err_px", "median_geo_err_px", "p90_geo_err_px", "mean_photo_err", "num_samples",
             "rmse_geo_err_px", "rmse_photo_err", "completeness", "completeness_geo", "completeness_photo",
             "completeness_masked_pixels", "completeness_good_pixels", "completeness_good_pixels_geo",
             "completeness_good_pixels_photo")
    assert st["num_samples"] > 1000
    for i, k in enumerate(names):
        assert shim["cstats"][i] == float(st[k]), k
    masked = ("masked_count", "all_count", "masked_geo_mean", "masked_photo_mean", "masked_geo_rmse",
              "masked_photo_rmse", "coverage", "masked_geo_median_approx", "masked_geo_p90_approx", "masked_geo_min",
              "masked_geo_max")
    for i, k in enumerate(masked):
        assert shim["cmasked"][i] == float(st[k]), k


def test_disparity_filter_matches_the_engine_and_the_oracle(pfd, oracle, shim):
    sc, fc = shim["sc"], shim["fc"]
    ppv = sc.mi * sc.mi
    with pfd.Context(0) as ctx:
        fid, views, (gray, centers, ids, cnt) = _check_frame(pfd, ctx, shim)
        before = ctx.download(fid)
        reason, stats = ctx.filter(fid, fc, sc.pitch)
        err = ctx.reprojection_error(fid, fc, sc.pitch)
        ctx.frame_free(fid)
    assert 0 < stats["removed"] < stats["valid_in"]
    assert list(shim["fstats"][:8]) == [float(v) for v in stats.values()]

    orc = oracle.Oracle(gray, centers, ids, cnt)
    st = dict(plane=before[0].copy(), cost=before[1].copy(), disp=before[2].copy(), sel=before[3].copy())
    o_reason, _ = oracle.filter_global(orc, fc, sc.pitch, st)
    assert np.array_equal(o_reason, reason)

    # the classes write InvalidatePixel into rejected pixels only
    dm, df = shim["dn_match"], shim["dn_filter"]
    for v, p in enumerate(views):
        r = reason[v * ppv:(v + 1) * ppv]
        keep = r == 0
        assert _same(df[p, keep, :11], dm[p, keep, :11]), f"problem {p}: a kept pixel changed"
        gone = df[p, ~keep]
        assert np.all(gone[:, 0:4] == [0, 0, 0, -1]) and np.all(gone[:, 4] == -1) and np.all(gone[:, 5] == 2)
        assert np.all(gone[:, 6:10] == [-1, -1, 0, 0]) and np.all(gone[:, 10].view(np.uint32) == 0)

    # DumpWholeFrameReprojectionError's figures
    e = err[np.isfinite(err) & (err >= 0) & (err <= np.float32(2.0))]
    assert e.size > 100
    n_le = int(np.count_nonzero(e <= np.float32(0.5)))
    s = np.cumsum(e.astype(np.float64))[-1]
    sq = np.cumsum(e.astype(np.float64) * e.astype(np.float64))[-1]
    fs = shim["fstats"]
    assert fs[8] == e.size and fs[9] == n_le
    assert fs[10] == s / e.size
    assert fs[11] == np.sqrt(sq / e.size)
    assert fs[12] == _quantile(np.sort(e), 0.9)


def test_adapt_mipm_frame_acmm_matches_the_engine(pfd, oracle):
    """AdaptMIPMFrameACMM with the reference's own level parameters (one level
    below a 24-pixel window: patch 5, 5 iterations, top_k 6, PatchMatchParamsLF's
    sigmas 5 and 3) against PFD_MATCHER_ACMM called directly on the same views,
    and both against the oracle's ACMM mode."""
    L = load_probe(pfd)
    w, sc = irregular_scene(pfd)
    n, ppv = sc.n, sc.mi * sc.mi
    dn = np.full((n, ppv, 13), np.nan, np.float32)
    levels = ctypes.c_int(0)
    msg = ctypes.create_string_buffer(256)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.shim_run_acmm(*sc.args(), p(sc.dn_init), SEED, p(dn), ctypes.byref(levels), msg)
    assert rc == 0, msg.value.decode()
    assert levels.value == 1
    views, lists = sc.expected_match_layout()
    centers, keys, ids, cnt, gray = sc.frame_arrays(views, lists, 16)
    P = pfd.PmParams(base=sc.pitch, patch_size=5, max_iterations=5, top_k=6, sigma_spatial=5.0, sigma_color=3.0)
    with pfd.Context(0) as ctx:
        fid = ctx.frame_upload(w.frame.raw, centers, keys, sc.mi, sc.mi, ids, cnt)
        ctx.set_matcher(True)
        ctx.patchmatch(fid, P, seed=SEED)
        plane, cost, disp, sel = ctx.download(fid)
        ctx.frame_free(fid)
    st = oracle.Oracle(gray, centers, ids, cnt, acmm=True).patchmatch(P, SEED)
    assert _same(plane, st["plane"]) and _same(cost, st["cost"]) and _same(sel, st["sel"])
    assert np.mean(cost < 1.0) > 0.3
    for v, pi in enumerate(views):
        s = slice(v * ppv, (v + 1) * ppv)
        if not sc.flags[pi] & HAS_DN:
            continue
        assert _same(dn[pi, :, 0:4], plane[s]), f"problem {pi}: ph_cuda differs"
        assert _same(dn[pi, :, 5], cost[s]), f"problem {pi}: c_cuda differs"
        assert _same(dn[pi, :, 6:10], disp[s]), f"problem {pi}: disp_v_cuda differs"
        assert np.array_equal(dn[pi, :, 10].view(np.uint32), sel[s]), f"problem {pi}: selected_views differs"
        assert np.all(dn[pi, :, 11] == 1.0)                   # eSS_ACMH_Finished
