"""Device parity of the consistency pass: pfd_filter (MIDisparityFilterCPU::
FilterGlobal, CheckModule/MIDisparityFilter.cpp:962-986) and
pfd_reprojection_error (ComputeTileReprojectionErrorMap, :695-842) against the
CPU oracle on the same PatchMatch state.  Reject reasons, counters and the
filtered state are integer or copy work and must match bit for bit; the
reprojection map is evaluated as written in both and must match bit for bit
too.  The filter is order dependent (a view reads its neighbours after the
views before it in map order were filtered in place), so this also checks the
wavefront schedule."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PITCH = 23.0


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def matched(pfd, ctx):
    """A 360x280 frame after a 2-iteration PatchMatch, views in map order
    (tile row, then column)."""
    w = pfd.make_workload(360, 280, PITCH, 5, seed=23, max_nb=6)
    order = np.lexsort((w.tilekeys[:, 0], w.tilekeys[:, 1]))
    assert np.array_equal(order, np.arange(len(order))), "views must be in map order"
    P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.patchmatch(fid, P, seed=3)
    state = ctx.download(fid)
    ctx.frame_free(fid)
    return w, state


def _fresh_frame(ctx, w, state, pfd):
    """Frame whose state is the stored PatchMatch result (the same seed, run again)."""
    P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.patchmatch(fid, P, seed=3)
    again = ctx.download(fid)
    assert all(_same(a, b) for a, b in zip(again, state)), "PatchMatch is not deterministic"
    return fid


def _as_dict(state):
    plane, cost, disp, sel = state
    return dict(plane=plane.copy(), cost=cost.copy(), disp=disp.copy(), sel=sel.copy())


CFGS = {
    "default": {},
    "all_views": dict(use_selected_views_only=False),
    "one_good_no_spike": dict(min_good_neighbors=1, enable_spike_filter=False),
    "geo_only": dict(enable_cycle_photo_filter=False, max_geo_err_px=0.25, spike_abs_diff=0.5),
    "keep_sel": dict(clear_selected_views_when_invalid=False, max_cost=1.2),
}


@pytest.mark.parametrize("name", list(CFGS))
def test_filter_matches_oracle(pfd, oracle, ctx, matched, name):
    w, state = matched
    cfg = pfd.FilterCfg(**CFGS[name])
    fid = _fresh_frame(ctx, w, state, pfd)
    reason, stats = ctx.filter(fid, cfg, PITCH)
    after = ctx.download(fid)
    ctx.frame_free(fid)

    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    st = _as_dict(state)
    o_reason, o_stats = oracle.filter_global(orc, cfg, PITCH, st)

    assert stats["valid_in"] > 0.3 * stats["total"]
    assert 0 < stats["removed"] < stats["valid_in"], "a check that removes nothing or everything proves little"
    bad = np.nonzero(reason != o_reason)[0]
    assert bad.size == 0, f"{bad.size} reasons differ, first at {bad[:5]}: gpu {reason[bad[:5]]} oracle {o_reason[bad[:5]]}"
    assert list(stats.values()) == [int(x) for x in o_stats]
    for nm, g, o in zip(("plane", "cost", "disp", "sel"), after, (st["plane"], st["cost"], st["disp"], st["sel"])):
        assert _same(g, o), f"{nm} differs after the filter"


def test_filter_is_order_dependent(pfd, oracle, matched):
    """Filtering the views in reverse map order changes some reasons on this
    frame, so the bit-exact match above does exercise the in-place order."""
    w, state = matched
    cfg = pfd.FilterCfg()
    V, n = w.centers.shape[0], w.mi * w.mi
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    ra, _ = oracle.filter_global(orc, cfg, PITCH, _as_dict(state))

    perm = np.arange(V)[::-1]
    inv = np.empty(V, np.int64)
    inv[perm] = np.arange(V)
    ids = w.nb_ids[perm].copy()
    ids[ids >= 0] = inv[ids[ids >= 0]]
    rev = oracle.Oracle(w.gray[perm], w.centers[perm], ids, w.nb_counts[perm])
    pix = (perm[:, None] * n + np.arange(n)[None, :]).ravel()
    st = {k: v[pix].copy() for k, v in _as_dict(state).items()}
    rr, _ = oracle.filter_global(rev, cfg, PITCH, st)
    back = np.empty_like(rr)
    back[pix] = rr
    assert np.count_nonzero(back != ra) > 0


@pytest.mark.parametrize("when", ["before", "after"])
def test_reprojection_error_matches_oracle(pfd, oracle, ctx, matched, when):
    w, state = matched
    cfg = pfd.FilterCfg(min_good_neighbors=1, enable_spike_filter=False)   # keeps about a third
    fid = _fresh_frame(ctx, w, state, pfd)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    st = _as_dict(state)
    if when == "after":
        ctx.filter(fid, cfg, PITCH)
        oracle.filter_global(orc, cfg, PITCH, st)
    err = ctx.reprojection_error(fid, cfg, PITCH)
    ctx.frame_free(fid)
    o_err = oracle.reprojection_error(orc, cfg, PITCH, st)
    assert np.mean(o_err >= 0) > 0.1
    bad = np.nonzero(~((err == o_err) | (np.isnan(err) & np.isnan(o_err))))[0]
    assert bad.size == 0, f"{bad.size} errors differ, first at {bad[:5]}: gpu {err[bad[:5]]} oracle {o_err[bad[:5]]}"


def test_filter_errors(pfd, ctx, matched):
    w, _ = matched
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    with pytest.raises(pfd.PfdError) as e:
        ctx.filter(fid, pfd.FilterCfg(), PITCH)          # no PatchMatch state yet
    assert e.value.code == -7
    ctx.pm_init(fid, pfd.PmParams(base=PITCH), 1)
    with pytest.raises(pfd.PfdError) as e:
        ctx.filter(fid, pfd.FilterCfg(), 0.0)
    assert e.value.code == -1
    with pytest.raises(pfd.PfdError) as e:
        ctx.filter(fid, pfd.FilterCfg(max_triplet=33), PITCH)
    assert e.value.code == -1
    ctx.frame_free(fid)
