"""Device parity with the CPU oracle at the two single-frame workloads' full
sizes (tests/configs.py).

small (1024x768, 6 neighbours, 11x11 NCC, 3 iterations): the whole path as
the bench runs it -- pfd_patchmatch, the cycle check on the matched state,
the disparity filter in place, its reprojection map and a 64-slice focal
stack -- bit for bit with the oracle, field by field.

full (4080x3068, 12 neighbours, 15x15 NCC, three blurred lens types):
  * the initialisation bit for bit on a block of 2048 views, and two
    half-sweeps on that block, each started from the device's full-frame
    state (the block's pixels read neighbours outside it);
  * 10^5 per-hypothesis cost vectors bit for bit;
  * the cycle check, the disparity filter and the focal stack of the whole
    frame bit for bit, on the state after 2 iterations.
"""
import numpy as np
import pytest

import configs
from scenes import random_hypotheses

pytestmark = pytest.mark.gpu


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


def _state_equal(gpu, st, what, rows=None):
    names = ("plane", "cost", "disp", "sel")
    for name, g in zip(names, gpu):
        o = st[name]
        if rows is not None:
            g, o = g[rows], o[rows]
        if not _same(g, o):
            bad = np.nonzero(~((g == o) | (np.isnan(g) & np.isnan(o))) if g.dtype.kind == "f" else g != o)[0]
            raise AssertionError(f"{what}: {name} differs at {bad.size} entries (first {bad[:4]})")


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


def _upload(ctx, w):
    return ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)


def _checks_equal(pfd, oracle, ctx, fid, orc, st, pitch, what):
    """Cycle check, then the filter in place and its reprojection map, device
    against oracle on the same state `st` (modified in place like the frame)."""
    ccfg, fcfg = pfd.CycleCfg(), pfd.FilterCfg()
    stats, geo, pho, tm = ctx.cycle_check(fid, ccfg, pitch)
    o_stats, o_geo, o_pho, o_tm = oracle.cycle_check(orc, ccfg, pitch, st)
    assert stats["num_samples"] > 1000
    assert _same(tm, o_tm), f"{what}: {np.count_nonzero(tm != o_tm)} texture-mask pixels differ"
    assert _same(geo, o_geo), f"{what}: {np.count_nonzero(geo != o_geo)} geometric errors differ"
    assert _same(pho, o_pho), f"{what}: {np.count_nonzero(pho != o_pho)} photometric errors differ"
    for k, v in o_stats.items():
        assert stats[k] == v, f"{what}: cycle statistic {k}: device {stats[k]!r} oracle {v!r}"
    reason, fstats = ctx.filter(fid, fcfg, pitch)
    o_reason, o_fstats = oracle.filter_global(orc, fcfg, pitch, st)
    assert fstats["removed"] > 0
    assert _same(reason, o_reason), f"{what}: {np.count_nonzero(reason != o_reason)} filter reasons differ"
    assert list(fstats.values()) == [int(x) for x in o_fstats], f"{what}: filter counters {fstats} vs {o_fstats}"
    _state_equal(ctx.download(fid), st, f"{what}: filtered state")
    err = ctx.reprojection_error(fid, fcfg, pitch)
    o_err = oracle.reprojection_error(orc, fcfg, pitch, st)
    assert _same(err, o_err), f"{what}: {np.count_nonzero(err != o_err)} reprojection errors differ"


def test_small_workload_whole_path_bitexact(pfd, oracle, ctx):
    cfg = configs.SMALL
    w = configs.workload(pfd, cfg)
    P = configs.params(pfd, cfg)
    pitch, seed = cfg["pitch"], 11
    fid = _upload(ctx, w)
    try:
        ctx.patchmatch(fid, P, seed)
        eng = ctx.download(fid)
        orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
        st = orc.patchmatch(P, seed)
        _state_equal(eng, st, "patchmatch")
        valid = (st["plane"][:, 3] > 0.05) & (st["cost"] < 2.0)
        assert valid.mean() > 0.5
        dv = np.abs(configs.virtual_depth(eng[0], pitch) - configs.virtual_depth(st["plane"], pitch))[valid]
        assert np.mean(dv <= 0.01) >= 0.995
        _checks_equal(pfd, oracle, ctx, fid, orc, st, pitch, "small")
        vds = configs.slice_vds()
        ow, oh = cfg["width"] // 2, cfg["height"] // 2
        stack = ctx.refocus(fid, vds, ow, oh)
        o_stack = oracle.refocus(orc, cfg["width"], cfg["height"], vds, ow, oh)
        assert np.mean(o_stack > 0) > 0.3
        assert _same(stack, o_stack), f"{np.count_nonzero(stack != o_stack)} focal-stack pixels differ"
    finally:
        ctx.frame_free(fid)


@pytest.fixture(scope="module")
def full(pfd):
    cfg = configs.FULL
    return cfg, configs.workload(pfd, cfg)


def test_full_workload_block_init_and_sweeps_bitexact(pfd, oracle, ctx, full):
    cfg, w = full
    P = configs.params(pfd, cfg)
    V = w.centers.shape[0]
    v0 = V // 2 - 1024
    views = (v0, v0 + 2048)
    ppv = w.mi * w.mi
    rows = slice(views[0] * ppv, views[1] * ppv)
    seed = 21
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    fid = _upload(ctx, w)
    try:
        ctx.pm_init(fid, P, seed)
        eng = ctx.download(fid)
        st = orc.init(P, seed, views=views)
        _state_equal(eng, st, "init, views %d-%d" % views, rows=rows)
        for it, ph in ((0, 0), (0, 1)):
            prev = dict(zip(("plane", "cost", "disp", "sel"), (a.copy() for a in eng)))
            ctx.pm_sweep(fid, P, seed, it, ph)
            eng = ctx.download(fid)
            st = orc.sweep(P, seed, it, ph, prev, views=views)
            _state_equal(eng, st, f"half-sweep {it}.{ph}, views %d-%d" % views, rows=rows)
    finally:
        ctx.frame_free(fid)


def test_full_workload_cost_vectors_bitexact(pfd, oracle, ctx, full):
    cfg, w = full
    P = configs.params(pfd, cfg)
    V = w.centers.shape[0]
    rs = np.random.RandomState(202)
    vids, pxy, planes = random_hypotheses(rs, V, w.mi, 100000, cfg["pitch"] / 2)
    fid = _upload(ctx, w)
    try:
        gpu = ctx.ncc_costs(fid, P, vids, pxy, planes)
    finally:
        ctx.frame_free(fid)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    ref, _ = orc.cost_vectors(P, vids, pxy, planes)
    assert (ref < 2.0).mean() > 0.2
    assert _same(gpu, ref), f"{np.count_nonzero(gpu != ref)} of {gpu.size} costs differ"


def test_full_workload_checks_and_stack_bitexact(pfd, oracle, ctx, full):
    cfg, w = full
    P = configs.params(pfd, cfg, iters=2)
    pitch = cfg["pitch"]
    fid = _upload(ctx, w)
    try:
        ctx.patchmatch(fid, P, 3)
        plane, cost, disp, sel = ctx.download(fid)
        st = dict(plane=plane.copy(), cost=cost.copy(), disp=disp.copy(), sel=sel.copy())
        orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
        _checks_equal(pfd, oracle, ctx, fid, orc, st, pitch, "full")
        vds = configs.slice_vds()
        ow, oh = cfg["width"] // 2, cfg["height"] // 2
        stack = ctx.refocus(fid, vds, ow, oh)
        o_stack = oracle.refocus(orc, cfg["width"], cfg["height"], vds, ow, oh)
        assert np.mean(o_stack > 0) > 0.3
        assert _same(stack, o_stack), f"{np.count_nonzero(stack != o_stack)} focal-stack pixels differ"
    finally:
        ctx.frame_free(fid)
