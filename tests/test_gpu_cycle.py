"""Device parity of the cycle check: pfd_cycle_check (MICycleCheckerCPU::CheckGlobal,
CheckModule/MICycleCheck.cpp:727-893) against the CPU oracle on the same
PatchMatch state.  The texture mask and the error maps must match bit for bit,
and so must every statistic: the per-tile double sums run in the reference's
pixel order on the device and are folded in key order on the host."""
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
def frame(pfd, ctx):
    w = pfd.make_workload(360, 280, PITCH, 5, seed=29, max_nb=6)
    P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.patchmatch(fid, P, seed=8)
    yield w, fid
    ctx.frame_free(fid)


CFGS = {
    "reference_call": {},                                   # MIStereoMatch.cpp:570-583
    "gated_clamped": dict(pixel_gate_enabled=True, gate_use_clamped=True, gate_geo_px=1.0, gate_photo_u=1.5),
    "unclamped_or_mask": dict(clamp_geo=False, clamp_photo=False, use_and=False, max_triplet=6),
}


@pytest.mark.parametrize("name", list(CFGS))
@pytest.mark.parametrize("filtered", [False, True])
def test_cycle_check_matches_oracle(pfd, oracle, ctx, frame, name, filtered):
    w, fid = frame
    cfg = pfd.CycleCfg(**CFGS[name])
    if filtered:
        # a fresh copy of the matched state, filtered: invalidated pixels take the NaN-free paths
        P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        ctx.patchmatch(fid, P, seed=8)
        ctx.filter(fid, pfd.FilterCfg(min_good_neighbors=1), PITCH)
    stats, geo, pho, tm = ctx.cycle_check(fid, cfg, PITCH)
    plane, cost, disp, sel = ctx.download(fid)
    if filtered:
        ctx.frame_free(fid)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    st = dict(plane=plane, cost=cost, disp=disp, sel=sel)
    o_stats, o_geo, o_pho, o_tm = oracle.cycle_check(orc, cfg, PITCH, st)
    assert stats["num_samples"] > 1000
    assert _same(tm, o_tm), f"{np.count_nonzero(tm != o_tm)} texture-mask pixels differ"
    assert _same(geo, o_geo), f"{np.count_nonzero(geo != o_geo)} geometric errors differ"
    assert _same(pho, o_pho), f"{np.count_nonzero(pho != o_pho)} photometric errors differ"
    for k, v in o_stats.items():
        assert stats[k] == v, f"{k}: device {stats[k]!r} oracle {v!r}"


def test_cycle_check_is_read_only_and_repeatable(pfd, ctx, frame):
    w, fid = frame
    before = ctx.download(fid)
    a = ctx.cycle_check(fid, pfd.CycleCfg(), PITCH)
    b = ctx.cycle_check(fid, pfd.CycleCfg(), PITCH, maps=False)
    after = ctx.download(fid)
    assert all(_same(x, y) for x, y in zip(before, after))
    assert a[0] == b[0] and b[1] is None


def test_enqueued_cycle_check_folds_the_same_statistics(pfd, ctx, frame):
    """Enqueued without outputs, the check does not synchronise; its
    statistics, folded later by pfd_cycle_check_stats (here after a filter has
    changed the state behind it), are the ones of the state it saw."""
    w, fid = frame
    cfg = pfd.CycleCfg()
    sync_stats = ctx.cycle_check(fid, cfg, PITCH, maps=False)[0]
    P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
    other = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.patchmatch(other, P, seed=8)
    assert ctx.cycle_check(other, cfg, PITCH, maps=False, stats=False) is None
    ctx.filter(other, pfd.FilterCfg(), PITCH, download=False)
    assert ctx.cycle_check_stats(other) == sync_stats
    ctx.frame_free(other)
    fresh = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    with pytest.raises(pfd.PfdError) as e:
        ctx.cycle_check_stats(fresh)
    assert e.value.code == -7
    ctx.frame_free(fresh)


def test_cycle_check_errors(pfd, ctx, frame):
    w, fid = frame
    with pytest.raises(pfd.PfdError) as e:
        ctx.cycle_check(fid, pfd.CycleCfg(), -1.0)
    assert e.value.code == -1
    fresh = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    with pytest.raises(pfd.PfdError) as e:
        ctx.cycle_check(fresh, pfd.CycleCfg(), PITCH)
    assert e.value.code == -7
    ctx.frame_free(fresh)
