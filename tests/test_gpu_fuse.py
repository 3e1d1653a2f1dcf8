"""Device parity of the virtual-depth fusion (pfd_fuse_virtual_depth,
LFRefocus::FuseVirtualDepth_BackProject, FocalStack/LFRefocus.cpp:1553-1794)
with the CPU oracle on a matched frame.  The result depends on the order in
which micro-images and pixels mask each other, so a bit-exact match of every
map and of the ordered point cloud also checks the wavefront schedule."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PITCH = 23.0
MLA_BASE = 20.7


@pytest.fixture(scope="module")
def matched(pfd):
    w = pfd.make_workload(420, 320, PITCH, 5, seed=31, max_nb=8)
    P = pfd.PmParams(base=PITCH, patch_size=11, max_iterations=2)
    lists, counts = pfd.neighbors_by_baseline(w.centers, w.tilekeys, PITCH, 24, rings=3)
    return w, P, lists, counts


def _frame(ctx, w, P):
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.patchmatch(fid, P, seed=4)
    return fid


@pytest.mark.parametrize("case", ["plain", "filtered_bgr_garbage"])
def test_fusion_matches_oracle(pfd, oracle, matched, case):
    w, P, lists, counts = matched
    V = w.centers.shape[0]
    rs = np.random.RandomState(7)
    is_ref = np.ones(V, np.uint8)
    bgr = None
    ls = lists.copy()
    if case != "plain":
        is_ref[rs.rand(V) < 0.1] = 0
        bgr = rs.randint(0, 256, size=(V, w.mi, w.mi, 3)).astype(np.uint8)
        ls[rs.rand(*ls.shape) < 0.05] = -1
    with pfd.Context(0) as ctx:
        fid = _frame(ctx, w, P)
        if case != "plain":
            ctx.filter(fid, pfd.FilterCfg(min_good_neighbors=1), PITCH)
        plane = ctx.download(fid)[0]
        vd, cf, aif, pts = ctx.fuse_virtual_depth(fid, ls, counts, is_ref, MLA_BASE, bgr=bgr)
        ctx.frame_free(fid)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    o_vd, o_cf, o_aif, o_pts = oracle.fuse_virtual_depth(orc, plane, ls, counts, is_ref, w.frame.raw.shape[1],
                                                         w.frame.raw.shape[0], MLA_BASE, bgr=bgr)
    candidates = int(np.sum(plane[:, 3] >= 1.0))
    assert len(o_pts) > 0.05 * candidates, "too few fused points for a meaningful comparison"
    assert len(o_pts) < candidates, "no pixel was masked or rejected"
    assert len(pts) == len(o_pts)
    assert np.array_equal(pts, o_pts), f"{np.count_nonzero(np.any(pts != o_pts, 1))} points differ"
    assert np.array_equal(vd, o_vd)
    assert np.array_equal(cf, o_cf)
    assert np.array_equal(aif, o_aif)


def test_fusion_errors(pfd, matched):
    w, P, lists, counts = matched
    V = w.centers.shape[0]
    with pfd.Context(0) as ctx:
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        with pytest.raises(pfd.PfdError) as e:
            ctx.fuse_virtual_depth(fid, lists, counts, np.ones(V, np.uint8), MLA_BASE)
        assert e.value.code == -7                      # no PatchMatch state yet
        ctx.pm_init(fid, P, 1)
        bad = lists.copy()
        bad[0, 0] = V
        with pytest.raises(pfd.PfdError) as e:
            ctx.fuse_virtual_depth(fid, bad, counts, np.ones(V, np.uint8), MLA_BASE)
        assert e.value.code == -1
        too_long = np.full((V, 129), -1, np.int32)
        with pytest.raises(pfd.PfdError) as e:
            ctx.fuse_virtual_depth(fid, too_long, np.zeros(V, np.int32), np.ones(V, np.uint8), MLA_BASE)
        assert e.value.code == -1
        ctx.frame_free(fid)
