"""The oracle's ACMM matcher (one pyramid level of AdaptMIPMFrameACMM) on the
CPU: its write-back stores what RecomputeSupportCostDisp_Frame computes from
the final plane, which makes the closing PostRefineMetadataFrame pass change
nothing, and it differs from the Frame matcher only where the reference's
files differ (blur gain, write-back)."""
import numpy as np
import pytest


def _topk(costs, nc, top_k):
    """ComputeSelectedViewsTopK_Frame (AdaptMIPMFrameACMM.cu:196-232) in numpy."""
    c = costs[:nc].astype(np.float32)
    valid = c < 2.0
    if not valid.any():
        return np.float32(2.0), 0
    k = min(int(valid.sum()), top_k)
    s = np.sort(c)[:k]
    m = np.float32(0.0)
    for v in s:
        m = np.float32(m + v)
    mask = 0
    for i in range(nc):
        if c[i] <= s[k - 1]:
            mask |= 1 << i
    return np.float32(m / np.float32(k)), mask


@pytest.fixture(scope="module")
def scene(pfd):
    w = pfd.make_workload(240, 180, 23.0, 4, seed=13, max_nb=8)
    rs = np.random.RandomState(2)
    blur = rs.randint(0, 256, size=(w.centers.shape[0], w.mi, w.mi)).astype(np.uint8)
    return w, blur


@pytest.mark.parametrize("with_blur", [False, True])
def test_acmm_write_back_is_the_top_k_of_the_final_plane(pfd, oracle, scene, with_blur):
    w, blur = scene
    bl = blur if with_blur else None
    P = pfd.PmParams(base=23.0, patch_size=5, max_iterations=1, top_k=6)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=bl, acmm=True)
    st = orc.init(P, 7)
    st = orc.sweep(P, 7, 0, 0, st)
    n = st["cost"].shape[0]
    ppv = w.mi * w.mi
    rs = np.random.RandomState(5)
    pix = rs.choice(np.nonzero((np.arange(n) % ppv // w.mi + np.arange(n) % w.mi) % 2 == 0)[0], 300, replace=False)
    vids = (pix // ppv).astype(np.int32)
    pxy = np.stack([pix % ppv % w.mi, pix % ppv // w.mi], 1).astype(np.int32)
    costs, _ = orc.cost_vectors(P, vids, pxy, st["plane"][pix])
    for i, t in enumerate(pix):
        nc = int(w.nb_counts[vids[i]])
        m, mask = _topk(costs[i], nc, 6)
        assert st["cost"][t] == m and int(st["sel"][t]) == mask


def test_acmm_post_refine_changes_nothing(pfd, oracle, scene):
    w, blur = scene
    P = pfd.PmParams(base=23.0, patch_size=5, max_iterations=2, top_k=6)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=blur, acmm=True)
    st = orc.init(P, 3)
    for it in range(2):
        for ph in range(2):
            st = orc.sweep(P, 3, it, ph, st)
    again = orc.acmm_post_refine(P, st)
    for k in ("plane", "cost", "disp", "sel"):
        assert np.array_equal(again[k], st[k], equal_nan=(k != "sel")), k
    full = orc.patchmatch(P, 3)
    for k in ("plane", "cost", "sel"):
        assert np.array_equal(full[k], st[k]), k


def test_acmm_differs_from_frame_only_through_its_rules(pfd, oracle, scene):
    w, blur = scene
    P = pfd.PmParams(base=23.0, patch_size=5, max_iterations=1, top_k=6)
    fr = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    ac = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, acmm=True)
    # without a blur channel the initialisations agree (same draws, no penalty)
    a, b = fr.init(P, 9), ac.init(P, 9)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=(k != "sel")), k
    # with one, the 0.8 gain changes the costs
    frb = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=blur)
    acb = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=blur, acmm=True)
    assert not np.array_equal(frb.init(P, 9)["cost"], acb.init(P, 9)["cost"])
    # after a sweep the stored costs are top-k means, not weighted costs
    sa, sb = fr.sweep(P, 9, 0, 0, a), ac.sweep(P, 9, 0, 0, b)
    assert not np.array_equal(sa["cost"], sb["cost"])
