"""Device similarities + host selection (pfd_select_neighbors,
SelectNeighbors::CollectMIANeighImagesForMatch) against the oracle, whose
similarity tests/test_select_cpu.py pins to OpenCV: every list, in order."""
import numpy as np
import pytest

from test_select_cpu import hex_array

pytestmark = pytest.mark.gpu


def test_lists_of_a_synthetic_frame_match_oracle(pfd, oracle):
    w = pfd.make_workload(640, 480, 23.2, 6, seed=21, max_nb=6)
    u = int(w.tilekeys[:, 0].max()) + 1
    v = int(w.tilekeys[:, 1].max()) + 1
    with pfd.Context(0) as ctx:
        ids, cnt = ctx.select_neighbors(w.centers, w.tilekeys, u, v, 23.2, w.gray)
    oids, ocnt, _ = oracle.select_neighbors(w.centers, w.tilekeys, u, v, 23.2, images=w.gray)
    assert np.array_equal(cnt, np.minimum(ocnt, 128))
    assert np.array_equal(ids, oids)
    assert np.any(cnt < 90) and np.median(cnt) > 6


def test_ransac_stop_matches_oracle(pfd, oracle):
    pitch = 23.2
    c, k = hex_array(20, 18, pitch)
    V, m = len(c), 16
    rs = np.random.RandomState(5)
    pattern = np.where(rs.rand(m, m) > 0.5, 200, 40).astype(np.uint8)
    imgs = np.repeat(pattern[None], V, 0).copy()
    imgs[rs.rand(V) < 0.3] ^= 0xFF
    with pfd.Context(0) as ctx:
        ids, cnt = ctx.select_neighbors(c, k, 20, 18, pitch, imgs)
    oids, ocnt, _ = oracle.select_neighbors(c, k, 20, 18, pitch, images=imgs)
    assert np.array_equal(cnt, ocnt) and np.array_equal(ids, oids)
    assert np.any(cnt < 90)


def test_frame_selection_matches_oracle_and_becomes_the_matching_lists(pfd, oracle):
    """pfd_frame_select_neighbors on the frame's device-cut micro-images gives
    the oracle's lists, and installs their first max_nb as the frame's
    matching lists: PatchMatch on the frame then equals PatchMatch on a frame
    created with those lists; the old state is refused until re-initialised."""
    pitch, K = 23.2, 8
    w = pfd.make_workload(640, 480, pitch, 6, seed=23, max_nb=K)
    u = int(w.tilekeys[:, 0].max()) + 1
    v = int(w.tilekeys[:, 1].max()) + 1
    P = pfd.PmParams(base=pitch, patch_size=11, max_iterations=1)
    oids, ocnt, _ = oracle.select_neighbors(w.centers, w.tilekeys, u, v, pitch, images=w.gray)
    with pfd.Context(0) as ctx:
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        ctx.patchmatch(fid, P, 3)
        ctx.filter(fid, pfd.FilterCfg(), pitch)        # a filter schedule built on the old lists
        ids, cnt = ctx.frame_select_neighbors(fid, u, v, pitch, max_list=128)
        assert np.array_equal(cnt, np.minimum(ocnt, 128)) and np.array_equal(ids, oids)
        with pytest.raises(pfd.PfdError) as e:
            ctx.pm_sweep(fid, P, 3, 0, 0)
        assert e.value.code == -7
        first = np.where(np.arange(K)[None, :] < np.minimum(cnt, K)[:, None], ids[:, :K], -1).astype(np.int32)
        fcnt = np.minimum(cnt, K).astype(np.int32)
        ref = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, first, fcnt)
        for f in (fid, ref):
            ctx.patchmatch(f, P, 3)
        a, b = ctx.download(fid), ctx.download(ref)
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
        ra, sa = ctx.filter(fid, pfd.FilterCfg(), pitch)
        rb, sb = ctx.filter(ref, pfd.FilterCfg(), pitch)
        assert np.array_equal(ra, rb) and sa == sb
        assert ctx.frame_select_neighbors(fid, u, v, pitch) is None
        ctx.frame_free(fid)
        ctx.frame_free(ref)
