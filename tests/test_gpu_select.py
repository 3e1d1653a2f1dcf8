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
