"""Device parity of the richness channel (pfd_frame_compute_richness) against
the oracle pinned to OpenCV: the normalised GLCM score, the 8-bit channel and
the richness values bit for bit, over frames whose sides are not multiples of
the kernel's 64 x 16 tile, frames without any 8x8 window, flat frames, and a
frame of the 4080 x 3068 sensor."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


def _check(oracle, raw, centers, mi, got):
    score, binary, counts = got
    ref_s, ref_b, ref_c = oracle.richness_tiles(raw, oracle.window_origins(centers, mi, mi), mi, mi)
    assert np.array_equal(score, ref_s), f"{np.count_nonzero(score != ref_s)} scores differ"
    assert np.array_equal(binary, ref_b)
    assert np.array_equal(counts, ref_c)
    return ref_c


@pytest.mark.parametrize("Wd,Ht,pitch,K", [(300, 220, 23.0, 6), (257, 131, 15.0, 8), (190, 97, 29.5, 6)])
def test_richness_channel_bitexact(pfd, oracle, ctx, Wd, Ht, pitch, K):
    w = pfd.make_workload(Wd, Ht, pitch, 4, seed=Wd + K, max_nb=K)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    got = ctx.frame_compute_richness(fid)
    ctx.frame_free(fid)
    counts = _check(oracle, w.frame.raw, w.centers, w.mi, got)
    assert counts.sum() > 0


def _frame(ctx, raw, mi):
    """Views whose windows touch every edge of the frame, and one inside."""
    Ht, Wd = raw.shape
    h = (mi - 1) * 0.5
    centers = np.array([[h, h], [Wd - 1 - h, h], [h, Ht - 1 - h], [Wd - 1 - h, Ht - 1 - h],
                        [(Wd - 1) * 0.5, (Ht - 1) * 0.5]], np.float32)
    keys = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [2, 2]], np.int32)
    V = centers.shape[0]
    fid = ctx.frame_upload(raw, centers, keys, mi, mi, np.full((V, 1), -1, np.int32), np.zeros(V, np.int32))
    return fid, centers


@pytest.mark.parametrize("Wd,Ht,kind", [(8, 8, "random"), (40, 8, "random"), (8, 33, "random"), (9, 9, "random"),
                                        (65, 17, "random"), (70, 50, "flat"), (129, 48, "sparse")])
def test_richness_small_and_degenerate_frames(pfd, oracle, ctx, Wd, Ht, kind):
    rs = np.random.RandomState(Wd * 100 + Ht)
    if kind == "flat":
        raw = np.full((Ht, Wd), 93, np.uint8)
    elif kind == "sparse":
        raw = np.where(rs.rand(Ht, Wd) < 0.05, 255, 20).astype(np.uint8)
    else:
        raw = rs.randint(0, 256, (Ht, Wd)).astype(np.uint8)
    mi = 6
    fid, centers = _frame(ctx, raw, mi)
    got = ctx.frame_compute_richness(fid)
    ctx.frame_free(fid)
    counts = _check(oracle, raw, centers, mi, got)
    if Wd <= 8 or Ht <= 8 or kind == "flat":
        assert counts.sum() == 0 and not got[0].any()
    if kind == "sparse":
        assert 0 < counts.sum() < counts.size * mi * mi


def test_richness_full_sensor_bitexact(pfd, oracle, ctx):
    """4080 x 3068 frame (26 928 views of 16 x 16), bit-exact with the oracle (a
    few seconds of CPU); a second call gives the same channel, and the channel
    and the counts agree with the score."""
    w = pfd.make_workload(4080, 3068, 23.0, 4, seed=5, max_nb=6)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    got = ctx.frame_compute_richness(fid)
    score2, _, counts2 = ctx.frame_compute_richness(fid)
    ctx.frame_free(fid)
    score, binary, counts = got
    assert np.array_equal(score, score2) and np.array_equal(counts, counts2)
    _check(oracle, w.frame.raw, w.centers, w.mi, got)
    assert np.array_equal(binary == 255, score > 10) and set(np.unique(binary)) <= {0, 255}
    assert np.array_equal(counts, (binary == 255).reshape(len(counts), -1).sum(1))
    assert score.min() >= 0 and score.max() <= 255


def test_compute_richness_needs_a_raw_frame(pfd, ctx):
    w = pfd.make_workload(200, 160, 23.0, 4, seed=2, max_nb=4)
    V = w.centers.shape[0]
    fid = ctx.frame_create(w.frame.raw.shape[1], w.frame.raw.shape[0], w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids,
                           w.nb_counts)
    ctx.frame_set_micro_images(fid, w.gray.reshape(V, w.mi, w.mi))
    with pytest.raises(pfd.PfdError):
        ctx.frame_compute_richness(fid)
    ctx.frame_free(fid)
    with pytest.raises(KeyError):
        ctx.frame_compute_richness(fid)          # the binding knows the frame is gone
    assert ctx._L.pfd_frame_compute_richness(ctx._h, fid, None, None, None) != 0


def test_richness_leaves_the_patchmatch_state_alone(pfd, ctx):
    """The channel is not an input of the matcher: a run after it equals a run
    without it, bit for bit."""
    w = pfd.make_workload(260, 200, 23.0, 4, seed=31, max_nb=6)
    P = pfd.PmParams(base=23.0, patch_size=11, max_iterations=1)
    out = []
    for rich in (False, True):
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        ctx.pm_init(fid, P, 9)
        if rich:
            ctx.frame_compute_richness(fid)
        for ph in range(2):
            ctx.pm_sweep(fid, P, 9, 0, ph)
        out.append(ctx.download(fid))
        ctx.frame_free(fid)
    for a, b in zip(*out):
        a, b = np.asarray(a), np.asarray(b)
        assert a.tobytes() == b.tobytes()
