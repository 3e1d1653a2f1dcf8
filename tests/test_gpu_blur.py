"""Device parity of the blur channel (pfd_frame_compute_blur) against the
oracle pinned to OpenCV: the channel and the blureness values bit for bit, and
PatchMatch over a frame whose blur came from the device equal to the oracle's
run with the oracle's channel."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


@pytest.mark.parametrize("pitch,K", [(23.0, 6), (15.0, 8)])
def test_blur_channel_bitexact(pfd, oracle, ctx, pitch, K):
    w = pfd.make_workload(300, 220, pitch, 4, seed=int(pitch) + K, max_nb=K)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    tiles, counts = ctx.frame_compute_blur(fid)
    ctx.frame_free(fid)
    ref_t, ref_c = oracle.blur_tiles(w.frame.raw, oracle.window_origins(w.centers, w.mi, w.mi), w.mi, w.mi)
    assert np.array_equal(tiles, ref_t), f"{np.count_nonzero(tiles != ref_t)} blur bytes differ"
    assert np.array_equal(counts, ref_c)
    assert 0 < counts.sum() < counts.size * w.mi * w.mi


def test_blur_channel_at_frame_borders(pfd, oracle, ctx):
    """Windows that touch every edge of the frame read the reflected border."""
    rs = np.random.RandomState(3)
    Wd, Ht, mi = 40, 30, 8
    raw = rs.randint(0, 256, (Ht, Wd)).astype(np.uint8)
    h = (mi - 1) * 0.5
    centers = np.array([[h, h], [Wd - 1 - h, h], [h, Ht - 1 - h], [Wd - 1 - h, Ht - 1 - h], [19.3, 14.8]],
                       np.float32)
    keys = np.array([[0, 0], [1, 0], [0, 1], [1, 1], [2, 2]], np.int32)
    V = centers.shape[0]
    ids = np.full((V, 1), -1, np.int32)
    cnt = np.zeros(V, np.int32)
    fid = ctx.frame_upload(raw, centers, keys, mi, mi, ids, cnt)
    tiles, counts = ctx.frame_compute_blur(fid)
    ctx.frame_free(fid)
    org = oracle.window_origins(centers, mi, mi)
    assert org.min() == 0 and org[:, 0].max() + mi == Wd and org[:, 1].max() + mi == Ht
    ref_t, ref_c = oracle.blur_tiles(raw, org, mi, mi)
    assert np.array_equal(tiles, ref_t)
    assert np.array_equal(counts, ref_c)


def test_device_blur_drives_patchmatch_bitexact(pfd, oracle, ctx):
    pitch, K = 23.0, 6
    w = pfd.make_workload(260, 200, pitch, 4, seed=21, max_nb=K)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    ctx.frame_compute_blur(fid, copy_back=False)
    P = pfd.PmParams(base=pitch, patch_size=11, max_iterations=1)
    bl, _ = oracle.blur_tiles(w.frame.raw, oracle.window_origins(w.centers, w.mi, w.mi), w.mi, w.mi)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=bl)
    seed = 4
    ctx.pm_init(fid, P, seed)
    st = orc.init(P, seed)
    for ph in range(2):
        ctx.pm_sweep(fid, P, seed, 0, ph)
        st = orc.sweep(P, seed, 0, ph, st)
    plane, cost, disp, sel = ctx.download(fid)
    ctx.frame_free(fid)
    assert _same(plane, st["plane"]) and _same(cost, st["cost"])
    assert _same(disp, st["disp"]) and _same(sel, st["sel"])
    # the penalty is live: the same run without blur ends elsewhere
    orc0 = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    st0 = orc0.init(P, seed)
    assert not _same(st0["cost"], orc.init(P, seed)["cost"])


def test_compute_blur_needs_a_raw_frame(pfd, ctx):
    w = pfd.make_workload(200, 160, 23.0, 4, seed=2, max_nb=4)
    V = w.centers.shape[0]
    fid = ctx.frame_create(w.frame.raw.shape[1], w.frame.raw.shape[0], w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids,
                           w.nb_counts)
    ctx.frame_set_micro_images(fid, w.gray.reshape(V, w.mi, w.mi))
    with pytest.raises(RuntimeError):
        ctx.frame_compute_blur(fid)
    ctx.frame_free(fid)
