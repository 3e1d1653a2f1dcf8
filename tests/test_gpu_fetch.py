"""Where the half-sweep reads neighbour samples (pfd_set_sweep_fetch).

FETCH_SHARED (the default) stages the tiles in shared memory and blends them
as the texture unit does; FETCH_TEXTURE fetches them with tex2DLayered from
the frame's micro-images held as layered float textures, as the reference's
tex2D does.  Both equal the CPU oracle bit for bit, with and without the blur
channel and under either moment mode; the textures follow new tiles (new
micro-images, a new raw frame) before the next sweep; a batch and a graph
replay read them like a single call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


def _check(got, want, what):
    for name, g in zip(("plane", "cost", "disp", "sel"), got):
        assert _same(g, want[name]), f"{what}: {name} differs ({np.count_nonzero(np.asarray(g) != want[name])})"


@pytest.mark.parametrize("fetch", [0, 1])
@pytest.mark.parametrize("blur,shifted", [(False, False), (True, False), (False, True), (True, True)])
def test_fetch_modes_match_the_oracle(pfd, oracle, fetch, blur, shifted):
    pitch = 23.2
    w = pfd.make_workload(300, 220, pitch, 4, seed=23 + 2 * blur + shifted, max_nb=12)
    V = w.centers.shape[0]
    bl = np.random.RandomState(5).randint(0, 256, size=(V, w.mi, w.mi)).astype(np.uint8) if blur else None
    P = pfd.PmParams(base=pitch, patch_size=15, max_iterations=2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=bl, shifted=shifted)
    want = orc.patchmatch(P, seed=8)
    with pfd.Context(0) as ctx:
        ctx.set_sweep_fetch(fetch)
        ctx.set_ncc_moments(shifted)
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=bl)
        ctx.patchmatch(fid, P, 8)
        _check(ctx.download(fid), want, f"fetch {fetch}")
        ctx.frame_free(fid)


def test_textures_follow_new_tiles(pfd, oracle):
    """New micro-images, then a new raw frame: each next PatchMatch reads the
    new tiles, with graphs on (the refill runs before the replay)."""
    pitch = 23.0
    a = pfd.make_workload(320, 240, pitch, 4, seed=41, max_nb=8)
    b = pfd.make_workload(320, 240, pitch, 5, seed=42, max_nb=8)
    assert np.array_equal(a.centers, b.centers)
    P = pfd.PmParams(base=pitch, patch_size=11, max_iterations=2)
    want_a = oracle.Oracle(a.gray, a.centers, a.nb_ids, a.nb_counts).patchmatch(P, seed=3)
    want_b = oracle.Oracle(b.gray, a.centers, a.nb_ids, a.nb_counts).patchmatch(P, seed=3)
    with pfd.Context(0) as ctx:
        ctx.set_sweep_fetch(pfd.FETCH_TEXTURE)
        ctx.set_graphs(True)
        fid = ctx.frame_upload(a.frame.raw, a.centers, a.tilekeys, a.mi, a.mi, a.nb_ids, a.nb_counts)
        for rep in range(3):                       # uncaptured, captured, replayed
            ctx.frame_set_micro_images(fid, b.gray)
            ctx.patchmatch(fid, P, 3)
            _check(ctx.download(fid), want_b, f"micro-images, call {rep}")
            ctx.frame_set_raw(fid, a.frame.raw)
            ctx.patchmatch(fid, P, 3)
            _check(ctx.download(fid), want_a, f"raw frame, call {rep}")
        ctx.frame_free(fid)


def test_batch_reads_textures(pfd, oracle):
    """A batch of two frames (one with a blur channel) under texture fetches
    equals each frame alone under shared-memory fetches."""
    pitch = 23.2
    works = [pfd.make_workload(300, 220, pitch, 4, seed=s, max_nb=12) for s in (61, 62)]
    bl = np.random.RandomState(9).randint(0, 256, size=(works[1].centers.shape[0], works[1].mi,
                                                         works[1].mi)).astype(np.uint8)
    blurs = [None, bl]
    P = pfd.PmParams(base=pitch, patch_size=15, max_iterations=2)
    want = []
    with pfd.Context(0) as ref:
        ref.set_sweep_fetch(pfd.FETCH_SHARED)
        for w, b in zip(works, blurs):
            f = ref.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=b)
            ref.patchmatch(f, P, 12)
            want.append(ref.download(f))
            ref.frame_free(f)
    with pfd.Context(0) as ctx:
        ctx.set_sweep_fetch(pfd.FETCH_TEXTURE)
        fids = [ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=b)
                for w, b in zip(works, blurs)]
        ctx.patchmatch_batch(fids, [P, P], [12, 12])
        for f, wnt in zip(fids, want):
            got = ctx.download(f)
            assert all(_same(x, y) for x, y in zip(got, wnt))
            ctx.frame_free(f)


def test_fetch_mode_errors(pfd):
    with pfd.Context(0) as ctx:
        for bad in (2, -1):
            with pytest.raises(pfd.PfdError) as e:
                ctx.set_sweep_fetch(bad)
            assert e.value.code == -1
