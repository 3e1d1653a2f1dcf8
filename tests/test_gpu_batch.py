"""The batching form: pfd_patchmatch_batch runs several frames' half-sweeps in
one persistent launch each, and every frame's result must be bit for bit what
pfd_patchmatch gives it alone -- frames of different sizes, lens pitches,
neighbour counts, patch sizes, iteration counts, with and without a blur
channel, under both matchers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


SPECS = [  # width, height, pitch, K, patch, iterations, blur
    (300, 220, 23.2, 12, 15, 2, False),
    (400, 300, 15.0, 6, 11, 1, False),
    (260, 200, 29.5, 16, 9, 3, True),
    (320, 240, 19.0, 8, 13, 2, False),
    (280, 210, 23.0, 10, 11, 2, True),
]


def _frames(pfd, ctx):
    out = []
    for i, (W, H, pitch, K, patch, iters, blur) in enumerate(SPECS):
        w = pfd.make_workload(W, H, pitch, 5, seed=60 + i, max_nb=K)
        bl = (np.random.RandomState(i).randint(0, 256, (w.centers.shape[0], w.mi, w.mi)).astype(np.uint8)
              if blur else None)
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=bl)
        P = pfd.PmParams(base=pitch, patch_size=patch, max_iterations=iters)
        out.append((fid, P, 1000 + i))
    return out


@pytest.mark.parametrize("acmm", [False, True])
def test_batch_equals_frames_alone(pfd, acmm):
    with pfd.Context(0) as ctx:
        ctx.set_matcher(acmm)
        fr = _frames(pfd, ctx)
        alone = []
        for fid, P, seed in fr:
            ctx.patchmatch(fid, P, seed)
            alone.append(ctx.download(fid))
        ids = [f for f, _, _ in fr]
        # a different order than the frames were created in, twice in a row
        order = [3, 0, 4, 1, 2]
        for rep in range(2):
            ctx.patchmatch_batch([ids[i] for i in order], [fr[i][1] for i in order], [fr[i][2] for i in order])
            for b, (fid, _, _) in enumerate(fr):
                got = ctx.download(fid)
                for name, x, y in zip(("plane", "cost", "disp", "sel"), got, alone[b]):
                    assert _same(x, y), f"rep {rep}, frame {b}: {name} differs at {np.count_nonzero(x != y)} entries"
        for fid, _, _ in fr:
            ctx.frame_free(fid)


def test_batch_rejects_bad_lists(pfd):
    with pfd.Context(0) as ctx:
        fr = _frames(pfd, ctx)[:2]
        ids = [f for f, _, _ in fr]
        with pytest.raises(pfd.PfdError):
            ctx.patchmatch_batch([ids[0], ids[0]], [fr[0][1], fr[0][1]], [1, 2])
        with pytest.raises(pfd.PfdError):
            ctx.patchmatch_batch([ids[0], 999], [fr[0][1], fr[1][1]], [1, 2])


def test_batch_with_grid_filling_frames(pfd):
    """A batch holding frames that fill the sweep's grid four times over (run as
    their own launches) and small frames (sharing launches): every frame equals
    pfd_patchmatch alone."""
    with pfd.Context(0) as ctx:
        big = pfd.make_workload(2048, 1536, 23.2, 4, seed=71, max_nb=8)
        assert big.centers.shape[0] >= 4 * 4 * 148       # four times a grid of 4 CTAs per SM on 148 SMs
        fr = _frames(pfd, ctx)[:2]
        fb = ctx.frame_upload(big.frame.raw, big.centers, big.tilekeys, big.mi, big.mi, big.nb_ids, big.nb_counts)
        fr.insert(1, (fb, pfd.PmParams(base=23.2, patch_size=11, max_iterations=1), 77))
        alone = []
        for fid, P, seed in fr:
            ctx.patchmatch(fid, P, seed)
            alone.append(ctx.download(fid))
        ctx.patchmatch_batch([f for f, _, _ in fr], [P for _, P, _ in fr], [s for _, _, s in fr])
        for b, (fid, _, _) in enumerate(fr):
            got = ctx.download(fid)
            for name, x, y in zip(("plane", "cost", "disp", "sel"), got, alone[b]):
                assert _same(x, y), f"frame {b}: {name} differs at {np.count_nonzero(x != y)} entries"
        for fid, _, _ in fr:
            ctx.frame_free(fid)
