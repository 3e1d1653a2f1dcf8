"""Launch shapes of the half-sweep and the autotuner (pfd_set_sweep_shape).

Every shape (warps per CTA, CTAs per SM) computes the same state bit for bit:
init + iterations in each fixed shape equal the CPU oracle; under
PFD_SHAPE_AUTOTUNE the first half-sweep of a new key is run in every shape
(trials with the stored cost vectors neither read nor written) and the result
equals the default shape's, frame by frame and in a batch; the chosen shape is
recorded per key."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


def _all_same(x, y):
    return all(_same(a, b) for a, b in zip(x, y))


@pytest.mark.parametrize("shape", [0, 1, 2, 3])
def test_every_shape_matches_the_oracle(pfd, oracle, shape):
    pitch = 23.2
    w = pfd.make_workload(300, 220, pitch, 4, seed=19, max_nb=12)
    P = pfd.PmParams(base=pitch, patch_size=15, max_iterations=2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    st = orc.patchmatch(P, seed=4)
    with pfd.Context(0) as ctx:
        ctx.set_sweep_shape(shape)
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        ctx.patchmatch(fid, P, 4)
        got = ctx.download(fid)
        ctx.frame_free(fid)
    for name, g in zip(("plane", "cost", "disp", "sel"), got):
        assert _same(g, st[name]), f"shape {shape}: {name} differs"


def test_shape_info_and_errors(pfd):
    seen = set()
    for s in range(pfd.SWEEP_SHAPES):
        warps, ctas = pfd.sweep_shape_info(s)
        assert 1 <= warps <= 32 and 1 <= ctas <= 8
        seen.add((warps, ctas))
    assert len(seen) == pfd.SWEEP_SHAPES
    with pytest.raises(ValueError):
        pfd.sweep_shape_info(pfd.SWEEP_SHAPES)
    with pfd.Context(0) as ctx:
        for bad in (pfd.SWEEP_SHAPES, -2):
            with pytest.raises(pfd.PfdError) as e:
                ctx.set_sweep_shape(bad)
            assert e.value.code == -1


def test_autotune_gives_the_default_result(pfd):
    """Two keys (different windows and neighbour counts): tuned once each, the
    state after every half-sweep equal to shape 0's, then a batch of both."""
    cases = [(23.2, 12, 15, 31), (16.0, 8, 11, 32)]
    works = [pfd.make_workload(320, 240, p, 5, seed=s, max_nb=K) for p, K, _, s in cases]
    params = [pfd.PmParams(base=p, patch_size=ps, max_iterations=2) for p, _, ps, _ in cases]
    with pfd.Context(0) as ref, pfd.Context(0) as tuned:
        tuned.set_sweep_shape(pfd.SHAPE_AUTOTUNE)
        want = []
        for w, P in zip(works, params):
            fr = ref.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
            ft = tuned.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
            ref.pm_init(fr, P, 9)
            tuned.pm_init(ft, P, 9)
            for it in range(2):
                for ph in range(2):
                    ref.pm_sweep(fr, P, 9, it, ph)
                    tuned.pm_sweep(ft, P, 9, it, ph)
                    assert _all_same(ref.download(fr), tuned.download(ft)), f"sweep {it}.{ph}"
            assert 0 <= tuned.tuned_sweep_shape(ft, P) < pfd.SWEEP_SHAPES
            want.append(ref.download(fr))
            ref.frame_free(fr)
            tuned.frame_free(ft)
        # a batch under the tuned shapes
        fids = [tuned.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
                for w in works]
        tuned.patchmatch_batch(fids, params, [9, 9])
        for f, wnt in zip(fids, want):
            assert _all_same(tuned.download(f), wnt)
            tuned.frame_free(f)
