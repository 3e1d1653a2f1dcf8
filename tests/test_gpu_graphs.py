"""CUDA graphs of pfd_patchmatch and the enqueue-only pfd_filter
(pfd_set_graphs): the first call with a key runs uncaptured, the second is
captured and replayed, later ones replay; every result equals the one without
graphs bit for bit, also after the frame gets new raw data, new neighbour
lists, a new seed, and after another frame grows the sweep scratch."""
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


def _upload(ctx, w):
    return ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)


def test_graph_replay_matches_plain_launches(pfd):
    pitch = 23.2
    w = pfd.make_workload(320, 240, pitch, 5, seed=41, max_nb=8)
    w2 = pfd.make_workload(320, 240, pitch, 5, seed=42, max_nb=8)
    big = pfd.make_workload(640, 480, pitch, 5, seed=43, max_nb=16)
    u, v = w.frame.n_cols, w.frame.n_rows
    P = pfd.PmParams(base=pitch, patch_size=13, max_iterations=2)
    fcfg = pfd.FilterCfg()
    with pfd.Context(0) as plain, pfd.Context(0) as g:
        g.set_graphs(True)
        fp, fg = _upload(plain, w), _upload(g, w)

        def step(seed, raw=None, select=False):
            for c, f in ((plain, fp), (g, fg)):
                if raw is not None:
                    c.frame_set_raw(f, raw)
                if select:
                    c.frame_select_neighbors(f, u, v, pitch)
                c.patchmatch(f, P, seed)
                c.filter(f, fcfg, pitch, download=False)
            assert _all_same(plain.download(fp), g.download(fg))

        for _ in range(4):                 # uncaptured, captured, replayed, replayed
            step(7)
        step(8)                            # a new seed: a new key
        step(8)
        step(8, raw=w2.frame.raw)          # new raw data through the same graphs
        step(8, select=True)               # new lists: the filter runs uncaptured again
        step(8)
        step(8)
        # another frame needs a larger sweep scratch: the graph holding the old one is dropped
        fb = _upload(g, big)
        g.patchmatch(fb, pfd.PmParams(base=pitch, patch_size=15, max_iterations=1), 3)
        step(8)
        step(8)
        g.frame_free(fb)
        n0 = g.launch_count()
        g.patchmatch(fg, P, 8)
        assert g.launch_count() - n0 == 1 + 2 * P.max_iterations      # a replay counts its kernels
        plain.frame_free(fp)
        g.frame_free(fg)
