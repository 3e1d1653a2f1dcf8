"""The request loop (include/pfd_serve.h): frames of different sizes, pitches,
neighbour counts and iteration counts, submitted together, run concurrently
in the server's slots, and each result must equal the same request computed
alone (pfd_frame_upload + pfd_patchmatch (+ pfd_filter) + pfd_download) bit
for bit.  Admission respects the HBM budget, and a request larger than the
budget is refused at submission."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


@pytest.fixture(scope="module")
def mix(pfd):
    specs = [(420, 320, 23.0, 6, 11, 2, 3), (300, 240, 17.5, 8, 9, 3, 5), (520, 400, 26.1, 12, 13, 1, 7),
             (360, 280, 23.2, 12, 15, 2, 11), (260, 200, 19.3, 6, 11, 4, 13), (640, 480, 23.2, 10, 11, 1, 17)]
    out = []
    for W, H, pitch, K, patch, iters, seed in specs:
        w = pfd.make_workload(W, H, pitch, 4, seed=seed, max_nb=K)
        P = pfd.PmParams(base=pitch, patch_size=patch, max_iterations=iters)
        out.append((w, P, seed, pitch))
    return out


def _alone(pfd, w, P, seed, pitch, filtered):
    with pfd.Context(0) as ctx:
        fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
        ctx.patchmatch(fid, P, seed)
        if filtered:
            ctx.filter(fid, pfd.FilterCfg(), pitch, download=False)
        st = ctx.download(fid)
        ctx.frame_free(fid)
    return st


@pytest.mark.parametrize("slots", [1, 3])
def test_results_equal_alone_and_in_the_mix(pfd, mix, slots):
    with pfd.Server(0, slots=slots) as srv:
        tickets = []
        for i, (w, P, seed, pitch) in enumerate(mix):
            fc = pfd.FilterCfg() if i % 2 else None
            tickets.append(srv.submit(w, P, seed, filter_cfg=fc, baseline_unit=pitch))
        results = [srv.wait(t, timeout_ms=120000) for t in tickets]
    for i, ((w, P, seed, pitch), r) in enumerate(zip(mix, results)):
        assert r is not None, f"request {i} timed out"
        ref = _alone(pfd, w, P, seed, pitch, filtered=bool(i % 2))
        for name, a, b in zip(("plane", "cost", "disp", "sel"), r[:4], ref):
            assert _same(a, b), f"request {i}: {name} differs"
        assert r[4] > 0.0


def test_budget_admission(pfd, mix):
    w, P, seed, pitch = mix[0]
    need = pfd.frame_bytes(w.frame.raw.shape[1], w.frame.raw.shape[0], w.centers.shape[0], w.mi, w.nb_ids.shape[1])
    with pfd.Server(0, hbm_budget=need + need // 2, slots=4) as srv:
        # room for one frame at a time: the second waits for the first
        t1 = srv.submit(w, P, seed)
        t2 = srv.submit(w, P, seed + 1)
        q, r, b = srv.load()
        assert r <= 1 and b <= need + need // 2
        assert srv.wait(t1, 120000) is not None and srv.wait(t2, 120000) is not None
        big = pfd.make_workload(1024, 768, 23.2, 4, seed=1, max_nb=12)
        with pytest.raises(pfd.PfdError) as e:
            srv.submit(big, pfd.PmParams(base=23.2), 1)
        assert e.value.code == -2
