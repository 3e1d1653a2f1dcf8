"""Device parity of the ACMM matcher at one pyramid level (PFD_MATCHER_ACMM)
against the oracle's ACMM mode: initialisation, every half-sweep, the closing
post-refine pass and a full pfd_patchmatch bit for bit, with and without a blur
channel; the calibration pass counts the reference's taps, including the
write-back's evaluation of the final plane on every view; switching matchers
never reuses a stored cost vector of the other one."""
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


def _state_equal(gpu, st, what):
    plane, cost, disp, sel = gpu
    assert _same(plane, st["plane"]), f"{what}: plane differs at {np.count_nonzero(np.any(plane != st['plane'], 1))} px"
    assert _same(cost, st["cost"]), f"{what}: cost differs at {np.count_nonzero(cost != st['cost'])} px"
    assert _same(disp, st["disp"]), f"{what}: disp differs"
    assert _same(sel, st["sel"]), f"{what}: selected views differ"


@pytest.mark.parametrize("blur,patch,K", [(False, 5, 8), (True, 5, 8), (False, 11, 12)])
def test_acmm_steps_bitexact(pfd, oracle, ctx, blur, patch, K):
    pitch = 23.2
    w = pfd.make_workload(260, 200, pitch, 4, seed=40 + K, max_nb=K)
    V = w.centers.shape[0]
    bl = np.random.RandomState(K).randint(0, 256, size=(V, w.mi, w.mi)).astype(np.uint8) if blur else None
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=bl)
    P = pfd.PmParams(base=pitch, patch_size=patch, max_iterations=2, top_k=6)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=bl, acmm=True)
    seed = 21
    try:
        ctx.set_matcher(True)
        ctx.pm_init(fid, P, seed)
        st = orc.init(P, seed)
        _state_equal(ctx.download(fid), st, "acmm init")
        for it in range(2):
            for ph in range(2):
                ctx.pm_sweep(fid, P, seed, it, ph)
                st = orc.sweep(P, seed, it, ph, st)
                _state_equal(ctx.download(fid), st, f"acmm sweep {it}.{ph}")
        ctx.acmm_post_refine(fid, P)
        st = orc.acmm_post_refine(P, st)
        _state_equal(ctx.download(fid), st, "acmm post-refine")
        ctx.patchmatch(fid, P, seed)
        _state_equal(ctx.download(fid), orc.patchmatch(P, seed), "acmm patchmatch")
    finally:
        ctx.set_matcher(False)
        ctx.frame_free(fid)


def test_acmm_tap_count_and_matcher_switch(pfd, oracle, ctx):
    pitch, K = 23.2, 12
    w = pfd.make_workload(260, 200, pitch, 4, seed=44, max_nb=K)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    P = pfd.PmParams(base=pitch, patch_size=7, max_iterations=2, top_k=6)
    oac = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, acmm=True)
    ofr = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    seed = 8
    try:
        ctx.set_matcher(True)
        ctx.pm_init(fid, P, seed)
        st = oac.init(P, seed)
        ctx.set_tap_counting(True)
        ctx.read_tap_count()
        ctx.pm_sweep(fid, P, seed, 0, 0)
        dev = ctx.read_tap_count()
        ctx.set_tap_counting(False)
        st, taps = oac.sweep_taps(P, seed, 0, 0, st)
        _state_equal(ctx.download(fid), st, "acmm counted sweep")
        assert dev == taps, f"device {dev} taps, reference {taps}"
        ctx.pm_sweep(fid, P, seed, 0, 1)
        st = oac.sweep(P, seed, 0, 1, st)
        _state_equal(ctx.download(fid), st, "acmm sweep 0.1")
        # the Frame matcher from here on: no ACMM cost vector may be reused
        ctx.set_matcher(False)
        for ph in range(2):
            ctx.pm_sweep(fid, P, seed, 1, ph)
            st = ofr.sweep(P, seed, 1, ph, st)
            _state_equal(ctx.download(fid), st, f"frame sweep 1.{ph} after ACMM ones")
    finally:
        ctx.set_tap_counting(False)
        ctx.set_matcher(False)
        ctx.frame_free(fid)
