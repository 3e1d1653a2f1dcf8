"""pfd_pm_sweep_noalloc: the PatchMatch half-sweep on the library's fixed scratch
array, for callers that may not allocate device memory once frames stream (an
application whose memory pool owns all free HBM, or a real-time loop in which
cudaMalloc/cudaFree, which can synchronise the device, are forbidden).

Its results must equal pfd_pm_sweep's bit for bit, the tolerance of every sweep
parity test here, on two calls in a row: the second call finds the first one's
leftovers in the shared array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


def _upload(ctx, w, blur=None):
    return ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=blur)


@pytest.mark.parametrize("pitch,K,patch,blur,mode", [(23.2, 12, 15, False, "reference"), (23.0, 6, 11, True, "reference"),
                                                     (23.2, 12, 15, False, "shifted"), (23.0, 8, 9, True, "acmm")])
def test_noalloc_sweep_matches_pfd_pm_sweep(pfd, pitch, K, patch, blur, mode):
    """Both NCC moment modes and both matchers (the sweep kernel's variants)."""
    w = pfd.make_workload(260, 200, pitch, 4, seed=5, max_nb=K)
    bl = None
    if blur:
        rs = np.random.RandomState(K)
        bl = rs.randint(0, 256, size=(w.centers.shape[0], w.mi, w.mi)).astype(np.uint8)
    P = pfd.PmParams(base=pitch, patch_size=patch, max_iterations=1)
    seed = 41
    with pfd.Context(0) as ctx:
        ctx.set_ncc_moments(mode == "shifted")
        ctx.set_matcher(mode == "acmm")
        fa = _upload(ctx, w, bl)          # pfd_pm_sweep (cudaMalloc'd scratch)
        fb = _upload(ctx, w, bl)          # pfd_pm_sweep_noalloc (fixed scratch)
        ctx.pm_init(fa, P, seed)
        ctx.pm_init(fb, P, seed)
        for phase in (0, 1):
            ctx.pm_sweep(fa, P, seed, 0, phase)
            ctx.pm_sweep_noalloc(fb, P, seed, 0, phase)
            a = ctx.download(fa)
            b = ctx.download(fb)
            for name, x, y in zip(("plane", "cost", "disp", "sel"), a, b):
                assert _same(x, y), f"call {phase + 1}: {name} differs at {np.count_nonzero(x != y)} entries"
        assert np.mean(a[1] < 2.0) > 0.3, "too few valid costs for a meaningful comparison"
        ctx.frame_free(fa)
        ctx.frame_free(fb)


def test_noalloc_sweep_takes_32_neighbours(pfd):
    """32 neighbours, the engine's maximum, need 54.7 KB of scratch per CTA
    (seven warps of cost vectors): the 8 MiB array still gives every SM of a
    B200 one CTA, and the sweep equals pfd_pm_sweep bit for bit."""
    w = pfd.make_workload(260, 200, 23.0, 4, seed=5, max_nb=32)
    P = pfd.PmParams(base=23.0, patch_size=11, max_iterations=1)
    with pfd.Context(0) as ctx:
        fa = _upload(ctx, w)
        fb = _upload(ctx, w)
        ctx.pm_init(fa, P, 1)
        ctx.pm_init(fb, P, 1)
        ctx.pm_sweep(fa, P, 1, 0, 0)
        ctx.pm_sweep_noalloc(fb, P, 1, 0, 0)
        assert all(_same(x, y) for x, y in zip(ctx.download(fa), ctx.download(fb)))
        ctx.frame_free(fa)
        ctx.frame_free(fb)


def test_noalloc_sweep_allocates_nothing(pfd):
    """On a fresh context that never ran pfd_pm_sweep, the no-alloc sweeps leave
    the context's device memory (frames and sweep scratch) and the device's free
    memory as they were, and give the results of pfd_pm_sweep on a second
    context."""
    import torch
    w = pfd.make_workload(260, 200, 23.2, 4, seed=9, max_nb=12)
    P = pfd.PmParams(base=23.2, patch_size=15, max_iterations=1)
    with pfd.Context(0) as ref:
        fr = _upload(ref, w)
        ref.pm_init(fr, P, 3)
        for phase in (0, 1):
            ref.pm_sweep(fr, P, 3, 0, phase)
        want = ref.download(fr)
        ref.frame_free(fr)
    with pfd.Context(0) as ctx:
        fb = _upload(ctx, w)
        ctx.pm_init(fb, P, 3)
        ctx.sync()
        used0 = ctx.bytes_in_use()
        free0, _ = torch.cuda.mem_get_info(0)
        for phase in (0, 1):
            ctx.pm_sweep_noalloc(fb, P, 3, 0, phase)
        ctx.sync()
        free1, _ = torch.cuda.mem_get_info(0)
        assert ctx.bytes_in_use() == used0
        assert free1 >= free0, f"free device memory fell by {free0 - free1} bytes"
        got = ctx.download(fb)
        assert all(_same(x, y) for x, y in zip(got, want))
        ctx.frame_free(fb)


def test_noalloc_sweep_counts_the_same_taps(pfd):
    """Tap counting through the fixed scratch counts what pfd_pm_sweep counts."""
    w = pfd.make_workload(260, 200, 23.2, 4, seed=13, max_nb=12)
    P = pfd.PmParams(base=23.2, patch_size=15, max_iterations=1)
    with pfd.Context(0) as ctx:
        fa = _upload(ctx, w)
        fb = _upload(ctx, w)
        ctx.pm_init(fa, P, 2)
        ctx.pm_init(fb, P, 2)
        ctx.set_tap_counting(True)
        ctx.read_tap_count()
        ctx.pm_sweep(fa, P, 2, 0, 0)
        ta = ctx.read_tap_count()
        ctx.pm_sweep_noalloc(fb, P, 2, 0, 0)
        tb = ctx.read_tap_count()
        ctx.set_tap_counting(False)
        assert ta == tb and ta > 0
        assert all(_same(x, y) for x, y in zip(ctx.download(fa), ctx.download(fb)))
        ctx.frame_free(fa)
        ctx.frame_free(fb)
