"""Device parity of the PatchMatch path: the sm_100a kernels, called through the
C ABI, against the CPU oracle on the same seeded inputs."""
import ctypes
import os

import numpy as np
import pytest

from scenes import fronto_parallel_scene, random_hypotheses

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TEX_PROBE = os.path.join(ROOT, "tests", "_build", "libtexprobe.so")


def _same(a, b):
    """Bitwise equality that treats NaN payloads as equal."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f":
        return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))
    return bool(np.array_equal(a, b))


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


def test_texture_semantics(oracle):
    """tex2D with the reference's texture settings (linear filter, unnormalised
    coordinates, wrap mode, AdaptMIPMFrame.cpp:240-246) equals the emulation
    the engine and the oracle use: (x - 0.5) rounded to 1/256, clamped texels."""
    L = ctypes.CDLL(TEX_PROBE)
    L.tex_probe.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    rs = np.random.RandomState(4)
    for (h, w) in [(16, 16), (21, 21), (11, 13)]:
        img = rs.randint(0, 256, size=(h, w)).astype(np.float32)
        n = 20000
        xs = rs.uniform(0, w, n).astype(np.float32)
        ys = rs.uniform(0, h, n).astype(np.float32)
        # coordinates on and around 1/512 rounding boundaries, near the edges, tiny values
        k = np.arange(2000)
        xs[:2000] = (rs.randint(0, w * 256, 2000) + 0.5 + (k % 3 - 1) * 1e-4) / 256.0
        ys[:2000] = (rs.randint(0, h * 256, 2000) + 0.5) / 256.0
        xs[2000:2100] = np.float32(w) - rs.uniform(0, 1e-3, 100).astype(np.float32)
        xs[2100:2200] = rs.uniform(0, 1e-5, 100).astype(np.float32)
        xs = np.clip(xs, 0, np.nextafter(np.float32(w), np.float32(0)))
        ys = np.clip(ys, 0, np.nextafter(np.float32(h), np.float32(0)))
        out = np.zeros(n, np.float32)
        for mode in (0, 1):             # wrap (the reference's setting), clamp
            rc = L.tex_probe(img.ctypes.data, w, h, xs.ctypes.data, ys.ctypes.data, n, mode, out.ctypes.data)
            assert rc == 0
            emu = np.array([oracle.tex_fetch(img, float(x), float(y)) for x, y in zip(xs, ys)], np.float32)
            bad = np.nonzero(out != emu)[0]
            assert bad.size == 0, (
                f"{bad.size}/{n} mismatches (mode {mode}); first: x={xs[bad[:4]]} y={ys[bad[:4]]} "
                f"hw={out[bad[:4]]} emu={emu[bad[:4]]}")


def _workload(pfd, width=256, height=192, pitch=23.0, planes=4, seed=7, K=6, **kw):
    return pfd.make_workload(width, height, pitch, planes, seed=seed, max_nb=K, **kw)


def _upload(ctx, w, blur=None):
    return ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts, blur=blur)


@pytest.mark.parametrize("pitch,K,patch,blur", [(23.0, 6, 11, False), (23.2, 12, 15, False), (23.0, 6, 11, True),
                                                (15.0, 8, 7, False)])
def test_ncc_costs_bitexact(pfd, oracle, ctx, pitch, K, patch, blur):
    w = _workload(pfd, 300, 220, pitch, K=K, seed=int(pitch * 10) + K)
    V = w.centers.shape[0]
    rs = np.random.RandomState(K + patch)
    bl = rs.randint(0, 256, size=(V, w.mi, w.mi)).astype(np.uint8) if blur else None
    fid = _upload(ctx, w, bl)
    P = pfd.PmParams(base=pitch, patch_size=patch, sigma_spatial=3.0, sigma_color=12.0)
    vids, pxy, planes = random_hypotheses(rs, V, w.mi, 3000, pitch / 2)
    gpu = ctx.ncc_costs(fid, P, vids, pxy, planes)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts, blur=bl)
    ref, _ = orc.cost_vectors(P, vids, pxy, planes)
    ctx.frame_free(fid)
    assert (ref < 2.0).mean() > 0.2, "too few valid costs for a meaningful check"
    diff = np.abs(gpu - ref)
    assert diff.max() <= 1e-5, f"max |gpu - oracle| = {diff.max()} at {np.unravel_index(diff.argmax(), diff.shape)}"
    assert _same(gpu, ref), f"{np.count_nonzero(gpu != ref)} costs differ in the last bits"


def test_known_answer_fronto_parallel_gpu(pfd, ctx):
    raw, centers, keys, ids, cnt = fronto_parallel_scene(d0=2)
    fid = ctx.frame_upload(raw, centers, keys, 16, 16, ids, cnt)
    P = pfd.PmParams(base=23.0, patch_size=11)
    pts = np.array([(x, y) for y in range(4, 12) for x in range(4, 12)], np.int32)
    vids = np.full(len(pts), 4, np.int32)
    good = ctx.ncc_costs(fid, P, vids, pts, np.array([[0, 0, 1, 2.0]] * len(pts), np.float32))
    bad = ctx.ncc_costs(fid, P, vids, pts, np.array([[0, 0, 1, 3.0]] * len(pts), np.float32))
    ctx.frame_free(fid)
    g = good[:, :8]
    assert np.abs(g[g < 2]).max() < 1e-5
    b = bad[:, :8]
    assert np.median(b[b < 2]) > 0.01


def _state_equal(gpu, orc_state, what):
    plane, cost, disp, sel = gpu
    assert _same(plane, orc_state["plane"]), f"{what}: plane differs at {np.count_nonzero(np.any(plane != orc_state['plane'], 1))} px"
    assert _same(cost, orc_state["cost"]), f"{what}: cost differs"
    assert _same(sel, orc_state["sel"]), f"{what}: selected views differ"
    assert _same(disp, orc_state["disp"]), f"{what}: disp differs"


@pytest.mark.parametrize("pitch,K,patch", [(23.0, 6, 11), (23.2, 12, 15)])
def test_init_and_sweeps_bitexact(pfd, oracle, ctx, pitch, K, patch):
    w = _workload(pfd, 260, 200, pitch, K=K, seed=3)
    fid = _upload(ctx, w)
    P = pfd.PmParams(base=pitch, patch_size=patch, max_iterations=2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    seed = 99
    ctx.pm_init(fid, P, seed)
    st = orc.init(P, seed)
    _state_equal(ctx.download(fid), st, "init")
    for it in range(2):
        for ph in range(2):
            ctx.pm_sweep(fid, P, seed, it, ph)
            st = orc.sweep(P, seed, it, ph, st)
            _state_equal(ctx.download(fid), st, f"sweep {it}.{ph}")
    ctx.frame_free(fid)


def test_sweeps_after_state_changes_bitexact(pfd, oracle, ctx):
    """The sweep reuses the stored cost vector of each pixel's current plane.
    Every way the state can change outside the sweeps must drop that store:
    the disparity filter (rejected pixels get new planes), an uploaded state,
    and a sweep whose NCC parameters differ from the ones that made the store."""
    pitch, K = 23.2, 12
    w = _workload(pfd, 260, 200, pitch, K=K, seed=8)
    fid = _upload(ctx, w)
    P = pfd.PmParams(base=pitch, patch_size=15, max_iterations=2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    seed = 5
    ctx.pm_init(fid, P, seed)
    st = orc.init(P, seed)
    ctx.pm_sweep(fid, P, seed, 0, 0)
    st = orc.sweep(P, seed, 0, 0, st)
    _state_equal(ctx.download(fid), st, "sweep 0.0")
    # the filter rewrites rejected pixels in place
    reason, _ = ctx.filter(fid, pfd.FilterCfg(), pitch)
    assert np.count_nonzero(reason) > 100
    plane, cost, disp, sel = ctx.download(fid)
    st = dict(plane=plane.copy(), cost=cost.copy(), disp=disp.copy(), sel=sel.copy())
    for ph in (1, 0):
        ctx.pm_sweep(fid, P, seed, 1, ph)
        st = orc.sweep(P, seed, 1, ph, st)
        _state_equal(ctx.download(fid), st, f"sweep 1.{ph} after the filter")
    # an uploaded state: planes moved between pixels
    rs = np.random.RandomState(1)
    perm = rs.permutation(st["plane"].shape[0])
    up = dict(plane=st["plane"][perm].copy(), cost=st["cost"].copy(), disp=st["disp"].copy(), sel=st["sel"].copy())
    ctx.state_upload(fid, up["plane"], up["cost"], up["disp"], up["sel"])
    ctx.pm_sweep(fid, P, seed, 2, 1)
    st = orc.sweep(P, seed, 2, 1, up)
    _state_equal(ctx.download(fid), st, "sweep after an uploaded state")
    # other NCC parameters than the stored vectors were made with
    P2 = pfd.PmParams(base=pitch, patch_size=11, max_iterations=2, sigma_color=10.0)
    for ph in (0, 1):
        ctx.pm_sweep(fid, P2, seed, 3, ph)
        st = orc.sweep(P2, seed, 3, ph, st)
        _state_equal(ctx.download(fid), st, f"sweep 3.{ph} with other parameters")
    ctx.frame_free(fid)


def test_tap_count_is_the_reference_work(pfd, oracle, ctx):
    """The calibration pass (tap counting on) evaluates what the reference's
    algorithm evaluates, with none of the device's shortcuts (shared rows for
    equal planes, the stored vector of the current plane, selected views only
    for proposals and refinement, speculative proposals), so its count of
    in-bounds NCC taps, the roofline's algorithmic unit, equals the oracle's
    count for every sweep; the state stays bit-exact."""
    pitch, K = 23.2, 12
    w = _workload(pfd, 260, 200, pitch, K=K, seed=12)
    fid = _upload(ctx, w)
    P = pfd.PmParams(base=pitch, patch_size=15, max_iterations=2)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    seed = 17
    ctx.pm_init(fid, P, seed)
    st = orc.init(P, seed)
    for it in range(2):
        for ph in range(2):
            counting = (it + ph) % 2 == 1             # counting and plain sweeps interleaved
            ctx.set_tap_counting(counting)
            ctx.read_tap_count()
            ctx.pm_sweep(fid, P, seed, it, ph)
            dev_taps = ctx.read_tap_count()
            st, taps = orc.sweep_taps(P, seed, it, ph, st)
            _state_equal(ctx.download(fid), st, f"sweep {it}.{ph}")
            if counting:
                assert dev_taps == taps, f"sweep {it}.{ph}: device {dev_taps} taps, reference {taps}"
    ctx.set_tap_counting(False)
    ctx.frame_free(fid)


def test_patchmatch_virtual_depth_parity(pfd, oracle, ctx):
    """Full pfd_patchmatch (3 iterations): >= 99.5% of valid pixels within 0.01
    virtual depth of the oracle (virtual depth = pitch / disparity)."""
    pitch = 23.0
    w = _workload(pfd, 320, 240, pitch, K=6, seed=17)
    fid = _upload(ctx, w)
    P = pfd.PmParams(base=pitch, patch_size=11, max_iterations=3)
    ctx.patchmatch(fid, P, seed=5)
    plane, cost, _, _ = ctx.download(fid)
    ctx.frame_free(fid)
    st = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts).patchmatch(P, seed=5)
    d_g, d_o = plane[:, 3], st["plane"][:, 3]
    valid = (d_o > 0.05) & (st["cost"] < 2.0)
    vd_g, vd_o = pitch / np.maximum(d_g, 1e-6), pitch / np.maximum(d_o, 1e-6)
    frac = np.mean(np.abs(vd_g[valid] - vd_o[valid]) <= 0.01)
    assert valid.mean() > 0.5
    assert frac >= 0.995, f"only {frac:.4f} of valid pixels within 0.01 virtual depth"


def test_error_paths(pfd, ctx):
    P = pfd.PmParams(base=23.0)
    with pytest.raises(pfd.PfdError) as e:
        ctx.patchmatch(12345, P, 1)
    assert e.value.code == -4
    w = _workload(pfd, 200, 160, 23.0, K=6, seed=1)
    fid = _upload(ctx, w)
    with pytest.raises(pfd.PfdError) as e:
        ctx.pm_sweep(fid, P, 1, 0, 0)
    assert e.value.code == -7
    with pytest.raises(pfd.PfdError) as e:
        ctx.patchmatch(fid, pfd.PmParams(base=23.0, patch_size=10), 1)
    assert e.value.code == -1
    bad = w.centers.copy()
    bad[0] = (2.0, 2.0)                      # window leaves the frame
    with pytest.raises(pfd.PfdError) as e:
        ctx.frame_create(200, 160, bad, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    assert e.value.code == -1
    ctx.frame_free(fid)


def test_hbm_budget_enforced(pfd):
    w = _workload(pfd, 200, 160, 23.0, K=6, seed=1)
    with pfd.Context(0, hbm_budget=64 * 1024) as small:
        with pytest.raises(pfd.PfdError) as e:
            _upload(small, w)
        assert e.value.code == -2
        assert small.bytes_in_use() == 0


@pytest.mark.parametrize("K", [16, 32])
def test_neighbour_count_extremes_bitexact(pfd, oracle, ctx, K):
    """Lists of 16 (the reference's m_max_neighbors) and 32 neighbours (the
    selected-view mask width), with views that have none or one: init and a
    full iteration bit-exact with the oracle (views without neighbours keep
    their state)."""
    pitch = 23.0
    w = _workload(pfd, 300, 240, pitch, K=6, seed=50 + K)
    ids, cnt = pfd.neighbors_by_baseline(w.centers, w.tilekeys, pitch, K, rings=4)
    V = w.centers.shape[0]
    cnt = cnt.copy()
    cnt[::7] = 0
    cnt[3::11] = np.minimum(cnt[3::11], 1)
    ids = ids.copy()
    for v in range(V):
        ids[v, cnt[v]:] = -1
    assert cnt.max() == K
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, ids, cnt)
    P = pfd.PmParams(base=pitch, patch_size=9, max_iterations=1)
    orc = oracle.Oracle(w.gray, w.centers, ids, cnt)
    seed = 77
    try:
        ctx.pm_init(fid, P, seed)
        st = orc.init(P, seed)
        _state_equal(ctx.download(fid), st, f"init K={K}")
        for ph in range(2):
            ctx.pm_sweep(fid, P, seed, 0, ph)
            st = orc.sweep(P, seed, 0, ph, st)
            _state_equal(ctx.download(fid), st, f"sweep 0.{ph} K={K}")
    finally:
        ctx.frame_free(fid)
