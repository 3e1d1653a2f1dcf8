"""The engine against the reference's own frame kernels.

oracle/ref compiles the reference's MIStereo/CudaUtil.cu (which includes
AdaptMIPMFrame.cu) and AdaptMIPMUtil.cu from the reference tree for sm_100a:
with the reference's flags (-O3 --use_fast_math --maxrregcount=128), and a
second time without --use_fast_math (IEEE division, square root and expf).
The tests run them beside the engine on the small (1024x768) and full
(4080x3068) workloads:
  * per-hypothesis cost vectors (ComputeMultiViewCostVector_Frame) on the
    same (view, pixel, plane) hypotheses;
  * the initialisation and one half-sweep started from the same state, with
    the reference's kernels drawing the engine's Philox streams, so all sides
    follow the same random numbers;
  * a whole run on the same stream, compared by virtual depth and by its error
    against the scene's true virtual depth.
The engine computes the reference's algorithm in IEEE single precision in a
fixed canonical order (bit-exact with the CPU oracle); the reference's build
uses fast-math division, square root and exp and lets the compiler fuse
multiply-adds.  The bounds below are the measured gap; each comparison is
stated beside the gap between the reference's two builds, which is the
reference's own sensitivity to its arithmetic.  With PFD_REPORT_DIR set, the
figures go to PFD_REPORT_DIR/refpin_<workload>.json.
"""
import json
import os
import sys

import numpy as np
import pytest

import configs
from scenes import random_hypotheses

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ref_frame  # noqa: E402

REPORT = {}


@pytest.fixture(scope="module")
def ctx(pfd):
    if not ref_frame.available():
        pytest.fail("oracle/_ref is not built: make -C oracle/ref (needs the reference tree)")
    c = pfd.Context(0)
    yield c
    c.close()
    out = os.environ.get("PFD_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        for name, rep in REPORT.items():
            with open(os.path.join(out, f"refpin_{name}.json"), "w") as fh:
                json.dump(rep, fh, indent=1)


def _upload(ctx, w):
    return ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)


def _quant(x):
    x = np.asarray(x, np.float64)
    if x.size == 0:
        return {}
    return {"max": float(x.max()), "p50": float(np.percentile(x, 50)), "p99": float(np.percentile(x, 99)),
            "p999": float(np.percentile(x, 99.9))}


def _cost_gap(a, b, k):
    va, vb = (a < 2.0) & k, (b < 2.0) & k
    both = va & vb
    d = np.abs(a[both].astype(np.float64) - b[both])
    return {"valid_both": int(both.sum()), "valid_first_only": int((va & ~vb).sum()),
            "valid_second_only": int((vb & ~va).sum()), "abs_diff": _quant(d),
            "within_1e-5": float(np.mean(d <= 1e-5)), "within_1e-4": float(np.mean(d <= 1e-4)),
            "bit_identical": float(np.mean(a[both] == b[both]))}


CASES = {"small": (configs.SMALL, 20000), "full": (configs.FULL, 100000)}


@pytest.mark.parametrize("name", ["small", "full"])
def test_ncc_costs_against_reference_kernels(pfd, ctx, name):
    """Per-hypothesis NCC cost: the engine (reference moments, IEEE canonical
    arithmetic) against ComputeMultiViewCostVector_Frame of the reference's
    build, beside the reference's IEEE build against its own."""
    cfg, n = CASES[name]
    w = configs.workload(pfd, cfg)
    P = configs.params(pfd, cfg)
    V = w.centers.shape[0]
    rs = np.random.RandomState(101)
    vids, pxy, planes = random_hypotheses(rs, V, w.mi, n, cfg["pitch"] / 2)
    fid = _upload(ctx, w)
    try:
        eng = ctx.ncc_costs(fid, P, vids, pxy, planes)
    finally:
        ctx.frame_free(fid)
    with ref_frame.RefFrame(w, philox=False) as ref:
        fast = ref.ncc_costs(P, vids, pxy, planes)
    with ref_frame.RefFrame(w, ieee=True) as ref:
        ieee = ref.ncc_costs(P, vids, pxy, planes)
    k = np.arange(w.nb_ids.shape[1])[None, :] < w.nb_counts[vids][:, None]
    rep = {"hypotheses": n, "costs": int(k.sum()), "engine_vs_reference": _cost_gap(eng, fast, k),
           "reference_ieee_vs_reference": _cost_gap(ieee, fast, k), "engine_vs_reference_ieee": _cost_gap(eng, ieee, k)}
    REPORT.setdefault(name, {})["ncc"] = rep
    print(name, "ncc", json.dumps(rep))
    g = rep["engine_vs_reference"]
    assert g["valid_both"] > 0.2 * k.sum(), "too few valid costs for a meaningful check"
    # validity (anchor out of the window, weight sum, minimum variance) agrees
    assert g["valid_first_only"] + g["valid_second_only"] <= 1e-4 * k.sum(), g
    assert g["abs_diff"]["p50"] <= 1e-5 and g["abs_diff"]["p99"] <= 1e-4, g
    assert g["within_1e-4"] >= 0.995, g


def _vd_agreement(pe, ce, pr, cr, pitch, rows=None):
    valid = (pr[:, 3] > 0.05) & (cr < 2.0)
    if rows is not None:
        valid &= rows
    vde, vdr = configs.virtual_depth(pe, pitch), configs.virtual_depth(pr, pitch)
    dv = np.abs(vde[valid] - vdr[valid])
    return {"valid_frac": float(valid.mean()), "within_0.01": float(np.mean(dv <= 0.01)),
            "within_0.05": float(np.mean(dv <= 0.05)),
            "plane_bit_identical": float(np.mean(np.all(pe[valid] == pr[valid], 1))),
            "cost_abs_diff": _quant(np.abs(ce[valid].astype(np.float64) - cr[valid]))}


def _updated(w, phase):
    mi = w.mi
    ys, xs = np.mgrid[0:mi, 0:mi]
    colour = (((xs + ys) & 1) == phase).reshape(-1)
    return np.tile(colour, w.centers.shape[0])


@pytest.mark.parametrize("name", ["small", "full"])
def test_init_and_half_sweep_against_reference_kernels(pfd, ctx, name):
    """The same Philox stream on all sides: RandomInitializationForFrame, and
    one CheckerboardUpdateFrame half-sweep started from the engine's
    initialised state, compared on the pixels it updates."""
    cfg, _ = CASES[name]
    w = configs.workload(pfd, cfg)
    P = configs.params(pfd, cfg)
    seed = 5
    upd = _updated(w, 0)
    fid = _upload(ctx, w)
    rep = {}
    try:
        ctx.pm_init(fid, P, seed)
        e0 = ctx.download(fid)
        ctx.pm_sweep(fid, P, seed, 0, 0)
        e1 = ctx.download(fid)
        for tag, ieee in (("reference", False), ("reference_ieee", True)):
            with ref_frame.RefFrame(w, philox=True, ieee=ieee) as ref:
                ref.init(P, seed)
                r0 = ref.download()
                ref.state_upload(*e0)
                ref.sweep(P, seed, 0, 0)
                r1 = ref.download()
            rep["init_engine_vs_" + tag] = _vd_agreement(e0[0], e0[1], r0[0], r0[1], cfg["pitch"])
            rep["half_sweep_engine_vs_" + tag] = _vd_agreement(e1[0], e1[1], r1[0], r1[1], cfg["pitch"], upd)
            rep["half_sweep_engine_vs_" + tag]["sel_identical"] = float(np.mean(e1[3][upd] == r1[3][upd]))
            if ieee:
                rep["half_sweep_reference_ieee_vs_reference"] = _vd_agreement(r1[0], r1[1], rf1[0], rf1[1],
                                                                              cfg["pitch"], upd)
            else:
                rf1 = r1
    finally:
        ctx.frame_free(fid)
    REPORT.setdefault(name, {})["steps"] = rep
    print(name, "steps", json.dumps(rep))
    assert rep["init_engine_vs_reference"]["within_0.01"] >= 0.999, rep
    assert rep["half_sweep_engine_vs_reference"]["within_0.01"] >= 0.99, rep


@pytest.mark.parametrize("name", ["small", "full"])
def test_patchmatch_against_reference_kernels(pfd, ctx, name):
    """A whole run (initialisation and every iteration) on the same Philox
    stream.  A random search diverges on any changed cost bit, so the depth
    maps are compared to each other (beside the reference's two builds on the
    small workload) and each against the scene's true virtual depth: the
    engine's depth error must match the reference's."""
    cfg, _ = CASES[name]
    w = configs.workload(pfd, cfg)
    P = configs.params(pfd, cfg)
    seed = 5
    fid = _upload(ctx, w)
    try:
        ctx.patchmatch(fid, P, seed)
        e = ctx.download(fid)
    finally:
        ctx.frame_free(fid)
    with ref_frame.RefFrame(w, philox=True) as ref:
        ms = ref.patchmatch(P, seed)
        r = ref.download()
    vd_map = pfd.synth_vd_map(w.frame)
    rep = {"engine_vs_reference": _vd_agreement(e[0], e[1], r[0], r[1], cfg["pitch"]),
           "reference_ms": {"init": ms[0], "sweeps": ms[1]},
           "depth_error_engine": pfd.depth_error(w, e[0], vd_map, cost=e[1]),
           "depth_error_reference": pfd.depth_error(w, r[0], vd_map, cost=r[1])}
    if name == "small":
        with ref_frame.RefFrame(w, ieee=True) as ref:
            ref.patchmatch(P, seed)
            ri = ref.download()
        rep["reference_ieee_vs_reference"] = _vd_agreement(ri[0], ri[1], r[0], r[1], cfg["pitch"])
        rep["depth_error_reference_ieee"] = pfd.depth_error(w, ri[0], vd_map, cost=ri[1])
    REPORT.setdefault(name, {})["run"] = rep
    print(name, "run", json.dumps(rep))
    de, dr = rep["depth_error_engine"], rep["depth_error_reference"]
    assert rep["engine_vs_reference"]["valid_frac"] > 0.5, rep
    assert abs(de["matched"] - dr["matched"]) <= 0.01, rep
    assert de["median_abs"] <= 1.05 * dr["median_abs"] + 0.01, rep
    assert de["within_0.5"] >= dr["within_0.5"] - 0.01, rep
