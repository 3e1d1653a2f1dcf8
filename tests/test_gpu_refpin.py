"""The engine against the reference's own frame kernels.

oracle/ref compiles the reference's MIStereo/CudaUtil.cu (which includes
AdaptMIPMFrame.cu) and AdaptMIPMUtil.cu from the reference tree with the
reference's flags (-O3 --use_fast_math --maxrregcount=128) for sm_100a; the
tests call them on the small (1024x768) and full (4080x3068) workloads beside
the engine:
  * per-hypothesis cost vectors (ComputeMultiViewCostVector_Frame) on the same
    (view, pixel, plane) hypotheses;
  * the initialisation and a half-sweep from one state, with the reference's
    kernels drawing the engine's Philox streams (libref_frame_philox.so), so
    both follow the same random numbers;
  * a whole run on the same stream, compared by virtual depth.
The reference's fast-math arithmetic (__expf, approximate division and square
root, compiler-chosen fused multiply-adds) differs from the engine's IEEE
canonical form in the last bits; the tests bound that difference.  With
PFD_REPORT_DIR set, the figures go to PFD_REPORT_DIR/refpin_<workload>.json.
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


CASES = {"small": (configs.SMALL, 20000), "full": (configs.FULL, 100000)}


@pytest.mark.parametrize("name", ["small", "full"])
def test_ncc_costs_against_reference_kernels(pfd, ctx, name):
    """Per-hypothesis NCC cost: the engine (reference moments, IEEE canonical
    arithmetic) against ComputeMultiViewCostVector_Frame compiled with the
    reference's fast-math flags, on the same hypotheses."""
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
        rk = ref.ncc_costs(P, vids, pxy, planes)
    k = np.arange(w.nb_ids.shape[1])[None, :] < w.nb_counts[vids][:, None]
    ve, vr = (eng < 2.0) & k, (rk < 2.0) & k
    both = ve & vr
    d = np.abs(eng[both].astype(np.float64) - rk[both])
    rep = {"hypotheses": n, "costs": int(k.sum()), "valid_both": int(both.sum()),
           "valid_engine_only": int((ve & ~vr).sum()), "valid_reference_only": int((vr & ~ve).sum()),
           "abs_diff": _quant(d), "within_1e-5": float(np.mean(d <= 1e-5)), "within_1e-4": float(np.mean(d <= 1e-4)),
           "bit_identical": float(np.mean(eng[both] == rk[both]))}
    REPORT.setdefault(name, {})["ncc"] = rep
    print(name, "ncc", json.dumps(rep))
    assert both.sum() > 0.2 * k.sum(), "too few valid costs for a meaningful check"
    # validity (anchor out of the window, weight sum, minimum variance) agrees
    assert (ve ^ vr).sum() <= 1e-4 * k.sum(), rep
    assert rep["within_1e-5"] >= 0.99, rep
    assert d.max() <= 5e-3, rep


def _vd_agreement(pe, ce, pr, cr, pitch):
    valid = (pr[:, 3] > 0.05) & (cr < 2.0)
    vde, vdr = configs.virtual_depth(pe, pitch), configs.virtual_depth(pr, pitch)
    dv = np.abs(vde[valid] - vdr[valid])
    return {"valid_frac": float(valid.mean()), "within_0.01": float(np.mean(dv <= 0.01)),
            "within_0.05": float(np.mean(dv <= 0.05)), "plane_bit_identical": float(np.mean(np.all(pe == pr, 1))),
            "cost_abs_diff": _quant(np.abs(ce[valid].astype(np.float64) - cr[valid]))}


@pytest.mark.parametrize("name", ["small", "full"])
def test_init_and_half_sweep_against_reference_kernels(pfd, ctx, name):
    """The same Philox stream on both sides: RandomInitializationForFrame and
    one CheckerboardUpdateFrame half-sweep, each started from the same state."""
    cfg, _ = CASES[name]
    w = configs.workload(pfd, cfg)
    P = configs.params(pfd, cfg)
    seed = 5
    fid = _upload(ctx, w)
    try:
        with ref_frame.RefFrame(w, philox=True) as ref:
            ctx.pm_init(fid, P, seed)
            ref.init(P, seed)
            e0 = ctx.download(fid)
            r0 = ref.download()
            rep = {"init": _vd_agreement(e0[0], e0[1], r0[0], r0[1], cfg["pitch"])}
            rep["init"]["sel_identical"] = float(np.mean(e0[3] == r0[3]))
            # one half-sweep from the engine's state on both sides
            ref.state_upload(*e0)
            ctx.pm_sweep(fid, P, seed, 0, 0)
            ref.sweep(P, seed, 0, 0)
            e1 = ctx.download(fid)
            r1 = ref.download()
            rep["half_sweep"] = _vd_agreement(e1[0], e1[1], r1[0], r1[1], cfg["pitch"])
            rep["half_sweep"]["sel_identical"] = float(np.mean(e1[3] == r1[3]))
    finally:
        ctx.frame_free(fid)
    REPORT.setdefault(name, {})["steps"] = rep
    print(name, "steps", json.dumps(rep))
    assert rep["init"]["within_0.01"] >= 0.99, rep
    assert rep["half_sweep"]["within_0.01"] >= 0.98, rep


@pytest.mark.parametrize("name", ["small", "full"])
def test_patchmatch_against_reference_kernels(pfd, ctx, name):
    """A whole run (initialisation and every iteration) on the same Philox
    stream: virtual depth of the engine against the reference's kernels."""
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
    rep = _vd_agreement(e[0], e[1], r[0], r[1], cfg["pitch"])
    rep["reference_ms"] = {"init": ms[0], "sweeps": ms[1]}
    REPORT.setdefault(name, {})["run"] = rep
    print(name, "run", json.dumps(rep))
    assert rep["valid_frac"] > 0.5, rep
    assert rep["within_0.05"] >= 0.5, rep
