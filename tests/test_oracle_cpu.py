"""The CPU oracle of the PatchMatch path: known answers, FP64 agreement, and
the committed golden fixtures (oracle regression pins)."""
import hashlib
import os

import numpy as np
import pytest

from scenes import fronto_parallel_scene, random_hypotheses, slice_windows

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_known_answer_fronto_parallel(pfd, oracle):
    """A fronto-parallel plane at the true disparity matches exactly (cost ~ 0);
    other disparities cost more."""
    d0 = 2
    raw, centers, keys, ids, cnt = fronto_parallel_scene(d0=d0)
    gray = slice_windows(raw, centers, 16)
    orc = oracle.Oracle(gray, centers, ids, cnt)
    P = pfd.PmParams(base=23.0, patch_size=11)
    vid = 4                                    # the centre lens sees all 8 neighbours
    pts = [(x, y) for y in range(4, 12) for x in range(4, 12)]
    for d, expect_zero in [(2.0, True), (1.0, False), (3.0, False), (2.5, False)]:
        planes = np.array([[0, 0, 1, d]] * len(pts), np.float32)
        costs, _ = orc.cost_vectors(P, np.full(len(pts), vid), np.array(pts), planes)
        c = costs[:, :cnt[vid]]
        valid = c < 2.0
        assert valid.mean() > 0.9
        if expect_zero:
            assert np.abs(c[valid]).max() < 1e-5
        else:
            assert np.median(c[valid]) > 0.01


def test_oracle_ncc_agrees_with_fp64(pfd, oracle):
    """FP32 canonical NCC vs an FP64 NCC with exact bilinear sampling: the only
    differences are float rounding and the 8-bit texture weights."""
    w = pfd.make_workload(256, 192, 23.0, 4, seed=3, max_nb=6)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    P = pfd.PmParams(base=23.0, patch_size=11)
    rs = np.random.RandomState(2)
    vids, pxy, planes = random_hypotheses(rs, w.centers.shape[0], w.mi, 400, 11.5)
    costs, _ = orc.cost_vectors(P, vids, pxy, planes)
    diffs = []
    for i in range(len(vids)):
        for k in range(int(w.nb_counts[vids[i]])):
            c32 = costs[i, k]
            c64 = orc.ncc_fp64(P, int(vids[i]), k, int(pxy[i, 0]), int(pxy[i, 1]), planes[i])
            if c32 < 2.0 and c64 < 2.0:
                diffs.append(abs(c32 - c64))
    diffs = np.array(diffs)
    assert len(diffs) > 500
    assert np.median(diffs) < 5e-3          # 8-bit texture weights dominate
    assert np.percentile(diffs, 99) < 0.05


def _golden_inputs(pfd):
    w = pfd.make_workload(208, 160, 23.0, 3, seed=11, max_nb=6)
    return w


def _digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_golden_oracle_regression(pfd, oracle):
    """The oracle reproduces the fixtures committed in tests/golden (generated by
    tests/golden/make_golden.py): synthetic input bytes, cost vectors of fixed
    hypotheses, and the full PatchMatch state."""
    path = os.path.join(GOLDEN, "oracle_small.npz")
    if not os.path.exists(path):
        pytest.skip("golden fixture not generated")
    g = np.load(path)
    w = _golden_inputs(pfd)
    assert _digest(w.frame.raw) == str(g["raw_sha256"])
    assert np.array_equal(w.nb_ids, g["nb_ids"])
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    P = pfd.PmParams(base=23.0, patch_size=11, max_iterations=2)
    costs, _ = orc.cost_vectors(P, g["hyp_vids"], g["hyp_pxy"], g["hyp_planes"])
    assert np.array_equal(costs, g["hyp_costs"])
    st = orc.patchmatch(P, seed=int(g["seed"]))
    assert _digest(st["plane"]) == str(g["pm_plane_sha256"])
    assert _digest(st["cost"]) == str(g["pm_cost_sha256"])
    assert _digest(st["sel"]) == str(g["pm_sel_sha256"])
    assert np.array_equal(st["cost"][::97], g["pm_cost_sub"])
