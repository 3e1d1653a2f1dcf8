"""Regenerates tests/golden/oracle_small.npz from the CPU oracle.

Run from the repository root:  python tests/golden/make_golden.py
The fixture pins the oracle (and the synthetic generator) against unintended
change; the device tests compare the CUDA path against the same numbers.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))

from conftest import load_pfd  # noqa: E402
from scenes import random_hypotheses  # noqa: E402
from test_oracle_cpu import _digest, _golden_inputs  # noqa: E402
import pfd_oracle  # noqa: E402


def main():
    pfd = load_pfd()
    pfd_oracle.build()
    w = _golden_inputs(pfd)
    orc = pfd_oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    P = pfd.PmParams(base=23.0, patch_size=11, max_iterations=2)
    rs = np.random.RandomState(21)
    vids, pxy, planes = random_hypotheses(rs, w.centers.shape[0], w.mi, 256, 11.5)
    costs, _ = orc.cost_vectors(P, vids, pxy, planes)
    seed = 20261203
    st = orc.patchmatch(P, seed=seed)
    np.savez_compressed(
        os.path.join(HERE, "oracle_small.npz"),
        raw_sha256=_digest(w.frame.raw), nb_ids=w.nb_ids,
        hyp_vids=vids, hyp_pxy=pxy, hyp_planes=planes, hyp_costs=costs,
        seed=np.int64(seed),
        pm_plane_sha256=_digest(st["plane"]), pm_cost_sha256=_digest(st["cost"]),
        pm_sel_sha256=_digest(st["sel"]), pm_cost_sub=st["cost"][::97])
    print("wrote", os.path.join(HERE, "oracle_small.npz"))


if __name__ == "__main__":
    main()
