"""Virtual-to-real depth oracle (FocalStack/LFRefocus.cpp:2515-2593,
FocalStack/VirtualToRealDepthFunc.cpp:3390-3450): known answers and a check of
the behavioural-model fit against numpy's SVD least squares, the route
cv::solve(DECOMP_SVD) takes in the reference."""
import numpy as np
import pytest

import pfd_oracle


@pytest.fixture(scope="module")
def orc_lib():
    pfd_oracle.build()
    return pfd_oracle


def test_point_form_known_answers(orc_lib):
    c = (0.0, 2.0, 5.0)                    # z = 2 v + 5
    v = np.array([0.0, 1.0, 2.5, 12.0], np.float32)
    assert np.array_equal(pfd_oracle.vd_to_rd_points(v, c), (2 * v + 5).astype(np.float32))
    # denominator 1 - v c0 within 1e-12 of zero: 0; negative depth: 0; NaN input: 0
    c = (0.5, 1.0, 0.0)                    # z = v / (1 - v / 2)
    out = pfd_oracle.vd_to_rd_points(np.array([2.0, 3.0, np.nan, 1.0], np.float32), c)
    assert out[0] == 0.0 and out[1] == 0.0 and out[2] == 0.0
    assert out[3] == np.float32(1.0 / 0.5)


def test_map_form_is_ieee(orc_lib):
    c = (0.5, 1.0, 0.0)
    out = pfd_oracle.vd_to_rd_map(np.array([2.0, 1.0, 4.0, np.inf], np.float32), c)
    # 2 -> 2 / 0 = inf -> 0 (no near-zero test in the map form); 4 -> 4 / -1 -> negative -> 0
    assert list(out) == [0.0, 2.0, 0.0, 0.0]
    v = np.linspace(2, 12, 101).astype(np.float32)
    c = (0.01, 3.0, -1.5)
    vv = v.astype(np.float64)
    ref = (vv * c[1] + c[2]) / (1.0 - vv * c[0])
    assert np.array_equal(pfd_oracle.vd_to_rd_map(v, c), ref)


def test_segments(orc_lib):
    segs = np.array([[2.0, 5.0, 0.0, 1.0, 0.0], [5.0, 9.0, 0.0, 2.0, 0.0], [9.0, 20.0, 0.0, 3.0, 1.0]])
    v = np.array([1.0, 2.0, 4.99, 5.0, 8.5, 9.0, 25.0], np.float32)
    out = pfd_oracle.vd_to_rd_segments(v, segs)
    exp = np.array([0.0, 2.0, np.float32(4.99), 10.0, 17.0, 28.0, 0.0], np.float32)
    assert np.array_equal(out, exp)


def test_behavioral_fit_recovers_model(orc_lib):
    rs = np.random.RandomState(3)
    c_true = np.array([-0.02, 40.0, 80.0])
    v = rs.uniform(2, 12, 5000).astype(np.float32)
    vv = v.astype(np.float64)
    aL = ((vv * c_true[1] + c_true[2]) / (1 - vv * c_true[0])).astype(np.float32)
    c = pfd_oracle.behavioral_fit(aL, v)
    X = np.stack([aL.astype(np.float64) * vv, vv, np.ones_like(vv)], 1)
    c_svd = np.linalg.lstsq(X, aL.astype(np.float64), rcond=None)[0]
    assert np.allclose(c, c_svd, rtol=1e-8, atol=1e-10)
    assert np.allclose(c, c_true, rtol=1e-4)
