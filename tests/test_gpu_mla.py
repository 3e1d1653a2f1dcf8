"""Device micro-lens centre detection (pfd_mla_centers, DepthSolver::
ComputeMLACentersFromWhiteImage, DepthSolver.cpp:710-870) against the CPU
oracle, which tests/test_mla_cpu.py pins to OpenCV: every map entry (key,
centre, area, small-area flag) and the Otsu threshold must be equal."""
import numpy as np
import pytest

from test_mla_cpu import white_image

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("W,H,pitch,seed", [(400, 300, 23.0, 7), (1024, 768, 23.2, 3), (4080, 3068, 23.2, 11)])
def test_mla_centers_match_oracle(pfd, oracle, W, H, pitch, seed):
    if W > 2000:
        rs = np.random.RandomState(seed)
        # the full-size white image from tiles of a smaller one keeps the test fast on the CPU side
        tile, _ = white_image(1020, 767, pitch, seed, x0=pitch * 0.5 + 1.3, y0=pitch * 0.5 + 0.7)
        bgr = np.ascontiguousarray(np.tile(tile, (4, 4, 1))[:H, :W])
    else:
        bgr, _ = white_image(W, H, pitch, seed)
    u_size = int(W / pitch) + 1
    v_size = int(H / (pitch * np.sqrt(3) / 2)) + 1
    with pfd.Context(0) as ctx:
        got, t = ctx.mla_centers(bgr, pitch, u_size, v_size)
    ref, t_ref = oracle.mla_centers(bgr, pitch, u_size, v_size)
    assert t == t_ref
    assert len(ref["col"]) > 100
    for k in ("col", "row", "cx", "cy", "area", "abandon"):
        assert np.array_equal(got[k], ref[k]), k


def test_mla_centers_odd_shapes(pfd, oracle):
    """Single pixels, spurs, diagonal chains, a ring, shapes on the border."""
    import cv2
    img = np.zeros((90, 120), np.uint8)
    img[5, 5] = 200
    img[10:13, 3:12] = 200
    img[13:20, 7] = 200
    for i in range(8):
        img[25 + i, 20 + i] = 200
    cv2.circle(img, (45, 15), 9, 200, -1)
    cv2.circle(img, (45, 15), 4, 0, -1)
    img[0:6, 115:120] = 200
    img[80:90, 0:3] = 200
    for x in range(10, 110, 12):
        cv2.circle(img, (x, 60), 4, 220, -1)
    with pfd.Context(0) as ctx:
        got, t = ctx.mla_centers(img, 12.0, 10, 9)
    ref, t_ref = oracle.mla_centers(img, 12.0, 10, 9)
    assert t == t_ref
    for k in ("col", "row", "cx", "cy", "area", "abandon"):
        assert np.array_equal(got[k], ref[k]), k


def test_lattice_fit_recovers_pitch_and_origin(pfd):
    """The FP64 hexagonal lattice fit through exact synthetic centres returns
    the generating origin, pitch and angle; through detected centres of a
    white image, the pitch within 0.01 px."""
    pitch, ang = 23.2, 0.0031
    u = np.array([np.cos(ang), np.sin(ang)]) * pitch
    v = np.array([-np.sin(ang), np.cos(ang)]) * pitch * np.sqrt(3) / 2
    cols, rows = np.meshgrid(np.arange(60), np.arange(40))
    c = np.array([12.5, 9.25]) + (cols.ravel() + 0.5 * (rows.ravel() & 1))[:, None] * u + rows.ravel()[:, None] * v
    lenses = dict(col=cols.ravel(), row=rows.ravel(), cx=c[:, 0].astype(np.float32), cy=c[:, 1].astype(np.float32),
                  area=np.full(c.shape[0], 300.0, np.float32), abandon=np.zeros(c.shape[0], np.int32))
    with pfd.Context(0) as ctx:
        fit = ctx.mla_lattice_fit(lenses)
        assert abs(fit["pitch"] - pitch) < 1e-5 and abs(fit["angle"] - ang) < 1e-6
        assert abs(fit["origin"][0] - 12.5) < 1e-4 and abs(fit["origin"][1] - 9.25) < 1e-4
        assert fit["rms"] < 1e-4 and fit["used"] == c.shape[0]       # centres are float32
        bgr, _ = white_image(1024, 768, 23.2, 3)
        m, _ = ctx.mla_centers(bgr, 23.2, 45, 39)
        fit = ctx.mla_lattice_fit(m)
    assert abs(fit["pitch"] - 23.2) < 0.01 and fit["rms"] < 0.3
