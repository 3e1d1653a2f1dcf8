"""Device parity of the virtual-to-real depth conversion (FP64): the map, point
and segmented forms match the oracle bit for bit; the behavioural-model fit
matches it to the conditioning of the 3x3 normal equations (relative 1e-9)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


def _vd(n, seed):
    rs = np.random.RandomState(seed)
    v = rs.uniform(2, 12, n).astype(np.float32)
    v[:7] = [0.0, np.nan, np.inf, -np.inf, -3.0, 1e30, 2.0]        # specials; 2.0 hits 1 - v c0 = 0 below
    return v


@pytest.mark.parametrize("n", [1, 3, 4, 1000, 1 << 20])
def test_map_matches_oracle(pfd, oracle, ctx, n):
    c = (0.5, 3.0, -1.5) if n > 7 else (0.01, 3.0, -1.5)
    v = _vd(max(n, 8), n)[:n]
    got = ctx.vd_to_rd_map(v, c)
    ref = oracle.vd_to_rd_map(v, c)
    assert got.dtype == np.float64 and np.array_equal(got, ref)


def test_points_and_segments_match_oracle(pfd, oracle, ctx):
    v = _vd(200003, 7)
    c = (0.5, 3.0, -1.5)
    assert np.array_equal(ctx.vd_to_rd_points(v, c), oracle.vd_to_rd_points(v, c))
    segs = np.array([[2.0, 5.0, 0.01, 1.0, 0.5], [5.0, 9.0, -0.02, 2.0, 0.0], [9.0, 20.0, 0.5, 3.0, 1.0],
                     [-5.0, 2.0, 0.0, -1.0, 0.0]])
    assert np.array_equal(ctx.vd_to_rd_segments(v, segs), oracle.vd_to_rd_segments(v, segs))


def test_device_arrays(pfd, ctx):
    import torch
    v = _vd(1 << 16, 9)
    c = (0.01, 3.0, -1.5)
    vt = torch.from_numpy(v).cuda()
    out = torch.empty(v.shape[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctx.vd_to_rd_map_device(vt.data_ptr(), v.shape[0], c, out.data_ptr())
    ctx.sync()
    assert np.array_equal(out.cpu().numpy(), ctx.vd_to_rd_map(v, c))


def test_behavioral_fit(pfd, oracle, ctx):
    rs = np.random.RandomState(5)
    c_true = np.array([-0.02, 40.0, 80.0])
    v = rs.uniform(2, 12, 300000).astype(np.float32)
    vv = v.astype(np.float64)
    aL = ((vv * c_true[1] + c_true[2]) / (1 - vv * c_true[0]) * (1 + rs.normal(0, 1e-3, v.shape))).astype(np.float32)
    got = ctx.fit_behavioral_model(aL, v)
    ref = oracle.behavioral_fit(aL, v)
    assert np.allclose(got, ref, rtol=1e-9, atol=0)
    with pytest.raises(pfd.PfdError) as e:
        ctx.fit_behavioral_model(aL[:2], v[:2])
    assert e.value.code == -1
