"""Device parity of the focal-stack render: pfd_refocus against the oracle's
orc_refocus (itself checked against a brute-force numpy form), bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(pfd):
    c = pfd.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("size,pitch,out,vds", [
    ((360, 280), 23.0, (180, 140), [1.0, 2.0, 3.7, 6.0, 9.5, 12.0, 14.0]),
    ((512, 384), 23.2, (256, 192), list(np.linspace(2.0, 12.0, 8))),
    ((300, 220), 15.0, (97, 83), [2.5, 11.0]),               # ragged tiles, small pitch
    ((300, 220), 29.0, (300, 220), [4.0]),                   # full resolution
])
def test_refocus_matches_oracle(pfd, oracle, ctx, size, pitch, out, vds):
    W, H = size
    w = pfd.make_workload(W, H, pitch, 4, seed=int(pitch * 7), max_nb=6)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    got = ctx.refocus(fid, vds, out[0], out[1])
    again = ctx.refocus(fid, vds, out[0], out[1])
    ctx.frame_free(fid)
    orc = oracle.Oracle(w.gray, w.centers, w.nb_ids, w.nb_counts)
    ref = oracle.refocus(orc, W, H, vds, out[0], out[1])
    assert np.mean(ref > 0) > 0.3
    bad = np.nonzero(got != ref)
    assert bad[0].size == 0, f"{bad[0].size} pixels differ, first {list(zip(*[b[:3] for b in bad]))}"
    assert np.array_equal(got, again)


def test_refocus_errors(pfd, ctx):
    w = pfd.make_workload(300, 220, 23.0, 4, seed=3, max_nb=6)
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    for bad in ([0.0], [-1.0], [float("nan")], []):
        with pytest.raises(pfd.PfdError) as e:
            ctx.refocus(fid, bad, 64, 64)
        assert e.value.code == -1
    ctx.frame_free(fid)
    # a virtual depth so large that one output tile sees more lenses (about
    # 4 000 here) than the kernel gathers (2 048): refused, context usable after
    w = pfd.make_workload(1024, 768, 15.0, 4, seed=3, max_nb=6)
    assert w.centers.shape[0] > 2048
    fid = ctx.frame_upload(w.frame.raw, w.centers, w.tilekeys, w.mi, w.mi, w.nb_ids, w.nb_counts)
    with pytest.raises(pfd.PfdError) as e:
        ctx.refocus(fid, [400.0], 512, 384)
    assert e.value.code == -1 and "lenses" in str(e.value)
    assert ctx.refocus(fid, [4.0], 512, 384).shape == (1, 384, 512)
    ctx.frame_free(fid)
