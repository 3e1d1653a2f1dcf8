"""Test scenes shared by the CPU and device tests."""
import numpy as np


def value_texture(h, w, seed, cell=6):
    """Smooth integer texture 0..255 (bilinear upsampling of random lattice values)."""
    rs = np.random.RandomState(seed)
    gh, gw = h // cell + 2, w // cell + 2
    lat = rs.randint(20, 236, size=(gh, gw)).astype(np.float64)
    ys, xs = np.mgrid[0:h, 0:w] / float(cell)
    y0, x0 = np.floor(ys).astype(int), np.floor(xs).astype(int)
    ty, tx = ys - y0, xs - x0
    v = (lat[y0, x0] * (1 - tx) * (1 - ty) + lat[y0, x0 + 1] * tx * (1 - ty) +
         lat[y0 + 1, x0] * (1 - tx) * ty + lat[y0 + 1, x0 + 1] * tx * ty)
    return np.clip(np.rint(v), 0, 255).astype(np.uint8)


def fronto_parallel_scene(d0=2, base=23.0, mi=16, grid=3, seed=5):
    """A grid x grid square lattice of lenses (spacing `base`) seeing a fronto-
    parallel plane of integer disparity d0: view (gx, gy) holds
    I(l) = T(l + (gx, gy) d0), so that for every pair the reference mapping
    src = ref + (c_ref - c_nb) / base * d0 lands exactly on integer texels with
    equal values.  Returns raw frame, centres, tile keys, neighbour lists."""
    margin = 4
    Wr = int(grid * base + 2 * margin + mi)
    Hr = Wr
    T = value_texture(Hr + grid * d0 + mi, Wr + grid * d0 + mi, seed)
    raw = np.zeros((Hr, Wr), np.uint8)
    centers, keys = [], []
    for gy in range(grid):
        for gx in range(grid):
            ox, oy = margin + int(gx * base), margin + int(gy * base)
            cx, cy = ox + (mi - 1) * 0.5, oy + (mi - 1) * 0.5
            centers.append((cx, cy))
            keys.append((gx, gy))
            raw[oy:oy + mi, ox:ox + mi] = T[gy * d0:gy * d0 + mi, gx * d0:gx * d0 + mi]
    centers = np.array(centers, np.float32)
    keys = np.array(keys, np.int32)
    V = grid * grid
    K = 8
    ids = np.full((V, K), -1, np.int32)
    cnt = np.zeros(V, np.int32)
    for v in range(V):
        gx, gy = keys[v]
        n = 0
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dx == 0 and dy == 0:
                    continue
                ux, uy = gx + dx, gy + dy
                if 0 <= ux < grid and 0 <= uy < grid:
                    ids[v, n] = uy * grid + ux
                    n += 1
        cnt[v] = n
    return raw, centers, keys, ids, cnt


def slice_windows(raw, centers, mi):
    o = np.trunc((centers.astype(np.float64) - (mi - 1) * 0.5).astype(np.float32)).astype(int)
    return np.stack([raw[y:y + mi, x:x + mi] for x, y in o])


def random_hypotheses(rs, V, mi, n, dmax):
    """n random (view, pixel, plane) hypotheses: unit normals with nz >= 0.3,
    disparity uniform in [0, dmax]."""
    vids = rs.randint(0, V, n).astype(np.int32)
    pxy = rs.randint(0, mi, size=(n, 2)).astype(np.int32)
    nrm = rs.randn(n, 3)
    nrm[:, 2] = np.abs(nrm[:, 2]) + 0.3 * np.linalg.norm(nrm, axis=1)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    d = rs.uniform(0, dmax, n)
    planes = np.concatenate([nrm, d[:, None]], axis=1).astype(np.float32)
    return vids, pxy, planes
