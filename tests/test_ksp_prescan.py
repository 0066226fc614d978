"""The Ksp pre-scan's exclusion test (valid_nucleus on the pre-scan state,
mpi3d-slab/NiCr3D_grains.cpp:687-703) as the CUDA path computes it in 3D: an
exact separable distance transform (k_ksp_edt_z, k_ksp_edt_y and the x pass of
k_ksp_candidates_edt in csrc/nicr_ksp.cu), restated here in numpy and checked
against the reference's box search on random occupancy, including axes
shorter than the search box (both offsets of a wrapped cell are visited) and
candidates near the x ends. CPU only."""
import math

import numpy as np
import pytest


def bounded_reach(radius, n):
    """3S:220: the whole axis when the radius reaches it, else ceil(radius)."""
    return n if radius >= n else int(math.ceil(radius))


def min_image(d, n):
    """3S:172, with C's round (half away from zero)."""
    q = d / n
    r = math.floor(abs(q) + 0.5) * (1 if q >= 0 else -1)
    return d - n * r


def periodic_range(c, radius, n):
    """3S:221-231 (1-based): the cells of the periodic neighbourhood."""
    r = bounded_reach(radius, n)
    if 2 * r + 1 >= n:
        return list(range(1, n + 1))
    lo, hi = c - r, c + r
    if lo < 1:
        return list(range(1, hi + 1)) + list(range(lo + n, n + 1))
    if hi > n:
        return list(range(1, hi - n + 1)) + list(range(lo, n + 1))
    return list(range(lo, hi + 1))


def reference_excluded(occ, x, y, z, limit):
    """True when an occupied cell of the box lies at sqrt(d^2) < limit (the
    reference's search, with its early exit on the first hit)."""
    nx, ny, nz = occ.shape
    sr = bounded_reach(limit, nx)
    for i in range(max(1, x - sr), min(nx, x + sr) + 1):
        for j in periodic_range(y, limit, ny):
            for k in periodic_range(z, limit, nz):
                if occ[i - 1, j - 1, k - 1]:
                    di, dj, dk = float(i - x), min_image(float(j - y), ny), min_image(float(k - z), nz)
                    if math.sqrt(di * di + dj * dj + dk * dk) < limit:
                        return True
    return False


INF = 1 << 29


def edt_excluded(occ, limit):
    """The CUDA path's three passes: the least offset^2 over the occupied
    cells within reach along z (periodic), then y (periodic), then x (within
    [1, nx]); excluded when sqrt of that least sum is below the limit."""
    nx, ny, nz = occ.shape
    Rz, Ry, Rx = bounded_reach(limit, nz), bounded_reach(limit, ny), bounded_reach(limit, nx)
    dz = np.full(occ.shape, INF, dtype=np.int64)
    for d in range(-Rz, Rz + 1):
        shifted = np.roll(occ, -d, axis=2)        # occ at column k + d (wrapped)
        dz = np.where(shifted, np.minimum(dz, d * d), dz)
    dyz = np.full(occ.shape, INF, dtype=np.int64)
    for d in range(-Ry, Ry + 1):
        v = np.roll(dz, -d, axis=1)
        dyz = np.where(v < INF, np.minimum(dyz, v + d * d), dyz)
    best = np.full(occ.shape, INF, dtype=np.int64)
    for d in range(-Rx, Rx + 1):
        lo, hi = max(0, -d), min(nx, nx - d)       # cells whose x + d lies inside the domain
        if lo >= hi:
            continue
        v = dyz[lo + d:hi + d]
        cur = best[lo:hi]
        best[lo:hi] = np.where(v < INF, np.minimum(cur, v + d * d), cur)
    return (best < INF) & (np.sqrt(best.astype(np.float64)) < limit)


@pytest.mark.parametrize("shape,limit,density,seed", [
    ((24, 20, 18), 8.5, 0.002, 1),     # the default r + gap
    ((24, 20, 18), 8.5, 0.03, 2),
    ((30, 7, 9), 8.5, 0.01, 3),        # y and z shorter than the box: whole axes, wrapped twice
    ((12, 16, 5), 3.5, 0.05, 4),
    ((20, 12, 12), 6.0, 0.02, 5),      # an integer limit: sqrt(36) < 6 is false
    ((9, 9, 9), 2.5, 0.1, 6),
])
def test_distance_transform_matches_box_search(shape, limit, density, seed):
    rng = np.random.default_rng(seed)
    occ = rng.random(shape) < density
    got = edt_excluded(occ, limit)
    nx, ny, nz = shape
    cells = [(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)]
    pick = rng.choice(len(cells), size=min(len(cells), 600), replace=False)
    for q in pick:
        i, j, k = cells[q]
        assert got[i, j, k] == reference_excluded(occ, i + 1, j + 1, k + 1, limit), (i, j, k)
