"""Coloured eta initialisation (nicr_config.eta_colours = K, an extension: the
reference keeps one eta per Voronoi grain, 3S:469-494). The Voronoi grains
are coloured into K eta fields from their face adjacency (DSatur), and every
cell gets tanh profiles across its nearest bisector. Checked against a numpy
restatement on a small grid (labels from a static-grain handle with the same
seeds, pinned to the reference elsewhere), in the slab form, and on the
benchmark's shape (64 seeds coloured into 8 eta)."""
import math

import numpy as np
import pytest

import nicr
from parity import assert_bitexact, assert_budget

pytestmark = pytest.mark.gpu


def cfg3(**kw):
    base = dict(nx=20, ny=16, nz=12, grains=1, grain_evolution=1, grain_diameter_grid=5.5, random_seed=7,
                bc="concentration", ck="legacy", bounds="legacy", nucleation="off", eta_colours=4)
    base.update(kw)
    return nicr.make_config(3, **base)


def c_round(x):
    """C round(): halves away from zero."""
    return np.trunc(x + np.copysign(0.5, x))


def min_image(d, period):
    return d - period * c_round(d / period)


def nearest_bisector(seeds, owner, shape):
    """Distance to the nearest bisector and its competitor per cell, in the
    operation order of the initialisation kernel (3S:395-406)."""
    nx, ny, nz = shape
    i, j, k = np.indices(shape).astype(float)
    x, y, z = (i + 1) - .5, (j + 1) - .5, (k + 1) - .5
    ng = len(seeds)
    yy = min_image(seeds[owner, 1] - y, float(ny))
    zz = min_image(seeds[owner, 2] - z, float(nz))
    ax = seeds[owner, 0] - x
    rbest = ax * ax + yy * yy + zz * zz
    oy, oz = y + yy, z + zz
    db = np.full(shape, np.inf)
    comp = np.full(shape, -1)
    np.seterr(invalid="ignore", divide="ignore")   # sep == 0 for the owner's own images: masked below
    for s in range(ng):
        d = np.full(shape, np.inf)
        for im in (-1, 0, 1):
            for jm in (-1, 0, 1):
                gy, gz = seeds[s, 1] + im * ny, seeds[s, 2] + jm * nz
                bx_, by_, bz_ = seeds[s, 0] - x, gy - y, gz - z
                rs = bx_ * bx_ + by_ * by_ + bz_ * bz_
                sx, sy, sz = seeds[s, 0] - seeds[owner, 0], gy - oy, gz - oz
                sep = np.sqrt(sx * sx + sy * sy + sz * sz)
                cand = np.maximum(0., (rs - rbest) / (2. * sep))
                d = np.where((sep > 1e-14) & (cand < d), cand, d)
        d = np.where(owner == s, np.inf, d)
        better = d < db
        comp = np.where(better, s, comp)
        db = np.where(better, d, db)
    return db, comp


def adjacency(owner, ng):
    adj = np.zeros((ng, ng), dtype=bool)
    for axis, periodic in ((0, False), (1, True), (2, True)):
        a = owner
        b = np.roll(owner, -1, axis=axis)
        if not periodic:
            a, b = np.take(owner, range(owner.shape[0] - 1), axis=0), np.take(owner, range(1, owner.shape[0]), axis=0)
        m = a != b
        adj[a[m], b[m]] = True
        adj[b[m], a[m]] = True
    return adj


def dsatur(adj, k):
    ng = len(adj)
    colour = [-1] * ng
    degree = adj.sum(axis=1)
    for _ in range(ng):
        best, bsat = -1, -1
        for a in range(ng):
            if colour[a] >= 0:
                continue
            sat = len({colour[b] for b in range(ng) if adj[a, b] and colour[b] >= 0})
            if best < 0 or sat > bsat or (sat == bsat and degree[a] > degree[best]):
                best, bsat = a, sat
        count = [0] * k
        for b in range(ng):
            if adj[best, b] and colour[b] >= 0:
                count[colour[b]] += 1
        colour[best] = min(range(k), key=lambda q: (count[q], q))
    return colour


def h(p):
    return p * p * p * (10. - 15. * p + 6. * p * p)


@pytest.mark.parametrize("k", [4, 64])
def test_coloured_init_matches_restatement(require_gpu, k):
    cfg = cfg3(eta_colours=k)
    sol = nicr.Solver(cfg)
    static = nicr.Solver(cfg3(grain_evolution=0, eta_colours=0))
    seeds, _ = sol.seeds()
    ng = len(seeds)
    assert sol.n_eta == k and ng > k // 2
    owner = static.get("grain").astype(int) - 1
    db, comp = nearest_bisector(seeds, owner, sol.shape)
    adj = adjacency(owner, ng)
    colour = dsatur(adj, k)
    if k >= ng:   # enough colours: no two adjacent grains share one
        assert not any(adj[a, b] and colour[a] == colour[b] for a in range(ng) for b in range(ng))
    metal = 1. - h(sol.get("p"))
    want = np.zeros((k,) + sol.shape)
    ca = np.array(colour)[owner]
    cb = np.where(comp >= 0, np.array(colour)[np.maximum(comp, 0)], -1)
    t = np.tanh(db)
    same = (cb < 0) | (cb == ca)
    idx = np.indices(sol.shape)
    want[(ca,) + tuple(idx)] = np.where(same, metal, metal * (.5 * (1. + t)))
    other = ~same
    want[(cb[other],) + tuple(ix[other] for ix in idx)] = (metal * (.5 * (1. - t)))[other]
    for c in range(k):
        got = sol.get("eta", c)
        assert np.max(np.abs(got - want[c])) <= 4.5e-16, c   # 2 ulps: numpy tanh vs the C library
    # cell sums: the metal fraction, at most two nonzero fields per cell
    stack = np.stack([sol.get("eta", c) for c in range(k)])
    assert np.max(np.abs(stack.sum(axis=0) - metal)) <= 4e-16
    assert (np.count_nonzero(stack, axis=0) <= 2).all()
    sol.close()
    static.close()


def test_coloured_init_in_slabs(require_gpu):
    cfg = cfg3(nx=40, nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12, exclusion_gap_grid=2.,
               eta_colours=6)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 3) as s:
        for g in range(6):
            assert_bitexact(f"eta{g + 1} initial", s.get("eta", g), solo.get("eta", g))
        assert_bitexact("gb initial", s.get("gb"), solo.get("gb"))
        s.run(12)
        solo.run(12)
        for f in ("o", "cr", "p", "gb"):
            assert_bitexact(f, s.get(f), solo.get(f))
        for g in range(6):
            assert_bitexact(f"eta{g + 1}", s.get("eta", g), solo.get("eta", g))
        assert_budget(s.budget(), solo.budget())
    solo.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp64-fast"])
def test_bench_shape_64_seeds_8_colours(require_gpu, precision):
    """64 seeds coloured into 8 eta on a 64^3 grid (the benchmark's grain
    density at a quarter of its edge) run 60 steps on the run() schedule."""
    n = 64
    d = (6.0 * n ** 3 / (math.pi * 64)) ** (1.0 / 3.0)
    cfg = nicr.make_config(3, nx=n, ny=n, nz=n, grains=1, grain_evolution=1, random_seed=2, grain_diameter_grid=d,
                           bc="concentration", ck="legacy", bounds="legacy", nucleation="ksp", eta_colours=8,
                           precision=precision)
    sol = nicr.Solver(cfg)
    seeds, vol = sol.seeds()
    assert len(seeds) == 64 and sol.n_eta == 8 and vol.sum() == n ** 3
    rc, done = sol.run(60)
    assert rc == 0 and done == 60
    e = np.stack([sol.get("eta", g) for g in range(8)])
    assert e.min() >= -1e-12 and e.max() <= 1 + 1e-12
    sol.close()
