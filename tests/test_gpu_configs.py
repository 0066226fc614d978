"""Parity on the workloads the benchmark specification names, at their
sizes (the oracle is the C restatement pinned to the reference by
tests/test_oracle.py):

* 2D 128^2 single crystal with a centre seed of radius 4, O supplied at the
  x=0 face, Cr 0.20 +- 0.005 (seeded noise outside the seed, the inlet
  column keeps its value), legacy Ck and bounds: the full 2000 steps, every
  field bit for bit and the budget.
* 3D 128^3 with 32 static Voronoi grains from seed 1 (grain diameter 50),
  Cr 0.22 +- 0.005, Ksp insertion on: 100 steps bit for bit (the full
  2000-step run takes the single-threaded oracle minutes; the GPU path
  is the same kernels at every step).
* The same 3D grid made supersaturated (O = 0.001 everywhere, the
  reference's own trick for exercising insertion) with a short nucleation
  period, so that ordered insertion across the periodic seams is active.
"""
import numpy as np
import pytest

import nicr
from oracle import Oracle, make_config
from parity import assert_bitexact, assert_budget

pytestmark = pytest.mark.gpu


def noisy(shape, base, amp, seed):
    return base + np.random.default_rng(seed).uniform(-amp, amp, size=shape)


def inject_both(sol, orc, o, cr, p, eta=None):
    sol.set_fields(o, cr, p, eta)
    orc.set_fields(o, cr, p, eta)
    sol.reset_inventory()
    orc.reset_inventory()


def compare(sol, orc, fields=("o", "cr", "p", "gb")):
    for f in fields:
        assert_bitexact(f, sol.get(f), orc.get(f))
    assert_budget(sol.budget(), orc.budget())


def test_2d_128_centre_seed_2000_steps(require_gpu):
    cfg = make_config(2, nx=128, ny=128, grains=0, nucleation="center", radius_grid=4.0, bc="concentration",
                      ck="legacy", bounds="legacy")
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p = orc.get("o"), orc.get("cr"), orc.get("p")
    noise = noisy(cr.shape, 0.20, 0.005, 0)
    keep = p > 0.5
    keep[0, :] = True                       # the inlet column keeps layerCr
    cr = np.where(keep, cr, noise)
    inject_both(sol, orc, o, cr, p)
    rc, done = orc.run(2000)
    assert rc == 0 and done == 2000
    sol.run(2000)
    compare(sol, orc, ("o", "cr", "p"))
    orc.refresh()
    for f in ("muO", "muCr", "mo", "mc"):
        assert_bitexact(f, sol.get(f), orc.get(f))


def grains_128(**kw):
    base = dict(nx=128, ny=128, nz=128, grains=1, grain_diameter_grid=50., random_seed=1, bc="concentration",
                ck="legacy", bounds="legacy", nucleation="ksp")
    base.update(kw)
    return make_config(3, **base)


def test_3d_128_32_grains(require_gpu):
    cfg = grains_128()
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    assert sol.info().n_seeds == 32
    assert_bitexact("grain", sol.get("grain"), orc.get("grain"))
    o, cr, p = orc.get("o"), orc.get("cr"), orc.get("p")
    cr = np.where(np.arange(128)[:, None, None] == 0, cr, noisy(cr.shape, 0.22, 0.005, 1))
    inject_both(sol, orc, o, cr, p)
    rc, done = orc.run(100)
    assert rc == 0 and done == 100
    sol.run(100)
    compare(sol, orc)


def test_3d_128_supersaturated_ksp(require_gpu):
    cfg = grains_128(dt=1e-12, nucleation_period=2e-11, radius_grid=2.5)
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o = np.full(orc.shape, 0.001)
    cr = orc.get("cr")
    cr = np.where(np.arange(128)[:, None, None] == 0, cr, noisy(cr.shape, 0.22, 0.005, 4))
    inject_both(sol, orc, o, cr, orc.get("p"))
    assert sol.stamp(64, 1, 1) == orc.stamp(64, 1, 1)        # across both periodic seams
    rc, done = orc.run(60)
    assert rc == 0 and done == 60
    sol.run(60)
    compare(sol, orc)
    assert sol.budget()["nuclei"] > 1
