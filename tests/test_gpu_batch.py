"""Batched multi-domain form (nicr_batch_*). Every domain of a batch must
evolve exactly as its own handle would: same fields bit for bit, same
accepted-step counts, nuclei, clipped cells and error messages; budget sums
to 1e-13 relative (the batch gives all its domains one X chunk, so the
per-CTA partial sums group differently than in a lone handle). Solo handles
are pinned to the oracle by test_gpu_parity.py; one batch domain is also
checked against the oracle directly."""
import numpy as np
import pytest

import nicr
from nicr.sweep import sweep_configs
from oracle import Oracle
from parity import assert_bitexact, assert_budget, compare_state, smooth_fields

pytestmark = pytest.mark.gpu

BASE = dict(bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12)


def mixed_configs():
    """Uneven 3D sweep domains (own Ksp, Cr, O supply, grain count), evolving
    eta in both arithmetic forms, a single crystal, and 2D domains."""
    cfgs = sweep_configs(4, seed=11, edges=(20, 33, 40), **BASE)
    cfgs.append(nicr.make_config(3, nx=24, ny=19, nz=35, grains=1, grain_evolution=1, grain_diameter_grid=10.,
                                 bc="mu", **BASE))
    cfgs.append(nicr.make_config(3, nx=24, ny=19, nz=35, grains=1, grain_evolution=1, grain_diameter_grid=10.,
                                 bc="mu", precision=1, **BASE))
    cfgs.append(nicr.make_config(3, nx=17, ny=16, nz=9, grains=0, bc="closed", ck="off", **BASE))
    cfgs.append(nicr.make_config(2, nx=61, ny=45, grains=1, grain_diameter_grid=12., bc="concentration", **BASE))
    cfgs.append(nicr.make_config(2, nx=33, ny=140, grains=1, grain_evolution=1, grain_diameter_grid=12., bc="mu",
                                 **BASE))
    return cfgs


def inject(sol, seed):
    o, cr, p, eta = smooth_fields(sol.shape, sol.n_eta, seed=seed)
    sol.set_fields(o, cr, p, eta if eta else None)
    sol.reset_inventory()


def assert_same_domain(a, b, label):
    for f in ("o", "cr", "p", "gb"):
        assert_bitexact(f"{label} {f}", a.get(f), b.get(f))
    for g in range(a.n_eta):
        assert_bitexact(f"{label} eta{g + 1}", a.get("eta", g), b.get("eta", g))
    assert_budget(a.budget(), b.budget())
    assert a.info().steps_done == b.info().steps_done, label


@pytest.mark.parametrize("mode", ["run", "step"])
def test_batch_matches_separate_handles(require_gpu, mode):
    cfgs = mixed_configs()
    solo = [nicr.Solver(c) for c in cfgs]
    with nicr.Batch(cfgs) as b:
        for i, (s, d) in enumerate(zip(solo, b.domains)):
            inject(s, 100 + i)
            inject(d, 100 + i)
            assert_same_domain(d, s, f"domain {i} initial")
        for chunk in (7, 1, 12):
            if mode == "run":
                done, rc = b.run(chunk)
                for s in solo:
                    s.run(chunk)
            else:
                done, rc = b.step(chunk)
                for s in solo:
                    s.step(chunk)
            assert rc == 0 and done == [chunk] * len(cfgs)
        for i, (s, d) in enumerate(zip(solo, b.domains)):
            assert_same_domain(d, s, f"domain {i}")
        if mode == "run":
            assert sum(d.budget()["nuclei"] for d in b.domains) > 0
        # fewer launches than the separate handles needed for the same steps
        assert b.kernel_launches < sum(nicr.lib().nicr_kernel_launches(s.h) for s in solo)
    for s in solo:
        s.close()


def test_batch_domain_matches_oracle(require_gpu):
    cfgs = mixed_configs()[:3]
    orc = Oracle(cfgs[1])
    with nicr.Batch(cfgs) as b:
        for i, d in enumerate(b.domains):
            inject(d, 7 + i)
        o, cr, p, _ = smooth_fields(orc.shape, 0, seed=8)
        orc.set_fields(o, cr, p)
        orc.reset_inventory()
        done, rc = b.run(20)
        assert rc == 0
        rc2, done2 = orc.run(20)
        assert rc2 == 0 and done2 == 20
        compare_state(b.domains[1], orc)


def test_failing_domain_stops_alone(require_gpu):
    cfgs = mixed_configs()[:3]
    cfgs[1].bounds = nicr._abi.BOUNDS["stop"]
    solo = nicr.Solver(cfgs[1])
    with nicr.Batch(cfgs) as b:
        for i, d in enumerate(b.domains):
            inject(d, 30 + i)
        inject(solo, 31)
        cr = b.domains[1].get("cr")
        cr[15, 5, 4] = -0.1
        for s in (b.domains[1], solo):
            s.set("cr", cr)
        before = b.domains[1].get("o")
        done, rc = b.run(5, check=False)
        rc_solo, done_solo = solo.run(5, check=False)
        assert rc_solo == nicr._abi.ERR_TRIAL_BOUNDS and done_solo == 0
        assert rc == nicr._abi.ERR_TRIAL_BOUNDS
        assert done == [5, 0, 5]
        assert b.last_error == "domain 1: " + solo.last_error
        assert b.domains[1].last_error == solo.last_error
        assert_bitexact("o after rejection", b.domains[1].get("o"), before)
        assert_same_domain(b.domains[1], solo, "failed domain")
    solo.close()


def test_more_domains_than_one_launch_holds(require_gpu):
    cfgs = sweep_configs(53, seed=5, edges=(12, 16, 20), **BASE)
    with nicr.Batch(cfgs) as b:
        for i, d in enumerate(b.domains):
            inject(d, i)
        done, rc = b.run(6)
        assert rc == 0 and done == [6] * 53
        for i in (0, 47, 48, 52):
            s = nicr.Solver(cfgs[i])
            inject(s, i)
            s.run(6)
            assert_same_domain(b.domains[i], s, f"domain {i}")
            s.close()


def test_borrowed_handle_survives_destroy_call(require_gpu):
    cfgs = mixed_configs()[:2]
    with nicr.Batch(cfgs) as b:
        h = b.domains[0].h
        nicr.lib().nicr_destroy(h)          # borrowed: ignored
        assert b.domains[0].info().nx == cfgs[0].nx
        b.step(2)
