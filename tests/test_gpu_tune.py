"""Autotuning (nicr_tune, nicr_batch_tune): it measures candidate X chunks and
occupancy variants on the live state without changing it, and stepping after
it gives the same fields, bit for bit, as an untuned handle (budgets to
1e-13: their per-CTA partial sums may group differently)."""
import numpy as np
import pytest

import nicr
from nicr.sweep import sweep_configs
from parity import assert_bitexact, assert_budget, smooth_fields

pytestmark = pytest.mark.gpu

BASE = dict(bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12)


def prepared(cfg, seed=5):
    s = nicr.Solver(cfg)
    o, cr, p, eta = smooth_fields(s.shape, s.n_eta, seed=seed)
    s.set_fields(o, cr, p, eta if eta else None)
    s.reset_inventory()
    return s


def fields(s):
    d = {f: s.get(f) for f in ("o", "cr", "p", "gb")}
    for g in range(s.n_eta):
        d[f"eta{g + 1}"] = s.get("eta", g)
    return d


@pytest.mark.parametrize("dim,shape,kw", [
    (3, (64, 32, 64), dict(grains=1, grain_evolution=1, grain_diameter_grid=12.)),
    (3, (45, 21, 40), dict(grains=1, grain_diameter_grid=12., precision=1)),
    (2, (128, 128), dict(grains=0, nucleation="center", radius_grid=4.0, bc="concentration")),
])
def test_tune_keeps_state_and_results(require_gpu, dim, shape, kw):
    d = dict(BASE, nx=shape[0], ny=shape[1])
    if dim == 3:
        d["nz"] = shape[2]
    d.update(kw)
    cfg = nicr.make_config(dim, **d)
    a, b = prepared(cfg), prepared(cfg)
    a.run(5)
    b.run(5)
    before, bud = fields(a), a.budget()
    chunk, minb = a.tune(2)
    assert 1 <= chunk <= shape[0]
    assert minb in ((2, 3) if dim == 3 else (0,))
    after = fields(a)
    for k in before:
        assert_bitexact(f"{k} after tune", after[k], before[k])
    assert a.budget() == bud and a.info().steps_done == 5
    a.run(11)
    b.run(11)
    fa, fb = fields(a), fields(b)
    for k in fa:
        assert_bitexact(k, fa[k], fb[k])
    assert_budget(a.budget(), b.budget())
    a.close()
    b.close()


def test_batch_tune(require_gpu):
    cfgs = sweep_configs(6, seed=21, edges=(16, 32, 48), **BASE)
    ref = [prepared(c, seed=i) for i, c in enumerate(cfgs)]
    with nicr.Batch(cfgs) as b:
        for i, d in enumerate(b.domains):
            o, cr, p, eta = smooth_fields(d.shape, d.n_eta, seed=i)
            d.set_fields(o, cr, p, eta if eta else None)
            d.reset_inventory()
        chunk = b.tune(2)
        assert chunk >= 1
        b.run(9)
        for s in ref:
            s.run(9)
        for d, s in zip(b.domains, ref):
            fa, fb = fields(d), fields(s)
            for k in fa:
                assert_bitexact(k, fa[k], fb[k])
            assert_budget(d.budget(), s.budget())
    for s in ref:
        s.close()
