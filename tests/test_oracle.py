"""The oracle is pinned to the reference: the C restatement must reproduce the
unmodified reference solver (oracle/_ref, built from the reference sources by
oracle/Makefile) bit for bit. Skipped where the reference build is absent."""
import numpy as np
import pytest

from oracle import Oracle, make_config, reference_available, run_reference
from parity import assert_bitexact, assert_budget, smooth_fields

needs_ref = pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built (reference sources absent)")


def oracle_budget_from_dump(d):
    names = ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")
    out = {n: tuple(d["budget"][q]) for q, n in enumerate(names)}
    out["initialO"], out["initialCr"] = tuple(d["initial"][0]), tuple(d["initial"][1])
    out["nuclei"], out["clipped"] = int(d["counts"][0]), int(d["counts"][1])
    return out


@needs_ref
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("mode", [dict(grains=0), dict(grains=1), dict(grains=1, grain_evolution=1),
                                  dict(grains=1, grain_evolution=1, eta_L=0.0)])
@pytest.mark.parametrize("bc", ["closed", "mu", "concentration"])
@pytest.mark.parametrize("ck", ["legacy", "off"])
def test_oracle_matches_reference(dim, mode, bc, ck):
    kw = dict(nx=25, ny=15, grain_diameter_grid=12., bounds="legacy", bc=bc, ck=ck, nucleation="ksp", dt=1e-12,
              radius_grid=2.5, **mode)
    if dim == 3:
        kw["nz"] = 13
    cfg = make_config(dim, **kw)
    orc = Oracle(cfg)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=3)
    inj = {"o": o, "cr": cr, "p": p, "eta": eta}
    stamp = ["stamp", 12, 1] + ([1] if dim == 3 else [])
    cmds = ["dump", stamp]
    for n in range(24):
        if n in (3, 14):
            cmds.append("nucleate")
        cmds.append(["step", 1])
    cmds.append("dump")
    ref = run_reference(cfg, cmds, inject=inj)
    orc.set_fields(o, cr, p, np.array(eta) if eta else None)
    d0 = ref["dumps"][0]
    for f in ("o", "cr", "p", "gb"):
        assert_bitexact(f"{f}@inject", orc.get(f).ravel(), d0[f])
    orc.stamp(12, 1, 1 if dim == 3 else 0)
    for n in range(24):
        if n in (3, 14):
            orc.nucleate()
        assert orc.step() == 0
    orc.refresh()
    d = ref["dumps"][1]
    for f in ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb"):
        assert_bitexact(f, orc.get(f).ravel(), d[f])
    for g in range(orc.neta):
        assert_bitexact(f"eta{g + 1}", orc.get(f"eta{g + 1}").ravel(), d[f"eta{g + 1}"])
    assert_budget(orc.budget(), oracle_budget_from_dump(d), rtol=0.0)
