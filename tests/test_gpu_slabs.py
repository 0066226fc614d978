"""Slab form (nicr_slabs_*): one 3D domain split along X into slabs, each
storing halo planes of its neighbours, all on one GPU here (the slab code
path is the same for slabs on different GPUs; only the copies' destination
memory differs). The group must evolve exactly as one handle on the same
configuration: same fields bit for bit after steps, Ksp scans (nuclei near
and across slab seams) and rejected trials, the same accepted-step counts,
nuclei, clipped cells and error messages; budget sums to 1e-13 relative
(per-slab double-double sums added). The exception is the register-marching
eta kernel of the reciprocal form (N <= 16 fields), whose slab instance is
compiled with FMA contraction apart from the whole-domain one: there the
fields agree to 1e-13 relative. One group is also checked against the
oracle directly."""
import numpy as np
import pytest

import nicr
from oracle import Oracle
from parity import assert_bitexact, assert_budget, compare_state, smooth_fields

pytestmark = pytest.mark.gpu

KSP = dict(bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12)


def grains_cfg(nx=40, ny=24, nz=32, **kw):
    base = dict(nx=nx, ny=ny, nz=nz, grains=1, grain_evolution=1, grain_diameter_grid=11., random_seed=3,
                bc="concentration", ck="legacy", **KSP)
    base.update(kw)
    return nicr.make_config(3, **base)


def inject(sol, seed, n_eta):
    o, cr, p, eta = smooth_fields(sol.shape, n_eta, seed=seed)
    sol.set("o", o)
    sol.set("cr", cr)
    sol.set("p", p)
    for g, e in enumerate(eta):
        sol.set("eta", e, g)
    sol.reset_inventory()


def assert_same(a, b, n_eta, label, fields=("o", "cr", "p", "gb")):
    for f in fields:
        assert_bitexact(f"{label} {f}", a.get(f), b.get(f))
    for g in range(n_eta):
        assert_bitexact(f"{label} eta{g + 1}", a.get("eta", g), b.get("eta", g))
    if n_eta:
        assert_bitexact(f"{label} eta_s2", a.get("eta_s2"), b.get("eta_s2"))
    assert_budget(a.budget(), b.budget())


def test_slab_partition(require_gpu):
    cfg = grains_cfg(nx=41)
    with nicr.Slabs(cfg, 3) as s:
        parts = [s.slab(i) for i in range(len(s))]
    assert [(q["x0"], q["x1"]) for q in parts] == [(0, 14), (14, 28), (28, 41)]
    assert all(q["halo"] == 9 and q["device"] == 0 for q in parts)   # ceil(2.5 + 6)
    with pytest.raises(nicr.NicrError):
        nicr.Slabs(grains_cfg(nx=40), 5)                              # 8 planes < halo 9
    with pytest.raises(nicr.NicrError):
        nicr.Slabs(nicr.make_config(2, nx=64, ny=64), 2)              # 3D only


@pytest.mark.parametrize("cfg_kw", [dict(grain_evolution=0), dict(grains=0, nucleation="center", radius_grid=4.0),
                                    dict()], ids=["static-grains", "centre-seed", "evolving-eta"])
def test_initial_state_matches(require_gpu, cfg_kw):
    """Every slab initialises its stored planes (halos included) in domain
    coordinates: Voronoi labels and mask, eta weights, centre seed."""
    cfg = grains_cfg(**cfg_kw)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 3) as s:
        fields = ("o", "cr", "p", "gb") + (("grain",) if cfg.grain_evolution == 0 else ())
        assert_same(s, solo, solo.n_eta, "initial", fields)
        d, e = s.diagnostics(), solo.diagnostics()
        for k in e:
            if isinstance(e[k], tuple):
                assert abs(sum(d[k]) - sum(e[k])) <= 1e-13 * (1 + abs(sum(e[k]))), k
            else:
                assert d[k] == e[k], k
    solo.close()


@pytest.mark.parametrize("nslabs", [2, 3])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp64-fast"])
@pytest.mark.parametrize("mode", ["run", "step"])
def test_slabs_match_single_handle(require_gpu, nslabs, precision, mode):
    cfg = grains_cfg(precision=precision)
    solo = nicr.Solver(cfg)
    n_eta = solo.n_eta
    with nicr.Slabs(cfg, nslabs) as s:
        inject(solo, 5, n_eta)
        inject(s, 5, n_eta)
        assert_same(s, solo, n_eta, "after set")
        for chunk in (7, 1, 12):
            rc, done = getattr(s, mode)(chunk)
            getattr(solo, mode)(chunk)
            assert rc == 0 and done == chunk
        assert s.steps_done == solo.info().steps_done == 20
        assert_same(s, solo, n_eta, f"{nslabs} slabs")
        if mode == "run":
            assert s.budget()["nuclei"] > 3    # scans fired and stamped across the domain
        d, e = s.diagnostics(), solo.diagnostics()
        for k in ("min_O", "max_O", "min_Cr", "max_Cr", "min_Ni", "min_phi", "max_phi"):
            assert d[k] == e[k], k
    solo.close()


@pytest.mark.parametrize("gap", [0.5, 6.0])
def test_dense_nuclei_across_seams(require_gpu, gap):
    """Small exclusion gaps pack nuclei at every seam; four slabs of 8-14
    planes make most exclusion zones reach a neighbour or the one beyond."""
    cfg = grains_cfg(nx=48 if gap < 1 else 56, exclusion_gap_grid=gap, grain_evolution=0)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 4) as s:
        inject(solo, 9, 0)
        inject(s, 9, 0)
        for _ in range(3):
            s.run(10)
            solo.run(10)
        assert_same(s, solo, 0, f"gap {gap}")
        assert s.budget()["nuclei"] == solo.budget()["nuclei"] > 4
        assert s.nucleate() == solo.nucleate()
        assert_same(s, solo, 0, f"gap {gap} after nucleate")
    solo.close()


@pytest.mark.parametrize("plane", [13, 14, 20])
def test_rejected_trial_rolls_back_every_slab(require_gpu, plane):
    """A failing trial in one slab (at a seam plane or inside) rejects the
    step in all slabs with the whole-domain message and first failing cell."""
    cfg = grains_cfg(bounds="stop", grain_evolution=0)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 3) as s:
        inject(solo, 4, 0)
        inject(s, 4, 0)
        s.run(6)
        solo.run(6)
        cr = solo.get("cr")
        cr[plane, 5, 4] = -0.1
        cr[plane + 10, 2, 2] = -0.2    # a later cell: the first one is reported
        solo.set("cr", cr)
        s.set("cr", cr)
        before = s.get("o")
        rc, done = s.run(8, check=False)
        rc_solo, done_solo = solo.run(8, check=False)
        assert rc == rc_solo == nicr._abi.ERR_TRIAL_BOUNDS
        assert done == done_solo == 0
        assert s.last_error == solo.last_error and s.last_error.startswith("Out-of-bounds trial at (")
        assert_bitexact("o after rejection", s.get("o"), before)
        assert_same(s, solo, 0, "rejected")
        # the group carries on from the restored state like the handle
        cr[plane, 5, 4] = 0.19
        cr[plane + 10, 2, 2] = 0.19
        s.set("cr", cr)
        solo.set("cr", cr)
        s.run(9)
        solo.run(9)
        assert_same(s, solo, 0, "after recovery")
    solo.close()


def test_slabs_match_oracle(require_gpu):
    cfg = grains_cfg(nx=36, ny=16, nz=16, grain_diameter_grid=9.)
    orc = Oracle(cfg)
    with nicr.Slabs(cfg, 2) as s:
        o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=12)
        s.set("o", o)
        s.set("cr", cr)
        s.set("p", p)
        for g, e in enumerate(eta):
            s.set("eta", e, g)
        orc.set_fields(o, cr, p, np.stack(eta) if eta else None)
        s.reset_inventory()
        orc.reset_inventory()
        rc, done = s.run(15)
        rc2, done2 = orc.run(15)
        assert rc == rc2 == 0 and done == done2 == 15
        compare_state(s, orc)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp64-fast"])
def test_128cube_8eta_two_slabs(require_gpu, precision):
    """The bench's shape at 128^3: 8 evolving eta, Ksp at the default radius
    and gap (halo 12), 2 slabs. The drop-in form is bit-identical. In the
    reciprocal form the slab instance of the eta march is compiled with FMA
    contraction separately from the whole-domain instance, so a few cells may
    round differently: fields within 1e-13 relative of the single handle."""
    shape = (128, 128, 128)
    d = (6.0 * np.prod(shape) / (np.pi * 8)) ** (1.0 / 3.0)
    cfg = nicr.make_config(3, nx=128, ny=128, nz=128, grains=1, grain_evolution=1, random_seed=2,
                           grain_diameter_grid=d, bc="concentration", ck="legacy", bounds="legacy",
                           nucleation="ksp", precision=precision)
    solo = nicr.Solver(cfg)
    assert solo.n_eta == 8
    with nicr.Slabs(cfg, 2) as s:
        assert s.slab(0)["halo"] == 12
        cr = 0.25 + np.random.default_rng(2).uniform(-0.01, 0.01, size=shape)
        cr[0] = solo.get("cr")[0]
        for sol in (s, solo):
            sol.set("cr", cr)
            sol.reset_inventory()
        s.run(40)
        solo.run(40)
        if precision == 0:
            assert_same(s, solo, 8, "128^3 8 eta")
        else:
            names = ["o", "cr", "p", "gb", "eta_s2"] + [f"eta{g + 1}" for g in range(8)]
            for f in names:
                a, b = s.get(f), solo.get(f)
                dev = float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)
                assert dev <= 1e-13, (f, dev)
            assert_budget(s.budget(), solo.budget(), rtol=1e-12)
    solo.close()


def test_grain_stats_and_vti_match(require_gpu, tmp_path):
    """nicr_slabs_get_grain_stats and nicr_slabs_write_vti give a single
    handle's values and file (grain statistics sum per slab: 1e-13)."""
    cfg = grains_cfg(eta_colours=5)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 3) as s:
        assert s.n_eta == solo.n_eta == 5
        inject(solo, 6, 5)
        inject(s, 6, 5)
        s.run(11)
        solo.run(11)
        a, b = s.grain_stats(), solo.grain_stats()
        for k in ("min_eta", "max_eta", "min_s2", "max_s2", "gb_max", "alive", "unassigned"):
            assert a[k] == b[k], k
        for k in ("sum_s2", "mask", "energy"):
            assert abs(sum(a[k]) - sum(b[k])) <= 1e-13 * (1 + abs(sum(b[k]))), k
        assert (a["cells"] == b["cells"]).all()
        assert np.allclose(a["amount"].sum(axis=1), b["amount"].sum(axis=1), rtol=1e-13, atol=0)
        s.write_vti(tmp_path / "slabs.vti")
        solo.write_vti(tmp_path / "solo.vti")
        assert (tmp_path / "slabs.vti").read_bytes() == (tmp_path / "solo.vti").read_bytes()
    solo.close()


@pytest.mark.parametrize("kw", [dict(bc="mu", ck="off"), dict(bc="closed"), dict(oxygen_diffusion=0),
                                dict(grains=0, nucleation="center", radius_grid=6.0),
                                dict(grain_evolution=0, bounds="stop")],
                         ids=["bc-mu-ck-off", "bc-closed", "o-off", "single-crystal-centre", "static-stop"])
def test_slab_modes(require_gpu, kw):
    """The boundary and physics modes around the seams: the mu boundary's
    surface flux (slab 0 only), closed boundaries, O transport off, a single
    crystal whose centre seed spans slabs, static grains with bounds=stop."""
    cfg = grains_cfg(**kw)
    solo = nicr.Solver(cfg)
    with nicr.Slabs(cfg, 3) as s:
        inject(solo, 8, solo.n_eta)
        inject(s, 8, solo.n_eta)
        for chunk in (5, 6):
            rc, done = s.run(chunk, check=False)
            rc1, done1 = solo.run(chunk, check=False)
            assert (rc, done) == (rc1, done1)
        assert_same(s, solo, solo.n_eta, str(kw))
    solo.close()
