"""The one-pass step (k_step_fused: the step kernel and the eta update in one
X march, eta planes staged by TMA, S and the GB mask rebuilt on chip) on the
3D evolving-grain grids it serves (1..8 eta fields, rows a multiple of 16,
columns a multiple of 32).

* Drop-in form against the oracle, bit for bit: single tiles (the periodic
  wrap of every halo box onto the tile itself), several tiles, 1 to 8 eta
  fields, the three boundary conditions, O off, Ck on and off, a stamp across
  both periodic seams and Ksp scans, graph-replayed runs.
The handles ask for the one-pass form (nicr_config.step_form = 1), which
the default (AUTO) also takes wherever the grid allows it.

* Against the two-kernel form (NICR_STEP_FORM=split) in child processes,
  with forced X chunks of 1, 3 and 7 planes (chunk prologues, chunk ends at
  the ghost plane): drop-in fields bit-identical, reciprocal form within
  1e-13 relative.
* Rejections: a bounds=stop trial and an eta trial outside [0, 1] give the
  oracle's message, and the state stays the last accepted one.
"""
import ctypes
import json
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import nicr
from conftest import ROOT
from oracle import Oracle, make_config
from parity import assert_bitexact, compare_state, smooth_fields

pytestmark = pytest.mark.gpu

STEP_FUSED = 8   # nicr_profile_read kernel index of the one-pass step


def cfg_for(shape, **kw):
    base = dict(nx=shape[0], ny=shape[1], nz=shape[2], grains=1, grain_evolution=1, bounds="legacy",
                nucleation="ksp", dt=1e-12, radius_grid=2.5, step_form=1)
    base.update(kw)
    return make_config(3, **base)


def fused_launches(sol):
    tot, cnt = ctypes.c_double(0), ctypes.c_longlong(0)
    nicr.lib().nicr_profile_read(sol.h, STEP_FUSED, ctypes.byref(tot), ctypes.byref(cnt))
    return cnt.value


# shape, grain diameter (-> number of eta fields), boundary condition, Ck, extra
CASES = {
    "single-tile-6eta-mu": ((24, 16, 32), 16., "mu", "legacy", {}),
    "2x2-tiles-8eta-concentration": ((37, 32, 64), 26., "concentration", "legacy", {}),
    "1x3-tiles-7eta-closed-ckoff": ((20, 16, 96), 24., "closed", "off", {}),
    "single-eta-mu": ((19, 16, 32), 40., "mu", "legacy", {}),
    "oxygen-off-5eta": ((23, 32, 32), 20., "concentration", "legacy", {"oxygen_diffusion": 0}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_onepass_drop_in_matches_oracle(require_gpu, name):
    shape, d, bc, ck, extra = CASES[name]
    cfg = cfg_for(shape, grain_diameter_grid=d, bc=bc, ck=ck, **extra)
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    assert 1 <= orc.neta <= 8, orc.neta
    compare_state(sol, orc)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=cfg.nx)
    orc.set_fields(o, cr, p, np.array(eta))
    sol.set_fields(o, cr, p, eta)
    assert sol.stamp(12, 1, 1) == orc.stamp(12, 1, 1)   # across both periodic seams
    nicr.lib().nicr_profile(sol.h, 1)                     # plain launches, counted per kernel
    for n in range(16):
        if n in (3, 11):
            orc.nucleate()
            sol.nucleate()
        assert orc.step() == 0, orc.error()
        sol.step(1)
    assert fused_launches(sol) == 16
    compare_state(sol, orc)
    nicr.lib().nicr_profile(sol.h, 0)
    for _ in range(20):                                   # graph-replayed runs of 16 and 4 steps
        assert orc.step() == 0, orc.error()
    sol.step(20)
    compare_state(sol, orc)
    sol.close()


CHILD = textwrap.dedent("""
    import sys, json, ctypes, numpy as np
    root, out, case = sys.argv[1], sys.argv[2], json.loads(sys.argv[3])
    sys.path.insert(0, root + "/ni-cr_oxidation_phase-field_simulation_b200"); sys.path.insert(0, root + "/tests")
    import nicr
    from parity import smooth_fields
    cfg = nicr.make_config(3, **case["cfg"])
    sol = nicr.Solver(cfg)
    o, cr, p, eta = smooth_fields(sol.shape, sol.n_eta, seed=5)
    sol.set_fields(o, cr, p, eta)
    sol.reset_inventory()
    L = nicr.lib()
    L.nicr_profile(sol.h, 1)
    rcs = [list(sol.run(case["steps"], check=False))]
    tot, cnt = ctypes.c_double(0), ctypes.c_longlong(0)
    L.nicr_profile_read(sol.h, 8, ctypes.byref(tot), ctypes.byref(cnt))
    L.nicr_profile(sol.h, 0)
    rcs.append(list(sol.run(case["steps"], check=False)))   # graphs
    names = ["o", "cr", "p", "gb", "eta_s2"] + ["eta%d" % (g + 1) for g in range(sol.n_eta)]
    np.savez(out, **{n: sol.get(n) for n in names})
    b = sol.budget()
    json.dump({"rcs": rcs, "fused": cnt.value, "nuclei": b["nuclei"], "clipped": b["clipped"],
               "budget": {k: [float(x) for x in b[k]] for k in ("ckO", "ckCr", "clipO", "clipCr", "bcO", "nucO")}},
              open(out + ".json", "w"))
""")


def run_child(tmp_path, tag, case, **env):
    out = str(tmp_path / tag)
    e = dict(os.environ, **env)
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), out, json.dumps(case)], env=e, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr + r.stdout
    return dict(np.load(out + ".npz")), json.load(open(out + ".json"))


SPLIT_CASES = {
    "chunk1": ({"NICR_XCHUNK": "1"}, dict(nx=21, ny=32, nz=32, grain_diameter_grid=20.)),
    "chunk3": ({"NICR_XCHUNK": "3"}, dict(nx=29, ny=16, nz=64, grain_diameter_grid=19.)),
    "chunk7": ({"NICR_XCHUNK": "7"}, dict(nx=45, ny=32, nz=32, grain_diameter_grid=22.)),
}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(SPLIT_CASES))
def test_onepass_matches_two_kernel_form(require_gpu, tmp_path, name, precision):
    env, shape = SPLIT_CASES[name]
    cfg = dict(shape, grains=1, grain_evolution=1, bounds="legacy", bc="mu", ck="legacy", nucleation="ksp",
               dt=1e-12, radius_grid=2.5, nucleation_period=6e-12, precision=precision, step_form=1)
    case = {"cfg": cfg, "steps": 24}
    a, ja = run_child(tmp_path, "onepass", case, **env)
    b, jb = run_child(tmp_path, "split", case, NICR_STEP_FORM="split", **env)   # overrides step_form
    assert ja["fused"] == 24 and jb["fused"] == 0
    assert ja["rcs"] == jb["rcs"] and ja["nuclei"] == jb["nuclei"] and ja["clipped"] == jb["clipped"]
    assert jb["nuclei"] > 0
    for n in b:
        if precision == 0:
            assert_bitexact(n, a[n], b[n])
        else:
            err = np.max(np.abs(a[n] - b[n])) / max(np.max(np.abs(b[n])), 1e-300)
            assert err <= 1e-13, (n, err)
    for k, v in jb["budget"].items():
        w, g = v[0] + v[1], ja["budget"][k][0] + ja["budget"][k][1]
        assert abs(g - w) <= 1e-13 * (1 + abs(w)), (k, g, w)


def test_onepass_bounds_stop_rejection(require_gpu):
    cfg = cfg_for((25, 16, 32), grain_diameter_grid=18., bounds="stop", bc="concentration", ck="legacy",
                  nucleation="off")
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta)
    cr[20, 5, 4] = -0.1
    cr[21, 15, 31] = -0.2
    orc.set_fields(o, cr, p, np.array(eta))
    sol.set_fields(o, cr, p, eta)
    before = sol.get("o").copy()
    rc = orc.step()
    assert rc == nicr._abi.ERR_TRIAL_BOUNDS
    nicr.lib().nicr_profile(sol.h, 1)
    rc2, done = sol.step(3, check=False)
    assert rc2 == rc and done == 0 and fused_launches(sol) >= 1
    assert sol.last_error == orc.error()
    assert_bitexact("o after rejection", sol.get("o"), before)
    compare_state(sol, orc)


def test_onepass_eta_rejection(require_gpu):
    cfg = cfg_for((22, 16, 32), grain_diameter_grid=18., bounds="legacy", bc="closed", ck="off",
                  nucleation="off")
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta)
    eta[1][21, 15, 0] = 2.0     # last plane, a corner of the periodic wrap
    eta[0][21, 15, 31] = 1.5
    orc.set_fields(o, cr, p, np.array(eta))
    sol.set_fields(o, cr, p, eta)
    rc = orc.step()
    assert rc == nicr._abi.ERR_ETA_RANGE
    nicr.lib().nicr_profile(sol.h, 1)
    rc2, done = sol.step(2, check=False)
    assert rc2 == rc and done == 0 and fused_launches(sol) >= 1
    assert sol.last_error == orc.error()
    compare_state(sol, orc)
