"""Step-pair CUDA graphs (used by nicr_step / nicr_run for pairs of steps):
the replayed pairs must give the same state, budgets and launch accounting as
launching every kernel (NICR_GRAPHS=0, run in a child process), across the
run() Ksp schedule (scans stay outside the graphs), parity changes after a
rejected trial, and odd step counts."""
import json
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

CHILD = textwrap.dedent("""
    import sys, json, numpy as np
    sys.path.insert(0, sys.argv[1] + "/ni-cr_oxidation_phase-field_simulation_b200"); sys.path.insert(0, sys.argv[1] + "/tests")
    import nicr
    from parity import smooth_fields
    case = json.loads(sys.argv[2]); out = sys.argv[3]
    cfg = nicr.make_config(case["dim"], **case["kw"])
    s = nicr.Solver(cfg)
    o, cr, p, eta = smooth_fields(s.shape, s.n_eta, seed=7)
    if case.get("bad"):
        cr[tuple(case["bad"])] = -0.1
    s.set_fields(o, cr, p, eta if eta else None)
    s.reset_inventory()
    rcs = []
    for n in case["chunks"]:
        rc, done = (s.run if case["mode"] == "run" else s.step)(n, check=False)
        rcs.append([rc, done])
        if rc:
            cr = s.get("cr"); cr[cr < 0] = 0.1; s.set("cr", cr)   # repair and go on
    arrs = {f: s.get(f) for f in ("o", "cr", "p", "gb")}
    for g in range(s.n_eta):
        arrs["eta%d" % g] = s.get("eta", g)
    b = s.budget()
    np.savez(out, **arrs)
    json.dump({"rcs": rcs, "budget": {k: (list(v) if not isinstance(v, int) else v) for k, v in b.items()},
               "steps": s.info().steps_done, "launches": nicr.lib().nicr_kernel_launches(s.h)}, open(out + ".json", "w"))
""")

CASES = {
    "2d-center-run": dict(dim=2, mode="run", chunks=[1, 7, 30],
                          kw=dict(nx=128, ny=128, grains=0, nucleation="center", radius_grid=4.0, bc="concentration",
                                  ck="legacy", bounds="legacy")),
    "3d-ksp-run": dict(dim=3, mode="run", chunks=[9, 13, 4],
                       kw=dict(nx=31, ny=21, nz=19, grains=1, grain_diameter_grid=12., bc="mu", bounds="legacy",
                               nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12)),
    "3d-evolving-step": dict(dim=3, mode="step", chunks=[2, 5, 10],
                             kw=dict(nx=25, ny=15, nz=13, grains=1, grain_evolution=1, grain_diameter_grid=12.,
                                     bounds="legacy", nucleation="off", dt=1e-12)),
    "3d-rejection": dict(dim=3, mode="step", chunks=[6, 6], bad=[20, 5, 4],
                         kw=dict(nx=25, ny=15, nz=13, grains=1, grain_diameter_grid=12., bounds="stop",
                                 nucleation="off", dt=1e-12)),
}


def run_child(case, out, graphs):
    env = dict(os.environ, NICR_GRAPHS="1" if graphs else "0")
    r = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), json.dumps(case), str(out)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return np.load(str(out) + ".npz"), json.load(open(str(out) + ".json"))


@pytest.mark.parametrize("name", list(CASES))
def test_graph_pairs_match_plain_launches(require_gpu, tmp_path, name):
    case = CASES[name]
    a, ja = run_child(case, tmp_path / "graphs", True)
    b, jb = run_child(case, tmp_path / "plain", False)
    for k in b.files:
        assert np.array_equal(a[k].view(np.int64), b[k].view(np.int64)), (name, k)
    assert ja["rcs"] == jb["rcs"] and ja["budget"] == jb["budget"] and ja["steps"] == jb["steps"]
    assert ja["launches"] == jb["launches"]
    if name == "3d-rejection":
        assert ja["rcs"][0][0] != 0


BATCH_CHILD = textwrap.dedent("""
    import sys, json, numpy as np
    sys.path.insert(0, sys.argv[1] + "/ni-cr_oxidation_phase-field_simulation_b200"); sys.path.insert(0, sys.argv[1] + "/tests")
    import nicr
    from nicr.sweep import sweep_configs
    from parity import smooth_fields
    out = sys.argv[2]
    base = dict(bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5, nucleation_period=5e-12)
    cfgs = sweep_configs(5, seed=11, edges=(20, 33, 40), **base)
    cfgs.append(nicr.make_config(3, nx=24, ny=19, nz=35, grains=1, grain_evolution=1, grain_diameter_grid=10., bc="mu", **base))
    cfgs.append(nicr.make_config(2, nx=61, ny=45, grains=1, grain_diameter_grid=12., **base))
    with nicr.Batch(cfgs) as b:
        for i, d in enumerate(b.domains):
            o, cr, p, eta = smooth_fields(d.shape, d.n_eta, seed=i)
            d.set_fields(o, cr, p, eta if eta else None)
            d.reset_inventory()
        res = []
        for n in (7, 12, 1, 9):
            res.append(b.run(n, check=False))
        arrs = {}
        for i, d in enumerate(b.domains):
            for f in ("o", "cr", "p", "gb"):
                arrs["%d_%s" % (i, f)] = d.get(f)
        np.savez(out, **arrs)
        json.dump({"res": res, "budgets": [d.budget() for d in b.domains], "launches": b.kernel_launches,
                   "nuclei": sum(d.budget()["nuclei"] for d in b.domains)}, open(out + ".json", "w"))
""")


def test_batch_graph_pairs_match_plain_launches(require_gpu, tmp_path):
    outs = []
    for graphs in ("1", "0"):
        out = tmp_path / f"batch{graphs}"
        env = dict(os.environ, NICR_GRAPHS=graphs)
        r = subprocess.run([sys.executable, "-c", BATCH_CHILD, str(ROOT), str(out)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        outs.append((np.load(str(out) + ".npz"), json.load(open(str(out) + ".json"))))
    (a, ja), (b, jb) = outs
    for k in b.files:
        assert np.array_equal(a[k].view(np.int64), b[k].view(np.int64)), k
    assert ja["res"] == jb["res"] and ja["budgets"] == jb["budgets"] and ja["launches"] == jb["launches"]
    assert ja["nuclei"] > 0

