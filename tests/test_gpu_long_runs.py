"""The specification's workloads at their full length against fixtures made
by the unmodified reference (tests/golden/long_runs.json, written by
tests/golden/make_golden.py with the reference's thread-per-rank build on all
host cores; cases in golden_cases.LONG_CASES):

* C2: 3D 128^3, 32 static Voronoi grains of seed 1, Cr 0.22 +- 0.005, Ksp on,
  2000 steps on the reference's run() schedule (scans at steps 500, 1000,
  1500 and 2000; the reference inserts no nucleus here, and clipping fires on
  ~16K cells per step);
* the same grid supersaturated (O = 0.001) with a stamp across both periodic
  seams, 2000 steps: ordered Ksp insertion at every scan (434 nuclei);
* the benchmark's per-cell work in the reference's own form: 256^3 with 8
  seeds of seed 2 and one evolving eta each, Cr 0.25 +- 0.01, one full
  nucleation period (500 steps, a scan at step 500), run twice: by the
  one-pass step kernel (the default) and by the two-kernel form
  (nicr_config.step_form).

The drop-in form must give every field bit for bit (SHA-256 of o, cr, phi,
mu_O, mu_Cr, M_O, M_Cr, gb, eta_s2 and each eta), the same nuclei and
clipped-cell counts, and budgets within 1e-13 relative (the reference sums
them in long double per rank, here in double-double per CTA)."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import nicr
from golden_cases import LONG_CASES, long_inputs
from parity import ld

pytestmark = pytest.mark.gpu
GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "long_runs.json").read_text())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


RUNS = [(name, 0) for name in LONG_CASES] + [("bench_256cube_8eta", 2)]


@pytest.mark.parametrize("name,step_form", RUNS)
def test_long_run_matches_reference_fixture(require_gpu, name, step_form):
    case, want = LONG_CASES[name], GOLD[name]
    cfg = nicr.make_config(3, **case["config"])
    cfg.step_form = step_form   # 0: the default (one pass where the grid allows it), 2: two kernels
    sol = nicr.Solver(cfg)
    o, cr, p = long_inputs(case, sol.get("o"), sol.get("cr"), sol.get("p"))
    sol.set_fields(o, cr, p)
    sol.reset_inventory()
    if case["stamp"]:
        sol.stamp(*case["stamp"])
    rc, done = sol.run(case["steps"], check=False)
    assert rc == 0 and done == case["steps"], sol.last_error
    got = {}
    for f in want["fields"]:
        if f.startswith("eta") and f != "eta_s2":
            got[f] = sha(sol.get("eta", int(f[3:]) - 1))
        else:
            got[f] = sha(sol.get(f))
    bad = [f for f in want["fields"] if got[f] != want["fields"][f]]
    assert not bad, f"fields differing from the reference after {case['steps']} steps: {bad}"
    b = sol.budget()
    assert b["nuclei"] == want["nuclei"] and b["clipped"] == want["clipped"], (b["nuclei"], b["clipped"])
    for n, pair in want["budget"].items():
        a, w = ld(b[n]), pair[0] + pair[1]
        assert abs(a - w) <= 1e-13 * (1.0 + abs(w)), (n, a, w)
    sol.close()
