"""Alternative eta-update kernels selectable by NICR_ETA_KERNEL: each must
give the same results as the default selection (drop-in form bit-identical
to the oracle). Each runs in a child process, where the variable is read."""
import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
TMA_CHILD = textwrap.dedent("""
    import sys, json, numpy as np
    root = sys.argv[1]
    sys.path.insert(0, root + "/ni-cr_oxidation_phase-field_simulation_b200"); sys.path.insert(0, root + "/tests")
    sys.path.insert(0, root + "/oracle")
    import nicr
    from oracle import Oracle
    from parity import compare_state, smooth_fields
    for shape, prec in (((20, 16, 64), 0), ((11, 24, 32), 0), ((20, 16, 64), 1)):
        cfg = nicr.make_config(3, nx=shape[0], ny=shape[1], nz=shape[2], grains=1, grain_evolution=1,
                               grain_diameter_grid=9., bounds="legacy", bc="mu", nucleation="ksp", dt=1e-12,
                               radius_grid=2.5, nucleation_period=5e-12, precision=prec)
        sol, orc = nicr.Solver(cfg), Oracle(cfg)
        o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=3)
        orc.set_fields(o, cr, p, np.array(eta)); sol.set_fields(o, cr, p, eta)
        assert orc.run(12) == (0, 12)
        sol.run(12)
        if prec == 0:
            compare_state(sol, orc)
        else:
            for g in range(orc.neta):
                a, b = sol.get("eta", g), orc.get("eta%d" % (g + 1))
                assert np.max(np.abs(a - b)) <= 1e-10, g
        print("ok", shape, prec, orc.neta)
""")



def test_tma_eta_kernel_matches_oracle(require_gpu):
    """The opt-in TMA-staged eta kernel (NICR_ETA_KERNEL=tma) on grids it
    accepts (rows a multiple of 8, columns of 32, wrap on both axes), drop-in
    form bit-identical to the oracle, reciprocal form within 1e-10."""
    env = dict(os.environ, NICR_ETA_KERNEL="tma")
    r = subprocess.run([sys.executable, "-c", TMA_CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr + r.stdout
    assert r.stdout.count("ok") == 3
