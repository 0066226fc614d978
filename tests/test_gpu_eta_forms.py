"""Alternative eta-update kernels selectable by NICR_ETA_KERNEL: each must
give the same results as the default selection (drop-in form bit-identical
to the oracle). Each runs in a child process, where the variable is read."""
import os
import subprocess
import sys
import textwrap

import numpy as np
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


FUSED_CHILD = textwrap.dedent("""
    import sys, numpy as np
    root = sys.argv[1]
    sys.path.insert(0, root + "/ni-cr_oxidation_phase-field_simulation_b200"); sys.path.insert(0, root + "/tests")
    import nicr
    from parity import smooth_fields
    cfg = nicr.make_config(3, nx=48, ny=32, nz=64, grains=1, grain_evolution=1, grain_diameter_grid=28.,
                           bounds="legacy", bc="concentration", nucleation="ksp", dt=1e-12, radius_grid=2.5,
                           nucleation_period=5e-12, precision=1)
    sol = nicr.Solver(cfg)
    assert 1 <= sol.n_eta <= 16, sol.n_eta
    o, cr, p, eta = smooth_fields(sol.shape, sol.n_eta, seed=3)
    sol.set_fields(o, cr, p, eta)
    sol.reset_inventory()
    import ctypes
    L = nicr.lib()
    L.nicr_profile(sol.h, 1)          # plain launches, timed per kernel
    sol.run(14)
    tot, cnt = ctypes.c_double(0), ctypes.c_longlong(0)
    L.nicr_profile_read(sol.h, 7, ctypes.byref(tot), ctypes.byref(cnt))   # 7: step_eta
    L.nicr_profile(sol.h, 0)
    sol.run(10)                       # step-pair graphs (the fused launch and its ticket reset captured)
    names = ["o", "cr", "p", "gb", "eta_s2"] + ["eta%d" % (g + 1) for g in range(sol.n_eta)]
    np.savez(sys.argv[2], **{n: sol.get(n) for n in names}, nuclei=sol.budget()["nuclei"], fused=cnt.value)
""")


def test_fused_step_eta_matches_separate_kernels(require_gpu, tmp_path):
    """The opt-in one-launch step (NICR_FUSED=1, k_step_eta) against the two
    launches, reciprocal form: the same bodies, contracted to FMA per kernel
    instance, so fields agree to 1e-13 relative and the nuclei exactly."""
    out = {}
    for fused in ("0", "1"):
        env = dict(os.environ, NICR_FUSED=fused)
        path = str(tmp_path / f"fused{fused}.npz")
        r = subprocess.run([sys.executable, "-c", FUSED_CHILD, str(ROOT), path], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr + r.stdout
        out[fused] = dict(np.load(path))
    assert out["1"]["fused"] > 0 and out["0"]["fused"] == 0
    assert out["0"]["nuclei"] == out["1"]["nuclei"]
    for n in out["0"]:
        if n in ("nuclei", "fused"):
            continue
        a, b = out["1"][n], out["0"][n]
        assert np.max(np.abs(a - b)) <= 1e-13 * max(np.max(np.abs(b)), 1e-300), n
