"""Parity of the CUDA path with the oracle (the C restatement of the reference,
itself pinned to the reference by tests/test_oracle.py). FP64 fields must be
bit-identical; budgets (long double in the reference, double-double here) agree
to 1e-13 relative."""
import numpy as np
import pytest

from oracle import Oracle, make_config
import nicr
from parity import compare_state, smooth_fields, assert_bitexact

pytestmark = pytest.mark.gpu

MODES = {
    "single": dict(grains=0),
    "static": dict(grains=1),
    "evolving": dict(grains=1, grain_evolution=1),
    "frozen": dict(grains=1, grain_evolution=1, eta_L=0.0),
}
SHAPES = {2: [(25, 15), (140, 37)], 3: [(25, 15, 13), (70, 21, 40)]}


def cfg_for(dim, shape, **kw):
    base = dict(nx=shape[0], ny=shape[1], grain_diameter_grid=12., bounds="legacy", nucleation="ksp",
                dt=1e-12, radius_grid=2.5)
    if dim == 3:
        base["nz"] = shape[2]
    base.update(kw)
    return make_config(dim, **base)


def run_pair(cfg, steps=24, nucleate_at=(3, 14), stamp=True):
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    compare_state(sol, orc)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=cfg.nx)
    orc.set_fields(o, cr, p, np.array(eta) if eta else None)
    sol.set_fields(o, cr, p, eta if eta else None)
    if stamp:
        args = (12, 1, 1) if cfg.dim == 3 else (12, 1)
        assert sol.stamp(*args, *(() if cfg.dim == 3 else (0,))) == orc.stamp(*args, *(() if cfg.dim == 3 else (0,)))
    for n in range(steps):
        if n in nucleate_at:
            orc.nucleate()
            sol.nucleate()
        assert orc.step() == 0, orc.error()
        sol.step(1)
    compare_state(sol, orc)
    return sol, orc


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("bc", ["closed", "mu", "concentration"])
@pytest.mark.parametrize("ck", ["legacy", "off"])
def test_regression_matrix(require_gpu, dim, mode, bc, ck):
    """The reference's 48-case regression matrix shape (verify.py:54-114):
    grain mode x bc x Ck (x O on/off below), stamp across seams, Ksp at 3 and 14."""
    cfg = cfg_for(dim, SHAPES[dim][0], bc=bc, ck=ck, **MODES[mode])
    run_pair(cfg)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("mode", ["single", "static", "evolving"])
def test_oxygen_off(require_gpu, dim, mode):
    cfg = cfg_for(dim, SHAPES[dim][0], bc="concentration", ck="legacy", oxygen_diffusion=0, **MODES[mode])
    run_pair(cfg, steps=10)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("mode", ["static", "evolving"])
def test_partial_tiles_and_chunks(require_gpu, dim, mode):
    """Grids that are not multiples of the CTA tile and stream in several X chunks."""
    cfg = cfg_for(dim, SHAPES[dim][1], bc="mu", ck="legacy", **MODES[mode])
    run_pair(cfg, steps=12, nucleate_at=(2,))


@pytest.mark.parametrize("dim", [2, 3])
def test_center_seed_and_left_edge_sites(require_gpu, dim):
    shape = (31, 25) if dim == 2 else (23, 17, 19)
    cfg = cfg_for(dim, shape, nucleation="center", radius_grid=3.5, left_edge_sites=2, grain_evolution=1,
                  grain_diameter_grid=10., bc="closed", ck="off")
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    assert sol.info().center_seed_cells == orc.center_seed_cells()
    xs, vs = sol.seeds()
    xo, vo = orc.seeds()
    assert_bitexact("seeds", xs, xo)
    assert np.array_equal(vs, vo)
    compare_state(sol, orc)
    for _ in range(20):
        orc.step()
    sol.step(20)
    compare_state(sol, orc)


def test_bounds_stop_rejection_message_and_rollback(require_gpu):
    cfg = cfg_for(3, (25, 15, 13), bounds="stop", bc="concentration", ck="legacy", grains=1)
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p, _ = smooth_fields(orc.shape, 0)
    cr[20, 5, 4] = -0.1
    orc.set_fields(o, cr, p)
    sol.set_fields(o, cr, p)
    before = sol.get("o").copy()
    rc = orc.step()
    assert rc == nicr._abi.ERR_TRIAL_BOUNDS
    rc2, done = sol.step(3, check=False)
    assert rc2 == rc and done == 0
    assert sol.last_error == orc.error()
    assert_bitexact("o after rejection", sol.get("o"), before)
    compare_state(sol, orc)


def test_eta_rejection(require_gpu):
    cfg = cfg_for(2, (25, 15), bounds="legacy", bc="closed", ck="off", grains=1, grain_evolution=1,
                  nucleation="off")
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta)
    eta[0][24, 5] = 2.0
    orc.set_fields(o, cr, p, np.array(eta))
    sol.set_fields(o, cr, p, eta)
    rc = orc.step()
    assert rc == nicr._abi.ERR_ETA_RANGE
    rc2, done = sol.step(2, check=False)
    assert rc2 == rc and done == 0
    assert sol.last_error == orc.error()
    compare_state(sol, orc)


@pytest.mark.parametrize("dim", [2, 3])
def test_run_schedule_with_ksp(require_gpu, dim):
    """run()'s physical-time nucleation schedule (3S:1368-1385) with supersaturated O."""
    shape = (31, 25) if dim == 2 else (31, 21, 19)
    cfg = cfg_for(dim, shape, nucleation_period=5e-12, bc="mu", ck="legacy", grains=1)
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    o, cr, p, _ = smooth_fields(orc.shape, 0)
    orc.set_fields(o, cr, p)
    sol.set_fields(o, cr, p)
    rc, done = orc.run(30)
    assert rc == 0 and done == 30
    rc2, done2 = sol.run(30)
    assert done2 == 30
    compare_state(sol, orc)
    assert sol.budget()["nuclei"] > 0


@pytest.mark.parametrize("b", [1e-16, 1.0000000000000002e-16, 1e-8, 2e-10, 1e-12, 3.3e-9, 0.7, 3.0,
                               1.9999999999999998, 1.4142135623730951, 2.0 ** -60, 2.0 ** 61, -3.0])
def test_verified_division_matches_ieee(require_gpu, b):
    """xdiv (double-word reciprocal, one Markstein correction step, IEEE
    division outside the guarded range) returns exactly a/b on the device for
    2^27 seeded numerators per divisor, a fifth of them with quotients next to
    a rounding midpoint; 2^61 and -3 lie outside the guarded divisor range."""
    import ctypes
    L = nicr.lib()
    L.nicr_check_division.argtypes = [ctypes.c_double, ctypes.c_longlong, ctypes.c_ulonglong,
                                      ctypes.POINTER(ctypes.c_longlong)]
    L.nicr_check_division.restype = ctypes.c_longlong
    tested = ctypes.c_longlong(0)
    bad = L.nicr_check_division(b, 1 << 27, 12345, ctypes.byref(tested))
    assert bad == 0 and tested.value > (1 << 26)


@pytest.mark.parametrize("dim,mode", [(3, "evolving"), (3, "static"), (2, "evolving")])
def test_fast_form_deviation_from_drop_in(require_gpu, dim, mode):
    """NICR_FP64_FAST (reciprocal divisions) stays within 1e-10 relative L-inf of
    the bit-identical form after 200 steps of the regression-like case."""
    shape = SHAPES[dim][1]
    kw = dict(bc="concentration", ck="legacy", nucleation="off", **MODES[mode])
    exact = nicr.Solver(cfg_for(dim, shape, **kw))
    fast = nicr.Solver(cfg_for(dim, shape, precision=1, **kw))
    o, cr, p, eta = smooth_fields(shape, exact.n_eta, seed=11)
    for s in (exact, fast):
        s.set_fields(o, cr, p, eta if eta else None)
        s.step(200)
    names = ["o", "cr", "p"] + [f"eta{g + 1}" for g in range(exact.n_eta)]
    for n in names:
        a, b = fast.get(n), exact.get(n)
        err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert err <= 1e-10, (n, err)


@pytest.mark.parametrize("dim,mode,step_form,shape", [(2, "static", 0, None), (3, "static", 0, None),
                                                      (3, "evolving", 2, None), (3, "evolving", 1, (45, 32, 32))])
def test_tiny_and_subnormal_numerators(require_gpu, dim, mode, step_form, shape):
    """O falling through every magnitude from 1e-3 to below the subnormals along
    X, and phi from 1e-50 to 1e-110 along the rows (h(phi) down to ~1e-330):
    flux, Laplacian and Ck numerators leave the exact-division range (biased
    exponent 123..1923) in most CTAs, whose chunks the drop-in form marches a
    second time with IEEE division for those; fields stay bit-identical. The
    last case runs the one-pass step kernel (rows a multiple of 16, columns of
    32), the others the two-kernel form."""
    import ctypes
    shape = shape or SHAPES[dim][1]
    extra = {"grain_diameter_grid": 26.} if step_form == 1 else {}   # <= 8 eta fields for the one pass
    cfg = cfg_for(dim, shape, bc="concentration", ck="legacy", nucleation="off", step_form=step_form,
                  **MODES[mode], **extra)
    sol, orc = nicr.Solver(cfg), Oracle(cfg)
    if step_form == 1:
        assert 1 <= orc.neta <= 8, orc.neta
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=7)
    idx = np.indices(orc.shape).astype(float)
    o = o * 10.0 ** (-330.0 * idx[0] / orc.shape[0])
    p = 10.0 ** (-50.0 - 60.0 * idx[1] / orc.shape[1])
    orc.set_fields(o, cr, p, np.array(eta) if eta else None)
    sol.set_fields(o, cr, p, eta if eta else None)
    nicr.lib().nicr_profile(sol.h, 1)
    for _ in range(6):
        assert orc.step() == 0, orc.error()
        sol.step(1)
    tot, cnt = ctypes.c_double(0), ctypes.c_longlong(0)
    nicr.lib().nicr_profile_read(sol.h, 8, ctypes.byref(tot), ctypes.byref(cnt))   # the one-pass kernel
    assert cnt.value == (6 if step_form == 1 else 0)
    compare_state(sol, orc)
