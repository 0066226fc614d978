"""Definitions shared by the golden-fixture generator and the tests that replay
it: the regression matrix (shape of mpi3d-slab/tests/verify.py:54-114 and
regression_driver.cpp:33-76), its seeded inputs and its command sequence."""
import numpy as np

MODES = {
    "single": dict(grains=0),
    "static": dict(grains=1),
    "evolving": dict(grains=1, grain_evolution=1),
    "frozen": dict(grains=1, grain_evolution=1, eta_L=0.0),
}


def regression_cases(dim: int):
    cases = []
    for mode, mkw in MODES.items():
        for bc in ("closed", "mu", "concentration"):
            for oxygen in (0, 1):
                for ck in ("off", "legacy"):
                    cfg = dict(nx=25, ny=15, grain_diameter_grid=12., bounds="legacy", bc=bc, ck=ck,
                               oxygen_diffusion=oxygen, nucleation="ksp", dt=1e-12, radius_grid=2.5, **mkw)
                    if dim == 3:
                        cfg["nz"] = 13
                    cases.append({"name": f"{mode}-{bc}-O{'on' if oxygen else 'off'}-ck{ck}", "config": cfg})
    return cases


def regression_inputs(cfg):
    """Seeded smooth inputs (PCG64, bit-reproducible): supersaturated O so that
    the Ksp scans insert nuclei, Cr near 0.19, phi = 0, eta near 0.2."""
    shape = (cfg.nx, cfg.ny, cfg.nz) if cfg.dim == 3 else (cfg.nx, cfg.ny)
    rng = np.random.default_rng(1000 + cfg.nx + 7 * cfg.dim)
    n = int(np.prod(shape))
    o = (.001 * (1. + .08 * rng.random(n))).reshape(shape)
    cr = (.19 + .001 * rng.random(n)).reshape(shape)
    p = np.zeros(shape)
    ng = _n_seeds(cfg)
    has_eta = cfg.grain_evolution and cfg.grains
    eta = [(.2 + .02 * rng.random(n)).reshape(shape) for _ in range(ng)] if has_eta else []
    return {"o": o, "cr": cr, "p": p, "eta": eta}


def _n_seeds(cfg):
    import math
    if not cfg.grains:
        return 1
    if cfg.dim == 3:
        v = float(cfg.nx) * cfg.ny * cfg.nz
        return max(1, round(6. * v / (math.pi * cfg.grain_diameter_grid ** 3)))
    a = float(cfg.nx) * cfg.ny
    return max(1, round(4. * a / (math.pi * cfg.grain_diameter_grid ** 2)))


def regression_commands(dim: int, ref_driver: bool):
    """regression_driver.cpp:46-57: stamp at (12,1,1), Ksp before steps 3 and
    14, eta_1(12,7,6) *= 0.95 before step 10 (when eta exists), 24 steps."""
    stamp = ["stamp", 12, 1] + ([1] if dim == 3 else [])
    cmds = [stamp]
    for n in range(24):
        if n in (3, 14):
            cmds.append("nucleate")
        if n == 10:
            cmds.append(["scale_eta_if", 0, 12, 7] + ([6] if dim == 3 else []) + [0.95])
        cmds.append(["step", 1])
    return cmds


# Long runs on the specification's workloads, on the reference's run()
# schedule (Ksp scans every nucleation period, 3S:1368-1385). Inputs are the
# handle's / reference's initial state with seeded noise on Cr (PCG64, the
# x = 0 inlet plane keeps its initial value) and, for the supersaturated
# case, O = 0.001 everywhere (the reference's own way of exercising
# insertion, 3S:1197).
def _grain_diameter_for(n_grains, shape):
    import math
    v = float(np.prod(shape))
    return (6.0 * v / (math.pi * n_grains)) ** (1.0 / 3.0)


_C2 = dict(nx=128, ny=128, nz=128, grains=1, grain_diameter_grid=50., random_seed=1, bc="concentration",
           ck="legacy", bounds="legacy", nucleation="ksp")
LONG_CASES = {
    # C2: 3D 128^3, 32 static Voronoi grains of seed 1, Cr 0.22 +- 0.005, Ksp
    # scans at steps 500, 1000, 1500 and 2000
    "c2_128cube_32grains": dict(config=_C2, steps=2000, cr=(0.22, 0.005, 1), o=None, stamp=None),
    # C2-ksp: the same grid supersaturated, a stamp across both periodic seams,
    # and the same scan cadence, so that ordered insertion fires at every scan
    "c2_128cube_32grains_supersaturated": dict(config=_C2, steps=2000, cr=(0.22, 0.005, 4), o=0.001,
                                               stamp=(64, 1, 1)),
    # the benchmark's per-cell work in the reference's own form: 256^3, 8 seeds
    # of seed 2 with one evolving eta each, Cr 0.25 +- 0.01, one full nucleation
    # period (a Ksp scan at step 500)
    "bench_256cube_8eta": dict(config=dict(nx=256, ny=256, nz=256, grains=1, grain_evolution=1, random_seed=2,
                                           bc="concentration", ck="legacy", bounds="legacy", nucleation="ksp",
                                           grain_diameter_grid=_grain_diameter_for(8, (256, 256, 256))),
                               steps=500, cr=(0.25, 0.01, 2), o=None, stamp=None),
}


def long_inputs(case, o0, cr0, p0):
    """The injected (o, cr, p) of a long case from the initial state."""
    base, amp, seed = case["cr"]
    cr = base + np.random.default_rng(seed).uniform(-amp, amp, size=cr0.shape)
    cr[0] = cr0[0]
    o = o0 if case["o"] is None else np.full(o0.shape, float(case["o"]))
    return o, cr, p0
