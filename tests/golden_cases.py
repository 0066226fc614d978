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
