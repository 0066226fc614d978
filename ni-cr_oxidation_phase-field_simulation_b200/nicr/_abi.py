"""ctypes mirror of include/nicr.h: the configuration struct and constants.

The struct layout must match ``nicr_config`` field for field; the test suite
checks ``ctypes.sizeof(NicrConfig)`` against the C library's view.
"""
from __future__ import annotations

import ctypes

OK = 0
ERR_INVALID_ARG = 1
ERR_TRIAL_NONFINITE = 2
ERR_TRIAL_BOUNDS = 3
ERR_ETA_RANGE = 4
ERR_CUDA = 5
ERR_NO_DEVICE = 6
ERR_STATE = 7
ERR_IO = 8

BC = {"concentration": 0, "mu": 1, "closed": 2}
CK = {"legacy": 0, "off": 1}
BOUNDS = {"stop": 0, "legacy": 1}
NUCLEATION = {"ksp": 0, "center": 1, "off": 2}

FIELD = {
    "o": 0, "cr": 1, "p": 2, "eta": 3, "muO": 4, "muCr": 5, "mo": 6, "mc": 7,
    "gb": 8, "grain": 9, "eta_s2": 10, "eta_pairs": 11, "gb_initial": 12,
}


class NicrConfig(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("steps", ctypes.c_int), ("output_every", ctypes.c_int),
        ("left_edge_sites", ctypes.c_int),
        ("max_eta_fields", ctypes.c_int),
        ("random_seed", ctypes.c_ulonglong),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("grain_diameter_grid", ctypes.c_double), ("gb_fwhm_grid", ctypes.c_double),
        ("gb_factor_o", ctypes.c_double), ("gb_factor_cr", ctypes.c_double),
        ("radius_grid", ctypes.c_double), ("exclusion_gap_grid", ctypes.c_double),
        ("nucleation_period", ctypes.c_double),
        ("mu_res", ctypes.c_double), ("surface_c_ref", ctypes.c_double),
        ("bc", ctypes.c_int), ("ck", ctypes.c_int), ("bounds", ctypes.c_int), ("nucleation", ctypes.c_int),
        ("grains", ctypes.c_int), ("oxygen_diffusion", ctypes.c_int),
        ("grain_evolution", ctypes.c_int), ("frozen_eta_cache", ctypes.c_int),
        ("eta_W", ctypes.c_double), ("eta_kappa", ctypes.c_double),
        ("eta_L", ctypes.c_double), ("eta_oxide_penalty", ctypes.c_double),
        ("eta_output_all", ctypes.c_int),
        ("output_vti", ctypes.c_int),
        ("output_float64", ctypes.c_int),
        ("compression_level", ctypes.c_int),
        ("ksp", ctypes.c_double), ("bulk_cr", ctypes.c_double), ("layer_o", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
        ("checkpoint_every", ctypes.c_int),
        ("eta_colours", ctypes.c_int),
        ("step_form", ctypes.c_int),
        ("reserved", ctypes.c_int * 3),
    ]


def default_config(dim: int) -> NicrConfig:
    """Reference defaults: Config{} (2D:39-58 / 3S:43-72) and Physics (3S:73-79)."""
    c = NicrConfig()
    c.dim = dim
    c.nx, c.ny, c.nz = 151, 101, (101 if dim == 3 else 1)
    c.steps, c.output_every = 0, 5000
    c.left_edge_sites = 0
    c.max_eta_fields = 512
    c.random_seed = 20260909
    c.dx = c.dy = c.dz = 1e-8
    c.dt = 2e-10
    c.grain_diameter_grid, c.gb_fwhm_grid = 50.0, 4.0
    c.gb_factor_o, c.gb_factor_cr = 28.2, 563.0
    c.radius_grid, c.exclusion_gap_grid, c.nucleation_period = 5.5, 6.0, 1e-7
    c.mu_res, c.surface_c_ref = 364688.0, 0.0023
    c.bc, c.ck, c.bounds, c.nucleation = BC["concentration"], CK["legacy"], BOUNDS["stop"], NUCLEATION["ksp"]
    c.grains, c.oxygen_diffusion, c.grain_evolution, c.frozen_eta_cache = 1, 1, 0, 1
    c.eta_W, c.eta_kappa, c.eta_L, c.eta_oxide_penalty = 1e4, 0.0, 0.2, -1.0
    c.eta_output_all = 1
    c.output_vti, c.output_float64, c.compression_level = 1, 0, 1
    c.ksp, c.bulk_cr, c.layer_o = 1.28e-7, 0.1986, 0.0023
    c.precision = 0
    c.device = 0
    return c


_ENUMS = {"bc": BC, "ck": CK, "bounds": BOUNDS, "nucleation": NUCLEATION}
_BOOLS = ("grains", "oxygen_diffusion", "grain_evolution", "frozen_eta_cache")


def make_config(dim: int, **kw) -> NicrConfig:
    """Reference defaults overridden by keyword arguments; string options
    ("bc", "ck", "bounds", "nucleation") and on/off switches are accepted."""
    c = default_config(dim)
    for k, v in kw.items():
        if k in _ENUMS and isinstance(v, str):
            v = _ENUMS[k][v]
        elif k in _BOOLS and isinstance(v, str):
            v = {"on": 1, "off": 0}[v]
        elif k == "dx":
            c.dy = c.dz = v
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def config_to_flags(c: NicrConfig) -> list[str]:
    """The reference CLI flags (parse, 3S:986-1082) that reproduce config c."""
    inv = {k: {v: s for s, v in m.items()} for k, m in _ENUMS.items()}
    onoff = lambda b: "on" if b else "off"
    f = ["--nx", str(c.nx), "--ny", str(c.ny)]
    if c.dim == 3:
        f += ["--nz", str(c.nz)]
    f += ["--dx", repr(c.dx), "--dt", repr(c.dt), "--seed", str(c.random_seed),
          "--grain-diameter-grid", repr(c.grain_diameter_grid), "--gb-width-grid", repr(c.gb_fwhm_grid),
          "--gb-factor-o", repr(c.gb_factor_o), "--gb-factor-cr", repr(c.gb_factor_cr),
          "--radius-grid", repr(c.radius_grid), "--nucleation-period", repr(c.nucleation_period),
          "--mu-res", repr(c.mu_res), "--surface-c-ref", repr(c.surface_c_ref),
          "--bc", inv["bc"][c.bc], "--ck", inv["ck"][c.ck], "--bounds", inv["bounds"][c.bounds],
          "--nucleation", inv["nucleation"][c.nucleation],
          "--grains", onoff(c.grains), "--oxygen-diffusion", onoff(c.oxygen_diffusion),
          "--grain-evolution", onoff(c.grain_evolution),
          "--eta-W", repr(c.eta_W), "--eta-kappa", repr(c.eta_kappa), "--eta-L", repr(c.eta_L),
          "--eta-oxide-penalty", repr(c.eta_oxide_penalty), "--max-eta-fields", str(c.max_eta_fields),
          "--left-edge-sites", str(c.left_edge_sites)]
    if c.dim == 3:
        f += ["--frozen-eta-cache", onoff(c.frozen_eta_cache),
              "--output-format", "vti" if c.output_vti else "vtk",
              "--output-precision", "float64" if c.output_float64 else "float32",
              "--compression-level", str(c.compression_level)]
    return f
