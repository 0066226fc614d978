"""Test infrastructure only: Python access to the CPU oracle.

* ``Oracle``: ctypes wrapper of the C restatement (oracle/_build/libnicr_oracle.so).
* ``run_reference``: runs the unmodified reference (oracle/_ref/ref{2,3}d, built
  by oracle/Makefile from the reference sources) through its driver and parses
  the tagged binary dumps it writes.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "ni-cr_oxidation_phase-field_simulation_b200"))
from nicr._abi import NicrConfig, config_to_flags, make_config  # noqa: E402

LIB_PATH = HERE / "_build" / "libnicr_oracle.so"
REF_DIR = HERE / "_ref"


def build(quiet: bool = True) -> None:
    """Builds the oracle library (and oracle/_ref when NICR_REF_DIR names the
    reference sources)."""
    import os
    out = subprocess.run(["make", "-C", str(HERE), "all", f"REF={os.environ.get('NICR_REF_DIR', '')}"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        lp = ctypes.POINTER(ctypes.c_longlong)
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_char_p, ctypes.c_int]
        L.oracle_destroy.argtypes = [P]
        L.oracle_ncells.restype = ctypes.c_longlong
        L.oracle_ncells.argtypes = [P]
        for f in ("oracle_neta", "oracle_nseeds", "oracle_center_seed_cells"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = ctypes.c_int
        L.oracle_get.argtypes = [P, ctypes.c_char_p, dp]
        L.oracle_set_fields.argtypes = [P, dp, dp, dp, dp]
        L.oracle_reset_inventory.argtypes = [P]
        L.oracle_refresh.argtypes = [P]
        L.oracle_invalidate.argtypes = [P]
        L.oracle_step.argtypes = [P]
        L.oracle_run.argtypes = [P, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.oracle_nucleate.argtypes = [P]
        L.oracle_stamp.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_scale_eta.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.oracle_error.restype = ctypes.c_char_p
        L.oracle_error.argtypes = [P]
        L.oracle_budget.argtypes = [P, dp, lp]
        L.oracle_seeds.argtypes = [P, dp, lp]
        L.oracle_log_values.argtypes = [P, dp]
        L.oracle_grain_values.argtypes = [P, dp, lp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


BUDGET_NAMES = ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")


class Oracle:
    """The C restatement of one reference Model (serial)."""

    def __init__(self, cfg: NicrConfig):
        self.cfg = cfg
        err = ctypes.create_string_buffer(1024)
        self.h = lib().oracle_create(ctypes.byref(cfg), err, 1024)
        if not self.h:
            raise RuntimeError(err.value.decode())
        self.n = lib().oracle_ncells(self.h)
        self.neta = lib().oracle_neta(self.h)
        self.shape = (cfg.nx, cfg.ny, cfg.nz) if cfg.dim == 3 else (cfg.nx, cfg.ny)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def get(self, name: str):
        out = np.empty(self.n)
        if lib().oracle_get(self.h, name.encode(), _dp(out)):
            return None
        return out.reshape(self.shape)

    def fields(self) -> dict:
        d = {k: self.get(k) for k in ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb", "grain", "eta_s2")}
        for g in range(self.neta):
            d[f"eta{g + 1}"] = self.get(f"eta{g + 1}")
        return {k: v for k, v in d.items() if v is not None}

    def set_fields(self, o, cr, p, eta=None):
        o, cr, p = (np.ascontiguousarray(x, dtype=np.float64).ravel() for x in (o, cr, p))
        e = None if eta is None else np.ascontiguousarray(eta, dtype=np.float64).ravel()
        lib().oracle_set_fields(self.h, _dp(o), _dp(cr), _dp(p), _dp(e) if e is not None else None)

    def reset_inventory(self):
        lib().oracle_reset_inventory(self.h)

    def refresh(self):
        lib().oracle_refresh(self.h)

    def invalidate(self):
        lib().oracle_invalidate(self.h)

    def step(self, n: int = 1) -> int:
        for _ in range(n):
            rc = lib().oracle_step(self.h)
            if rc:
                return rc
        return 0

    def run(self, n: int):
        done = ctypes.c_int(0)
        rc = lib().oracle_run(self.h, n, ctypes.byref(done))
        return rc, done.value

    def nucleate(self):
        lib().oracle_nucleate(self.h)

    def stamp(self, x, y, z=0) -> int:
        return lib().oracle_stamp(self.h, x, y, z)

    def scale_eta(self, g, i, j, k, f):
        lib().oracle_scale_eta(self.h, g, i, j, k, f)

    def error(self) -> str:
        return lib().oracle_error(self.h).decode()

    def budget(self) -> dict:
        hl = np.zeros(20)
        cnt = np.zeros(2, dtype=np.int64)
        lib().oracle_budget(self.h, _dp(hl), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        d = {n: (hl[2 * q], hl[2 * q + 1]) for q, n in enumerate(BUDGET_NAMES)}
        d["initialO"] = (hl[16], hl[17])
        d["initialCr"] = (hl[18], hl[19])
        d["nuclei"], d["clipped"] = int(cnt[0]), int(cnt[1])
        return d

    def seeds(self):
        ns = lib().oracle_nseeds(self.h)
        xyz = np.zeros(ns * self.cfg.dim)
        vol = np.zeros(ns, dtype=np.int64)
        lib().oracle_seeds(self.h, _dp(xyz), vol.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
        return xyz.reshape(ns, self.cfg.dim), vol

    def center_seed_cells(self) -> int:
        return lib().oracle_center_seed_cells(self.h)

    def log_values(self) -> dict:
        out = np.zeros(15)
        lib().oracle_log_values(self.h, _dp(out))
        return {"sum_O": (out[0], out[1]), "sum_Cr": (out[2], out[3]), "sum_phi": (out[4], out[5]),
                "sum_h": (out[6], out[7]), "min_O": out[8], "max_O": out[9], "min_Cr": out[10],
                "max_Cr": out[11], "min_Ni": out[12], "min_phi": out[13], "max_phi": out[14]}

    def grain_values(self):
        out = np.zeros(13)
        cells = np.zeros(max(self.neta, 1), dtype=np.int64)
        amount = np.zeros(2 * max(self.neta, 1))
        if lib().oracle_grain_values(self.h, _dp(out), cells.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dp(amount)):
            return None
        return {"min_eta": out[0], "max_eta": out[1], "min_s2": out[2], "max_s2": out[3],
                "sum_s2": (out[4], out[5]), "mask": (out[6], out[7]), "energy": (out[8], out[9]),
                "gb_max": out[10], "alive": int(out[11]), "unassigned": int(out[12]),
                "cells": cells[: self.neta], "amount": amount[: 2 * self.neta].reshape(-1, 2)}


# ------------------------------------------------------------------ reference
def read_dump(path) -> dict:
    """Parses a NICRDUMP file written by oracle/ref_driver.cpp."""
    b = Path(path).read_bytes()
    assert b[:8] == b"NICRDUMP"
    off, out = 8, {}
    while off < len(b):
        name = b[off:off + 32].split(b"\0", 1)[0].decode()
        kind, _pad, count = struct.unpack_from("<iiq", b, off + 32)
        off += 48
        if kind == 1:
            out[name] = np.frombuffer(b, dtype="<f8", count=count, offset=off).copy(); off += 8 * count
        elif kind == 2:
            out[name] = np.frombuffer(b, dtype="<i8", count=count, offset=off).copy(); off += 8 * count
        else:
            out[name] = np.frombuffer(b, dtype="<f8", count=2 * count, offset=off).reshape(count, 2).copy(); off += 16 * count
    return out


def reference_available(dim: int = 3) -> bool:
    return (REF_DIR / f"ref{dim}d").exists()


def run_reference(cfg: NicrConfig, commands: list, inject: dict | None = None, workdir=None,
                  threads: int = 0, timeout: float = 600) -> dict:
    """Runs the unmodified reference on cfg. commands are driver commands;
    "dump" entries (no argument) are replaced by numbered dump files whose
    parsed contents are returned under "dumps". inject = {"o":..,"cr":..,"p":..,"eta":[..]}."""
    exe = REF_DIR / (f"ref{cfg.dim}d_threads" if threads else f"ref{cfg.dim}d")
    if not exe.exists():
        raise FileNotFoundError(exe)
    tmp = tempfile.TemporaryDirectory(prefix="nicr-ref-") if workdir is None else None
    wd = Path(workdir or tmp.name)
    cmd_args, dumps = [], []
    if inject is not None:
        arrays = [inject["o"], inject["cr"], inject["p"]] + list(inject.get("eta", []))
        path = wd / "inject.bin"
        with open(path, "wb") as f:
            for a in arrays:
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        cmd_args += ["inject", str(path)]
    for c in commands:
        c = [str(x) for x in (c if isinstance(c, (list, tuple)) else [c])]
        if c[0] == "dump" and len(c) == 1:
            p = wd / f"dump{len(dumps)}.bin"
            dumps.append(p)
            c = ["dump", str(p)]
        cmd_args += c
    argv = [str(exe)] + ([str(threads)] if threads else []) + config_to_flags(cfg) + ["--"] + cmd_args
    r = subprocess.run(argv, capture_output=True, text=True, timeout=timeout, cwd=wd)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr}\n{r.stdout}")
    res = {"stdout": r.stdout, "dumps": [read_dump(p) for p in dumps], "workdir": wd, "_tmp": tmp}
    return res


__all__ = ["Oracle", "make_config", "run_reference", "read_dump", "reference_available", "build", "BUDGET_NAMES"]
