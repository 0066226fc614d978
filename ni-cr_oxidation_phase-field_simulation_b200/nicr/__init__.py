"""Python access to the B200 Ni-Cr oxidation solver through its C-ABI.

``Solver`` wraps one ``nicr_handle`` (include/nicr.h): a domain resident on the
GPU. The methods mirror the reference's ``Model`` members (step, refresh,
nucleate, stamp, log/grain_log values) and exchange fields as numpy arrays in
the reference's interior order (X slowest). The compute runs only in the CUDA
library ``lib/libnicr.so``; importing this module raises if it is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from ._abi import (BC, BOUNDS, CK, FIELD, NUCLEATION, NicrConfig, config_to_flags, default_config,
                   make_config)

PKG = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ["NICR_LIBRARY"]) if os.environ.get("NICR_LIBRARY") else PKG / "lib" / "libnicr.so"

_lib = None


class NicrError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class NicrInfo(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("n_seeds", ctypes.c_int), ("n_eta", ctypes.c_int), ("center_seed_cells", ctypes.c_int),
                ("grain_map_retained", ctypes.c_int), ("n_cells", ctypes.c_longlong),
                ("steps_done", ctypes.c_longlong), ("device_bytes", ctypes.c_size_t)]


class NicrBudget(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 2) for n in ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")] + \
               [("nuclei", ctypes.c_longlong), ("clipped", ctypes.c_longlong),
                ("initialO", ctypes.c_double * 2), ("initialCr", ctypes.c_double * 2)]


class NicrDiagnostics(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 2) for n in ("sum_O", "sum_Cr", "sum_phi", "sum_h")] + \
               [(n, ctypes.c_double) for n in ("min_O", "max_O", "min_Cr", "max_Cr", "min_Ni", "min_phi", "max_phi")]


class NicrGrainStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("min_eta", "max_eta", "min_s2", "max_s2")] + \
               [(n, ctypes.c_double * 2) for n in ("sum_s2", "mask", "energy")] + \
               [("gb_max", ctypes.c_double), ("alive", ctypes.c_longlong), ("unassigned", ctypes.c_longlong)]


def library_path() -> Path:
    return LIB_PATH


def lib():
    """Loads lib/libnicr.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"CUDA library {LIB_PATH} is missing: run `make -C {PKG}` (or __graft_entry__.build())")
    L = ctypes.CDLL(str(LIB_PATH))
    H = ctypes.c_void_p
    ip = ctypes.POINTER(ctypes.c_int)
    dp = ctypes.POINTER(ctypes.c_double)
    L.nicr_config_default.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_int]
    L.nicr_config_default.restype = None
    L.nicr_config_parse.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_char_p), ctypes.c_char_p, ctypes.c_size_t, ip,
                                    ctypes.c_char_p, ctypes.c_size_t]
    L.nicr_create.argtypes = [ctypes.POINTER(NicrConfig), ctypes.POINTER(H)]
    L.nicr_destroy.argtypes = [H]
    L.nicr_destroy.restype = None
    L.nicr_last_error.argtypes = [H]
    L.nicr_last_error.restype = ctypes.c_char_p
    L.nicr_get_info.argtypes = [H, ctypes.POINTER(NicrInfo)]
    L.nicr_get_seeds.argtypes = [H, dp, ctypes.POINTER(ctypes.c_longlong)]
    L.nicr_set_field.argtypes = [H, ctypes.c_int, ctypes.c_int, dp]
    L.nicr_get_field.argtypes = [H, ctypes.c_int, ctypes.c_int, dp]
    for f in ("nicr_refresh", "nicr_invalidate_eta_cache", "nicr_reset_inventory"):
        getattr(L, f).argtypes = [H]
    L.nicr_step.argtypes = [H, ctypes.c_int, ip]
    L.nicr_run.argtypes = [H, ctypes.c_int, ip]
    L.nicr_nucleate.argtypes = [H, ip]
    L.nicr_stamp.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip]
    L.nicr_get_budget.argtypes = [H, ctypes.POINTER(NicrBudget)]
    L.nicr_get_diagnostics.argtypes = [H, ctypes.POINTER(NicrDiagnostics)]
    L.nicr_get_grain_stats.argtypes = [H, ctypes.POINTER(NicrGrainStats), ctypes.POINTER(ctypes.c_longlong), dp]
    L.nicr_write_vtk.argtypes = [H, ctypes.c_char_p]
    L.nicr_write_vti.argtypes = [H, ctypes.c_char_p]
    L.nicr_write_vti_async.argtypes = [H, ctypes.c_char_p]
    L.nicr_output_wait.argtypes = [H]
    L.nicr_write_metadata.argtypes = [H, ctypes.c_char_p]
    L.nicr_format_log_row.argtypes = [H, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    L.nicr_format_grain_rows.argtypes = [H, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p,
                                         ctypes.c_size_t]
    L.nicr_main.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
    L.nicr_stream.argtypes = [H]
    L.nicr_stream.restype = ctypes.c_void_p
    L.nicr_field_device.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_longlong)]
    L.nicr_tune.argtypes = [H, ctypes.c_int, ip, ip]
    L.nicr_batch_tune.argtypes = [H, ctypes.c_int, ip]
    L.nicr_save_state.argtypes = [H, ctypes.c_char_p]
    L.nicr_load_state.argtypes = [H, ctypes.c_char_p]
    L.nicr_batch_create.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_int, ctypes.POINTER(H)]
    L.nicr_batch_destroy.argtypes = [H]
    L.nicr_batch_destroy.restype = None
    L.nicr_batch_size.argtypes = [H]
    L.nicr_batch_domain.argtypes = [H, ctypes.c_int]
    L.nicr_batch_domain.restype = H
    L.nicr_batch_step.argtypes = [H, ctypes.c_int, ip]
    L.nicr_batch_run.argtypes = [H, ctypes.c_int, ip]
    L.nicr_batch_last_error.argtypes = [H]
    L.nicr_batch_last_error.restype = ctypes.c_char_p
    L.nicr_batch_kernel_launches.argtypes = [H]
    L.nicr_batch_kernel_launches.restype = ctypes.c_longlong
    L.nicr_batch_stream.argtypes = [H]
    L.nicr_batch_stream.restype = ctypes.c_void_p
    L.nicr_kernel_launches.argtypes = [H]
    L.nicr_kernel_launches.restype = ctypes.c_longlong
    L.nicr_slabs_create.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_int, ip, ctypes.POINTER(H)]
    L.nicr_slabs_destroy.argtypes = [H]
    L.nicr_slabs_destroy.restype = None
    L.nicr_slabs_count.argtypes = [H]
    L.nicr_slabs_info.argtypes = [H, ctypes.c_int, ip, ip, ip, ip]
    L.nicr_slabs_step.argtypes = [H, ctypes.c_int, ip]
    L.nicr_slabs_run.argtypes = [H, ctypes.c_int, ip]
    L.nicr_slabs_nucleate.argtypes = [H, ip]
    L.nicr_slabs_get_field.argtypes = [H, ctypes.c_int, ctypes.c_int, dp]
    L.nicr_slabs_set_field.argtypes = [H, ctypes.c_int, ctypes.c_int, dp]
    L.nicr_slabs_reset_inventory.argtypes = [H]
    L.nicr_slabs_get_budget.argtypes = [H, ctypes.POINTER(NicrBudget)]
    L.nicr_slabs_get_diagnostics.argtypes = [H, ctypes.POINTER(NicrDiagnostics)]
    L.nicr_slabs_steps_done.argtypes = [H]
    L.nicr_slabs_steps_done.restype = ctypes.c_longlong
    L.nicr_slabs_kernel_launches.argtypes = [H]
    L.nicr_slabs_kernel_launches.restype = ctypes.c_longlong
    L.nicr_slabs_get_grain_stats.argtypes = [H, ctypes.POINTER(NicrGrainStats), ctypes.POINTER(ctypes.c_longlong), dp]
    L.nicr_slabs_write_vti.argtypes = [H, ctypes.c_char_p]
    L.nicr_slabs_n_eta.argtypes = [H]
    L.nicr_slabs_stream.argtypes = [H, ctypes.c_int]
    L.nicr_slabs_stream.restype = ctypes.c_void_p
    vp = ctypes.POINTER(ctypes.c_void_p)
    L.nicr_slab_create.argtypes = [ctypes.POINTER(NicrConfig), ctypes.c_int, ctypes.c_int, ctypes.POINTER(H)]
    L.nicr_slab_info.argtypes = [H, ip, ip, ip, ip, ip, ip]
    L.nicr_slab_region.argtypes = [H, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                   ctypes.POINTER(ctypes.c_longlong)]
    L.nicr_slab_adjacency.argtypes = [H, ctypes.POINTER(ctypes.c_ubyte)]
    L.nicr_colour_grains.argtypes = [ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int, ctypes.c_int, ip]
    L.nicr_slab_set_colours.argtypes = [H, ip]
    L.nicr_slab_begin.argtypes = [H, ctypes.c_int, ctypes.c_int]
    L.nicr_slab_scan_due.argtypes = [H, ctypes.c_int]
    L.nicr_slab_note_step.argtypes = [H, ctypes.c_int, ctypes.c_int]
    L.nicr_slab_failed.argtypes = [H, ip]
    L.nicr_slab_launch.argtypes = [H]
    L.nicr_slab_agree_word.argtypes = [H]
    L.nicr_slab_agree_word.restype = ctypes.c_void_p
    L.nicr_slab_commit.argtypes = [H]
    L.nicr_slab_end.argtypes = [H, ctypes.c_int, ip]
    L.nicr_slab_scan_candidates.argtypes = [H]
    L.nicr_slab_scan_resolve.argtypes = [H, ip, ctypes.c_int, ip, ctypes.c_int, ip, ip]
    L.nicr_slab_scan_apply.argtypes = [H, ip, ctypes.c_int]
    L.nicr_slab_box_half.argtypes = [H]
    L.nicr_slabs_last_error.argtypes = [H]
    L.nicr_slabs_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def c_default_config(dim: int) -> NicrConfig:
    c = NicrConfig()
    lib().nicr_config_default(ctypes.byref(c), dim)
    return c


def parse_args(dim: int, argv: list[str]):
    """nicr_config_parse: returns (config, out_dir, self_test) or raises NicrError."""
    c = NicrConfig()
    arr = (ctypes.c_char_p * max(1, len(argv)))(*[a.encode() for a in argv])
    out = ctypes.create_string_buffer(4096)
    err = ctypes.create_string_buffer(8192)
    st = ctypes.c_int(0)
    rc = lib().nicr_config_parse(ctypes.byref(c), dim, len(argv), arr, out, 4096, ctypes.byref(st), err, 8192)
    if rc != 0:
        raise NicrError(rc, err.value.decode())
    return c, out.value.decode(), bool(st.value)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _DeviceArray:
    """__cuda_array_interface__ of an FP64 device array owned by a handle."""

    def __init__(self, ptr: int, shape, strides):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "strides": tuple(strides), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3, "stream": None}


class Solver:
    """One simulation domain on the GPU (the reference's Model)."""

    def __init__(self, cfg: NicrConfig | None = None, dim: int = 3, **kw):
        if cfg is None:
            cfg = make_config(dim, **kw)
        self.cfg = cfg
        self.owner = None
        self.h = ctypes.c_void_p()
        rc = lib().nicr_create(ctypes.byref(cfg), ctypes.byref(self.h))
        if rc != 0:
            raise NicrError(rc, lib().nicr_last_error(None).decode())
        self._describe()

    def _describe(self):
        cfg = self.cfg
        self.info_ = self.info()
        self.shape = (cfg.nx, cfg.ny, cfg.nz) if cfg.dim == 3 else (cfg.nx, cfg.ny)
        self.n = int(np.prod(self.shape))

    @classmethod
    def _borrowed(cls, handle: int, cfg: NicrConfig, owner):
        """A domain handle owned by a Batch (freed with the batch)."""
        s = cls.__new__(cls)
        s.cfg = cfg
        s.owner = owner
        s.h = ctypes.c_void_p(handle)
        s._describe()
        return s

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            if getattr(self, "owner", None) is None:
                lib().nicr_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -------------------------------------------------------------- helpers
    def _check(self, rc: int):
        if rc != 0:
            raise NicrError(rc, self.last_error)
        return rc

    @property
    def last_error(self) -> str:
        return lib().nicr_last_error(self.h).decode()

    def info(self) -> NicrInfo:
        i = NicrInfo()
        self._check(lib().nicr_get_info(self.h, ctypes.byref(i)))
        return i

    @property
    def n_eta(self) -> int:
        return self.info().n_eta

    def seeds(self):
        i = self.info()
        xyz = np.zeros(i.n_seeds * self.cfg.dim)
        vol = np.zeros(i.n_seeds, dtype=np.int64)
        self._check(lib().nicr_get_seeds(self.h, _dp(xyz), vol.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return xyz.reshape(i.n_seeds, self.cfg.dim), vol

    def get(self, name: str, index: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Field values in interior order; `out` (contiguous float64, one value
        per cell, e.g. pinned host memory) receives them without a copy."""
        if name.startswith("eta") and name[3:].isdigit():
            index, name = int(name[3:]) - 1, "eta"
        if out is None:
            out = np.empty(self.n)
        elif out.dtype != np.float64 or out.size != self.n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array with one value per cell")
        self._check(lib().nicr_get_field(self.h, FIELD[name], index, _dp(out)))
        return out.reshape(self.shape)

    def set(self, name: str, arr, index: int = 0):
        if name.startswith("eta") and name[3:].isdigit():
            index, name = int(name[3:]) - 1, "eta"
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        if a.size != self.n:
            raise ValueError(f"field has {a.size} values, grid has {self.n}")
        self._check(lib().nicr_set_field(self.h, FIELD[name], index, _dp(a)))

    def set_fields(self, o, cr, p, eta=None):
        self.set("o", o)
        self.set("cr", cr)
        self.set("p", p)
        if eta is not None:
            for g, e in enumerate(eta):
                self.set("eta", e, g)

    def refresh(self):
        self._check(lib().nicr_refresh(self.h))

    def invalidate_eta_cache(self):
        self._check(lib().nicr_invalidate_eta_cache(self.h))

    def reset_inventory(self):
        self._check(lib().nicr_reset_inventory(self.h))

    def step(self, n: int = 1, check: bool = True):
        done = ctypes.c_int(0)
        rc = lib().nicr_step(self.h, n, ctypes.byref(done))
        if check:
            self._check(rc)
        return rc, done.value

    def run(self, n: int, check: bool = True):
        done = ctypes.c_int(0)
        rc = lib().nicr_run(self.h, n, ctypes.byref(done))
        if check:
            self._check(rc)
        return rc, done.value

    def nucleate(self) -> int:
        k = ctypes.c_int(0)
        self._check(lib().nicr_nucleate(self.h, ctypes.byref(k)))
        return k.value

    def stamp(self, x: int, y: int, z: int = 0) -> int:
        k = ctypes.c_int(0)
        self._check(lib().nicr_stamp(self.h, x, y, z, ctypes.byref(k)))
        return k.value

    def budget(self) -> dict:
        b = NicrBudget()
        self._check(lib().nicr_get_budget(self.h, ctypes.byref(b)))
        d = {n: (getattr(b, n)[0], getattr(b, n)[1]) for n in
             ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr", "initialO", "initialCr")}
        d["nuclei"], d["clipped"] = int(b.nuclei), int(b.clipped)
        return d

    def diagnostics(self) -> dict:
        d = NicrDiagnostics()
        self._check(lib().nicr_get_diagnostics(self.h, ctypes.byref(d)))
        out = {n: (getattr(d, n)[0], getattr(d, n)[1]) for n in ("sum_O", "sum_Cr", "sum_phi", "sum_h")}
        for n in ("min_O", "max_O", "min_Cr", "max_Cr", "min_Ni", "min_phi", "max_phi"):
            out[n] = getattr(d, n)
        return out

    def grain_stats(self):
        ne = max(1, self.n_eta)
        s = NicrGrainStats()
        cells = np.zeros(ne, dtype=np.int64)
        amount = np.zeros(2 * ne)
        self._check(lib().nicr_get_grain_stats(self.h, ctypes.byref(s), cells.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dp(amount)))
        out = {n: getattr(s, n) for n in ("min_eta", "max_eta", "min_s2", "max_s2", "gb_max")}
        for n in ("sum_s2", "mask", "energy"):
            out[n] = (getattr(s, n)[0], getattr(s, n)[1])
        out["alive"], out["unassigned"] = int(s.alive), int(s.unassigned)
        out["cells"] = cells[: self.n_eta]
        out["amount"] = amount[: 2 * self.n_eta].reshape(-1, 2)
        return out

    def tune(self, reps: int = 3):
        """Measures and keeps the fastest X chunk / occupancy variant (nicr_tune);
        returns (xchunk, minb). The state is unchanged."""
        c, m = ctypes.c_int(0), ctypes.c_int(0)
        self._check(lib().nicr_tune(self.h, reps, ctypes.byref(c), ctypes.byref(m)))
        return c.value, m.value

    def save(self, path):
        """Checkpoint of the current state (nicr_save_state)."""
        self._check(lib().nicr_save_state(self.h, str(path).encode()))

    def load(self, path):
        """Restores a checkpoint written from the same configuration (nicr_load_state)."""
        self._check(lib().nicr_load_state(self.h, str(path).encode()))

    def write_vtk(self, path):
        self._check(lib().nicr_write_vtk(self.h, str(path).encode()))

    def write_vti(self, path):
        self._check(lib().nicr_write_vti(self.h, str(path).encode()))

    def write_vti_async(self, path):
        """Starts a VTI frame of the current state; stepping may continue at once."""
        self._check(lib().nicr_write_vti_async(self.h, str(path).encode()))

    def output_wait(self):
        """Completes the pending asynchronous frame (raises its error)."""
        self._check(lib().nicr_output_wait(self.h))

    def write_metadata(self, out_dir):
        self._check(lib().nicr_write_metadata(self.h, str(out_dir).encode()))

    def log_row(self, n: int) -> str:
        buf = ctypes.create_string_buffer(8192)
        self._check(lib().nicr_format_log_row(self.h, n, buf, 8192))
        return buf.value.decode()

    def grain_rows(self, n: int):
        sz = 4096 + 256 * max(1, self.n_eta)
        a, b = ctypes.create_string_buffer(sz), ctypes.create_string_buffer(sz)
        self._check(lib().nicr_format_grain_rows(self.h, n, a, sz, b, sz))
        return a.value.decode(), b.value.decode()

    def stream(self) -> int:
        return lib().nicr_stream(self.h) or 0

    def device_view(self, name: str, index: int = 0, writable: bool = False):
        """The field's device storage as a torch tensor (no copy), shaped like
        get(): valid until the next call that steps, nucleates, loads or sets
        fields (nicr_field_device). writable=True for o, cr, p and eta; the
        caller synchronises its stream before the next call on the handle."""
        import torch
        if name.startswith("eta") and name[3:].isdigit():
            index, name = int(name[3:]) - 1, "eta"
        ptr, pitch = ctypes.c_void_p(), ctypes.c_longlong()
        self._check(lib().nicr_field_device(self.h, FIELD[name], index, int(writable), ctypes.byref(ptr),
                                            ctypes.byref(pitch)))
        i = self.info()
        rows = i.ny if i.dim == 3 else 1
        cols = i.nz if i.dim == 3 else i.ny
        # torch takes no read-only CUDA arrays: a read view must not be written
        view = _DeviceArray(ptr.value, (i.nx, rows, cols), (rows * pitch.value * 8, pitch.value * 8, 8))
        t = torch.as_tensor(view, device=f"cuda:{self.cfg.device}")
        return t if i.dim == 3 else t[:, 0, :]


class Batch:
    """Independent domains on one GPU advanced together (nicr_batch_*): one
    step launch per group of up to 48 domains, one commit launch per step.
    ``domains[i]`` is a Solver view of domain i (owned by the batch)."""

    def __init__(self, cfgs):
        cfgs = list(cfgs)
        arr = (NicrConfig * len(cfgs))(*cfgs)
        self.b = ctypes.c_void_p()
        rc = lib().nicr_batch_create(arr, len(cfgs), ctypes.byref(self.b))
        if rc != 0:
            raise NicrError(rc, lib().nicr_batch_last_error(None).decode())
        self.domains = [Solver._borrowed(lib().nicr_batch_domain(self.b, i), cfgs[i], self)
                        for i in range(len(cfgs))]

    def __len__(self):
        return len(self.domains)

    def close(self):
        if getattr(self, "b", None) and self.b.value:
            for d in self.domains:
                d.h = ctypes.c_void_p()
            lib().nicr_batch_destroy(self.b)
            self.b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def last_error(self) -> str:
        return lib().nicr_batch_last_error(self.b).decode()

    def _advance(self, fn, n: int, check: bool):
        done = (ctypes.c_int * len(self.domains))()
        rc = fn(self.b, n, done)
        if check and rc != 0:
            raise NicrError(rc, self.last_error)
        return list(done), rc

    def step(self, n: int = 1, check: bool = True):
        """Model::step x n on every domain; returns (completed per domain, status)."""
        return self._advance(lib().nicr_batch_step, n, check)

    def run(self, n: int, check: bool = True):
        """n steps of every domain on its run() schedule (Ksp scans)."""
        return self._advance(lib().nicr_batch_run, n, check)

    def tune(self, reps: int = 3) -> int:
        """Measures and keeps the fastest common X chunk (nicr_batch_tune)."""
        c = ctypes.c_int(0)
        rc = lib().nicr_batch_tune(self.b, reps, ctypes.byref(c))
        if rc != 0:
            raise NicrError(rc, self.last_error)
        return c.value

    @property
    def kernel_launches(self) -> int:
        return int(lib().nicr_batch_kernel_launches(self.b))

    @property
    def stream(self) -> int:
        return lib().nicr_batch_stream(self.b) or 0


class Slabs:
    """One 3D domain split along X into slabs (nicr_slabs_*), slab i on GPU
    devices[i] (several slabs may share a GPU). Fields, budgets and
    diagnostics are whole-domain, as a Solver's."""

    def __init__(self, cfg: NicrConfig, nslabs: int, devices=None):
        self.cfg = cfg
        self.s = ctypes.c_void_p()
        dev = None
        if devices is not None:
            devices = list(devices)
            if len(devices) != nslabs:
                raise ValueError("one device per slab")
            dev = (ctypes.c_int * nslabs)(*devices)
        rc = lib().nicr_slabs_create(ctypes.byref(cfg), nslabs, dev, ctypes.byref(self.s))
        if rc != 0:
            raise NicrError(rc, lib().nicr_slabs_last_error(None).decode())
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        self.n = int(np.prod(self.shape))

    def close(self):
        if getattr(self, "s", None) and self.s.value:
            lib().nicr_slabs_destroy(self.s)
            self.s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise NicrError(rc, self.last_error)
        return rc

    @property
    def last_error(self) -> str:
        return lib().nicr_slabs_last_error(self.s).decode()

    def __len__(self):
        return lib().nicr_slabs_count(self.s)

    def slab(self, i: int) -> dict:
        """Domain planes [x0, x1) of slab i, its device and the halo width."""
        v = [ctypes.c_int(0) for _ in range(4)]
        self._check(lib().nicr_slabs_info(self.s, i, *[ctypes.byref(q) for q in v]))
        return {"x0": v[0].value, "x1": v[1].value, "device": v[2].value, "halo": v[3].value}

    def get(self, name: str, index: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        if name.startswith("eta") and name[3:].isdigit():
            index, name = int(name[3:]) - 1, "eta"
        if out is None:
            out = np.empty(self.n)
        elif out.dtype != np.float64 or out.size != self.n or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous float64 array with one value per cell")
        self._check(lib().nicr_slabs_get_field(self.s, FIELD[name], index, _dp(out)))
        return out.reshape(self.shape)

    def set(self, name: str, arr, index: int = 0):
        if name.startswith("eta") and name[3:].isdigit():
            index, name = int(name[3:]) - 1, "eta"
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        if a.size != self.n:
            raise ValueError(f"field has {a.size} values, grid has {self.n}")
        self._check(lib().nicr_slabs_set_field(self.s, FIELD[name], index, _dp(a)))

    def reset_inventory(self):
        self._check(lib().nicr_slabs_reset_inventory(self.s))

    def step(self, n: int = 1, check: bool = True):
        done = ctypes.c_int(0)
        rc = lib().nicr_slabs_step(self.s, n, ctypes.byref(done))
        if check:
            self._check(rc)
        return rc, done.value

    def run(self, n: int, check: bool = True):
        done = ctypes.c_int(0)
        rc = lib().nicr_slabs_run(self.s, n, ctypes.byref(done))
        if check:
            self._check(rc)
        return rc, done.value

    def nucleate(self) -> int:
        k = ctypes.c_int(0)
        self._check(lib().nicr_slabs_nucleate(self.s, ctypes.byref(k)))
        return k.value

    def budget(self) -> dict:
        b = NicrBudget()
        self._check(lib().nicr_slabs_get_budget(self.s, ctypes.byref(b)))
        d = {n: (getattr(b, n)[0], getattr(b, n)[1]) for n in
             ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr", "initialO", "initialCr")}
        d["nuclei"], d["clipped"] = int(b.nuclei), int(b.clipped)
        return d

    def diagnostics(self) -> dict:
        d = NicrDiagnostics()
        self._check(lib().nicr_slabs_get_diagnostics(self.s, ctypes.byref(d)))
        out = {n: (getattr(d, n)[0], getattr(d, n)[1]) for n in ("sum_O", "sum_Cr", "sum_phi", "sum_h")}
        for n in ("min_O", "max_O", "min_Cr", "max_Cr", "min_Ni", "min_phi", "max_phi"):
            out[n] = getattr(d, n)
        return out

    def grain_stats(self):
        """nicr_slabs_get_grain_stats, in the form Solver.grain_stats returns."""
        ne = max(1, self.n_eta)
        s = NicrGrainStats()
        cells = np.zeros(ne, dtype=np.int64)
        amount = np.zeros(2 * ne)
        self._check(lib().nicr_slabs_get_grain_stats(self.s, ctypes.byref(s),
                                                     cells.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                                                     _dp(amount)))
        out = {n: getattr(s, n) for n in ("min_eta", "max_eta", "min_s2", "max_s2", "gb_max")}
        for n in ("sum_s2", "mask", "energy"):
            out[n] = (getattr(s, n)[0], getattr(s, n)[1])
        out["alive"], out["unassigned"] = int(s.alive), int(s.unassigned)
        out["cells"] = cells[: self.n_eta]
        out["amount"] = amount[: 2 * self.n_eta].reshape(-1, 2)
        return out

    def write_vti(self, path):
        self._check(lib().nicr_slabs_write_vti(self.s, str(path).encode()))

    @property
    def n_eta(self) -> int:
        return int(lib().nicr_slabs_n_eta(self.s))

    @property
    def steps_done(self) -> int:
        return int(lib().nicr_slabs_steps_done(self.s))

    @property
    def kernel_launches(self) -> int:
        return int(lib().nicr_slabs_kernel_launches(self.s))

    def stream(self, i: int) -> int:
        """The CUDA stream slab i enqueues on."""
        return lib().nicr_slabs_stream(self.s, i) or 0


def main(dim: int, argv: list[str]) -> int:
    """Runs the solver program (the reference's run()) with argv."""
    args = ["nicr%dd" % dim] + list(argv)
    arr = (ctypes.c_char_p * len(args))(*[a.encode() for a in args])
    return lib().nicr_main(dim, len(args), arr)


__all__ = ["Solver", "Batch", "Slabs", "NicrError", "NicrConfig", "make_config", "default_config", "c_default_config", "parse_args",
           "config_to_flags", "main", "lib", "library_path", "BC", "CK", "BOUNDS", "NUCLEATION", "FIELD"]
