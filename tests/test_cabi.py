"""C-ABI surface checks that need no GPU: the library loads, exports every
entry point include/nicr.h declares, and its config struct, defaults and
command-line parser agree with the reference's (parse, 3S:986-1082)."""
import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT
import nicr
from nicr import _abi


def declared_functions():
    text = (ROOT / "include" / "nicr.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nicr_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = nicr.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("dim", [2, 3])
def test_default_config_matches_python_mirror(dim):
    c = nicr.c_default_config(dim)
    p = _abi.default_config(dim)
    for name, _t in _abi.NicrConfig._fields_:
        if name == "reserved":
            continue
        assert getattr(c, name) == getattr(p, name), name


def test_parse_reference_flags():
    c, out, st = nicr.parse_args(3, ["--nx", "64", "--ny", "32", "--nz", "16", "--bc", "mu", "--ck", "off",
                                     "--bounds", "legacy", "--grain-evolution", "on", "--out", "x", "--self-test"])
    assert (c.nx, c.ny, c.nz) == (64, 32, 16)
    assert c.bc == _abi.BC["mu"] and c.ck == _abi.CK["off"] and c.bounds == _abi.BOUNDS["legacy"]
    assert c.grain_evolution == 1 and out == "x" and st


@pytest.mark.parametrize("argv,msg", [
    (["--bc", "wall"], "Invalid bc."),
    (["--nx", "2"], "Invalid parameter bounds (Ksp nucleation period must be >= dt)."),
    (["--grains", "maybe"], "--grains expects on or off (received: maybe)"),
    (["--bogus", "1"], "Unknown argument: --bogus"),
    (["--nucleation", "ksp", "--radius-grid", "60", "--ny", "100", "--nz", "100"],
     "Ksp sphere radius must be less than min(ny,nz)/2 to avoid periodic self-overlap."),
    (["--compression-level", "12"], "--compression-level must lie in [0,9]."),
    (["--steps"], "Missing value for --steps"),
])
def test_parse_errors_match_reference_messages(argv, msg):
    with pytest.raises(nicr.NicrError) as e:
        nicr.parse_args(3, argv)
    assert e.value.message == msg


def test_version_strings():
    with pytest.raises(nicr.NicrError) as e:
        nicr.parse_args(3, ["--version"])
    assert e.value.code == 100 and e.value.message.strip() == "mpi-eta-3d-xslab-optimized-v1"
    with pytest.raises(nicr.NicrError) as e:
        nicr.parse_args(2, ["--version"])
    assert e.value.message.strip() == "mpi-eta-v1"
