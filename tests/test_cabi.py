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


def _dsatur(adj, k):
    """DSatur as nicr_colour_grains states it: most distinct coloured
    neighbour colours, then most neighbours, then lowest index; the lowest
    colour no coloured neighbour has, else the one fewest of them have."""
    ng = len(adj)
    colour = [-1] * ng
    degree = [int(sum(row)) for row in adj]
    for _ in range(ng):
        best, bsat = -1, -1
        for a in range(ng):
            if colour[a] >= 0:
                continue
            sat = len({colour[b] for b in range(ng) if adj[a][b] and colour[b] >= 0})
            if best < 0 or sat > bsat or (sat == bsat and degree[a] > degree[best]):
                best, bsat = a, sat
        count = [0] * k
        for b in range(ng):
            if adj[best][b] and colour[b] >= 0:
                count[colour[b]] += 1
        colour[best] = min(range(k), key=lambda q: (count[q], q))
    return colour


@pytest.mark.parametrize("ng,density,k", [(12, 0.3, 4), (40, 0.25, 8), (64, 0.12, 8), (30, 0.6, 5), (1, 0.0, 3)])
def test_colour_grains_is_dsatur(ng, density, k):
    """The grain colouring of the coloured eta initialisation (host code, no
    GPU): DSatur with the stated tie rules on random symmetric graphs."""
    import ctypes
    import numpy as np
    L = nicr.lib()
    rng = np.random.default_rng(ng * 7 + k)
    upper = np.triu(rng.random((ng, ng)) < density, 1)
    adj = (upper | upper.T).astype(np.uint8)
    out = np.zeros(ng, dtype=np.int32)
    rc = L.nicr_colour_grains(adj.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), ng, k,
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert rc == 0
    assert out.tolist() == _dsatur(adj.tolist(), k)
    if k >= ng:
        assert not any(adj[a, b] and out[a] == out[b] for a in range(ng) for b in range(ng))


def _noalloc():
    f = nicr.lib().nicr_step_noalloc
    f.argtypes = [ctypes.POINTER(nicr.NicrConfig)] + [ctypes.c_void_p] * 10
    f.restype = ctypes.c_int
    return f


def _no_gpu():
    from conftest import gpu_available
    return not gpu_available()


@pytest.mark.skipif(not _no_gpu(), reason="passes placeholder pointers; runs only where no GPU can be reached")
@pytest.mark.parametrize("precision", [2, -1, 7])
def test_noalloc_rejects_unknown_precision_before_the_device(precision):
    """nicr_step_noalloc accepts the forms nicr_create accepts (NICR_FP64 and
    NICR_FP64_FAST) and rejects others before any CUDA call. Non-null
    placeholder pointers get the call past its null checks: without the
    precision check it would reach the (absent) device and return
    NICR_ERR_NO_DEVICE or NICR_ERR_CUDA instead."""
    cfg = nicr.make_config(3, nx=16, ny=16, nz=32, grains=0, nucleation="off", precision=precision)
    ptrs = [ctypes.c_void_p(256 * (k + 1)) for k in range(10)]
    assert _noalloc()(ctypes.byref(cfg), *ptrs) == _abi.ERR_INVALID_ARG
    cfg.precision = 1
    assert _noalloc()(ctypes.byref(cfg), *ptrs) in (_abi.ERR_NO_DEVICE, _abi.ERR_CUDA)


def test_noalloc_rejects_too_many_tiles_before_the_device():
    """More than 8192 step tiles per X plane (3D: ceil(ny/8)*ceil(nz/32)) do
    not fit the scratch array at any X chunk: rejected before any CUDA call."""
    cfg = nicr.make_config(3, nx=4, ny=8 * 129, nz=32 * 64, grains=0, nucleation="off")
    assert _noalloc()(ctypes.byref(cfg), *([None] * 10)) == _abi.ERR_INVALID_ARG
