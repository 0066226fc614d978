"""The 3D program over a slab group (--slabs N): the same output files as
the single-GPU program on the same flags. VTI frames and grains.csv byte for
byte; diagnostics.csv, grain_diagnostics.csv and grain_history.csv value for
value (integer columns exactly, sums to 1e-13 relative: budgets and
reductions are summed per slab); parameters.txt differs only in the backend
and device-memory lines. Also a rejected trial (bounds=stop): the same
STOPPED.txt message and state_at_failure frame."""
import csv
import math
import os

import pytest

import nicr

pytestmark = pytest.mark.gpu

BASE = ["--nx", "40", "--ny", "24", "--nz", "32", "--grain-diameter-grid", "11", "--grain-evolution", "on",
        "--seed", "3", "--nucleation", "ksp", "--dt", "1e-12", "--radius-grid", "2.5", "--nucleation-period", "5e-12",
        "--steps", "30", "--output-every", "10", "--bounds", "legacy"]


def run(tmp_path, name, extra):
    out = str(tmp_path / name)
    assert nicr.main(3, BASE + extra + ["--out", out]) == 0
    return out


def read(path):
    with open(path, "rb") as f:
        return f.read()


def assert_csv_close(a, b, rtol=1e-13):
    with open(a) as fa, open(b) as fb:
        ra, rb = list(csv.reader(fa)), list(csv.reader(fb))
    assert len(ra) == len(rb) and ra[0] == rb[0], a
    for la, lb in zip(ra[1:], rb[1:]):
        for x, y, col in zip(la, lb, ra[0]):
            if x == y:
                continue
            fx, fy = float(x), float(y)
            assert not (x.lstrip("-").isdigit() and y.lstrip("-").isdigit()), (a, col, x, y)
            assert abs(fx - fy) <= rtol * (1.0 + abs(fy)) or math.isclose(fx, fy, rel_tol=rtol), (a, col, x, y)


def compare_outputs(one, many):
    names = sorted(os.listdir(one))
    assert names == sorted(os.listdir(many))
    for n in names:
        pa, pb = os.path.join(one, n), os.path.join(many, n)
        if n.endswith(".vti") or n == "grains.csv":
            assert read(pa) == read(pb), n
        elif n.endswith(".csv"):
            assert_csv_close(pa, pb)
        elif n == "parameters.txt":
            la = [x for x in open(pa).read().splitlines() if not x.startswith(("execution_backend=", "device_field"))]
            lb = [x for x in open(pb).read().splitlines() if not x.startswith(("execution_backend=", "device_field"))]
            assert la == lb
        else:
            assert read(pa) == read(pb), n
    return names


@pytest.mark.parametrize("extra", [[], ["--eta-colours", "5"], ["--grain-evolution", "off"]],
                         ids=["eta-per-grain", "coloured", "static-grains"])
def test_program_slabs_match_single_gpu(require_gpu, tmp_path, extra):
    one = run(tmp_path, "one", extra)
    for k in (2, 3):
        many = run(tmp_path, f"slabs{k}", extra + ["--slabs", str(k), "--slab-devices", ",".join(["0"] * k)])
        names = compare_outputs(one, many)
        assert "fields_30.vti" in names and "diagnostics.csv" in names


def test_program_slabs_failure(require_gpu, tmp_path):
    extra = ["--bounds", "stop", "--grain-evolution", "off"]
    one = str(tmp_path / "one")
    many = str(tmp_path / "many")
    r1 = nicr.main(3, BASE + extra + ["--out", one])
    r2 = nicr.main(3, BASE + extra + ["--slabs", "2", "--slab-devices", "0,0", "--out", many])
    assert r1 == r2
    if r1 != 0:
        assert read(os.path.join(one, "STOPPED.txt")) == read(os.path.join(many, "STOPPED.txt"))
        assert read(os.path.join(one, "state_at_failure.vti")) == read(os.path.join(many, "state_at_failure.vti"))
    compare_outputs(one, many)


def test_program_slabs_rejects_unsupported(require_gpu, tmp_path):
    assert nicr.main(3, BASE + ["--slabs", "2", "--output-format", "vtk", "--out", str(tmp_path / "a")]) == 1
    assert nicr.main(3, BASE + ["--slabs", "2", "--checkpoint-every", "10", "--out", str(tmp_path / "b")]) == 1
    assert nicr.main(3, BASE + ["--slabs", "9", "--out", str(tmp_path / "c")]) == 1   # 4 planes < halo 9
