"""The CUDA path against the golden fixtures made from the unmodified
reference: the regression matrix (bit-identical fields), the reference's stored
2D example and the verify_mpi.py cases through the nicr2d program (VTK files
byte-identical; diagnostics within the reference's own cross-layout tolerance
1e-10*(1+|x|), mpi2d/tests/verify_mpi.py:39)."""
import csv
import hashlib
import io
import json
from pathlib import Path

import numpy as np
import pytest

import nicr
from golden_cases import regression_inputs
from parity import ld

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def file_sha(p):
    return hashlib.sha256(Path(p).read_bytes()).hexdigest()


@pytest.mark.parametrize("dim", [2, 3])
def test_regression_fixtures_bit_identical(require_gpu, dim):
    cases = json.loads((GOLD / f"regression_{dim}d.json").read_text())
    for case in cases:
        cfg = nicr.make_config(dim, **case["config"])
        sol = nicr.Solver(cfg)
        inj = regression_inputs(cfg)
        sol.set_fields(inj["o"], inj["cr"], inj["p"], inj["eta"] or None)
        sol.stamp(12, 1, 1 if dim == 3 else 0)
        for n in range(24):
            if n in (3, 14):
                sol.nucleate()
            if n == 10 and sol.n_eta:
                e = sol.get("eta", 0)
                idx = (11, 6, 5) if dim == 3 else (11, 6)
                e[idx] *= 0.95
                sol.set("eta", e, 0)
            sol.step(1)
        for name, want in case["fields"].items():
            assert sha(sol.get(name)) == want, (case["name"], name)
        b = sol.budget()
        for n, (hi, lo) in case["budget"].items():
            assert abs(ld(b[n]) - (hi + lo)) <= 1e-13 * (1 + abs(hi)), (case["name"], n)
        assert (b["nuclei"], b["clipped"]) == (case["nuclei"], case["clipped"]), case["name"]
        sol.close()


def rows(text):
    return list(csv.reader(io.StringIO(text)))


def assert_csv_close(got_text, want_text, header=True):
    got, want = rows(got_text), rows(want_text)
    if header:
        assert got[0] == want[0]
        got, want = got[1:], want[1:]
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            x, y = float(x), float(y)
            assert abs(x - y) <= 1e-10 * (1 + abs(y)), (x, y)


def test_example_center_through_nicr2d(require_gpu, tmp_path):
    """The reference's stored example (mpi2d/example_center): VTK frames and the
    grain map byte-identical, CSV rows within tolerance."""
    d = json.loads((GOLD / "example_center_2d.json").read_text())
    out = tmp_path / "ex"
    assert nicr.main(2, d["args"] + ["--out", str(out)]) == 0
    for f in ("fields_0.vtk", "fields_500.vtk", "grains.csv"):
        assert file_sha(out / f) == d["sha256"][f], f
    for f in ("diagnostics.csv", "grain_diagnostics.csv", "grain_history.csv"):
        assert_csv_close((out / f).read_text(), d["text"][f])


@pytest.mark.parametrize("case", ["mu", "anchored", "center", "O_off", "legacy_Ck"])
def test_verify_mpi_cases_through_nicr2d(require_gpu, tmp_path, case):
    d = json.loads((GOLD / "verify_mpi_2d.json").read_text())[case]
    out = tmp_path / case
    assert nicr.main(2, d["args"] + ["--out", str(out)]) == 0
    for f, want in d["vtk_sha256"].items():
        assert file_sha(out / f) == want, f
    got = rows((out / "diagnostics.csv").read_text())[1:]
    want = rows(d["diagnostics"])
    assert len(got) == len(want)
    for a, b in zip(got, want):
        for x, y in zip(a, b):
            assert abs(float(x) - float(y)) <= 1e-10 * (1 + abs(float(y))), (case, x, y)
    got = rows((out / "grain_diagnostics.csv").read_text())[1:]
    want = rows(d["grain_diagnostics"])
    for a, b in zip(got, want):
        for x, y in zip(a, b):
            assert abs(float(x) - float(y)) <= 1e-10 * (1 + abs(float(y))), (case, x, y)


def decode_vti(path):
    """Appended raw zlib VTI (the layout mpi3d-slab/tests/verify.py decodes)."""
    import re
    import struct
    import zlib
    content = Path(path).read_bytes()
    prefix, data = content.split(b'<AppendedData encoding="raw">\n_', 1)
    arrays = {}
    for m in re.finditer(rb'<DataArray type="(\w+)" Name="(\w+)" NumberOfComponents="1" format="appended" offset="(\d+)"',
                         prefix):
        kind, name, offset = m.group(1).decode(), m.group(2).decode(), int(m.group(3))
        n, bs, last = struct.unpack_from("<QQQ", data, offset)
        sizes = struct.unpack_from("<" + "Q" * n, data, offset + 24)
        cur = offset + 24 + 8 * n
        raw = b""
        for sz in sizes:
            raw += zlib.decompress(data[cur:cur + sz])
            cur += sz
        arrays[name] = np.frombuffer(raw, dtype="<f4" if kind == "Float32" else "<f8")
    return arrays


@pytest.mark.parametrize("case", ["static_mu", "eta_concentration"])
def test_nicr3d_program_vtk_and_vti(require_gpu, tmp_path, case):
    d = json.loads((GOLD / "cli_3d.json").read_text())[case]
    out = tmp_path / "vtk"
    assert nicr.main(3, d["args"] + ["--output-format", "vtk", "--out", str(out)]) == 0
    for f, want in d["vtk_sha256"].items():
        assert file_sha(out / f) == want, f
    got = rows((out / "diagnostics.csv").read_text())[1:]
    for a, b in zip(got, rows(d["diagnostics"])):
        for x, y in zip(a, b):
            assert abs(float(x) - float(y)) <= 1e-10 * (1 + abs(float(y))), (x, y)
    # VTI, Float32 and Float64: payload == cast of the reference's ASCII values (verify.py:96-101)
    steps = d["args"][d["args"].index("--steps") + 1]
    for prec in ("float32", "float64"):
        o2 = tmp_path / prec
        assert nicr.main(3, d["args"] + ["--output-precision", prec, "--out", str(o2)]) == 0
        arrays = decode_vti(o2 / f"fields_{steps}.vti")
        assert list(arrays) == ["phi", "conc_O", "conc_Cr", "mu_O", "mu_Cr", "grain_sum", "GB_mask"]
        for name, a in arrays.items():
            assert hashlib.sha256(a.tobytes()).hexdigest() == d["vti_payload_sha256"][prec][name], (prec, name)


@pytest.mark.parametrize("dim", [2, 3])
def test_self_test_program(require_gpu, dim):
    assert nicr.main(dim, ["--self-test"]) == 0


def test_bounds_stop_writes_stopped_file(require_gpu, tmp_path):
    """With the default bounds=stop these inputs are rejected in the first
    steps (O undershoots at the inlet); run() writes STOPPED.txt and the state
    at failure, and exits 1 (3S:1386-1390)."""
    out = tmp_path / "stop"
    rc = nicr.main(3, ["--nx", "24", "--ny", "16", "--nz", "14", "--steps", "50", "--output-every", "25",
                       "--bc", "concentration", "--out", str(out)])
    if rc == 0:
        pytest.skip("no rejection for these inputs")
    assert rc == 1
    text = (out / "STOPPED.txt").read_text()
    assert text.startswith("Last accepted time step:")
    assert (out / "state_at_failure.vti").exists()
