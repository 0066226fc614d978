"""The correctly rounded division by a run constant (xdiv in
csrc/nicr_physics.h: double-word reciprocal, one Markstein correction step,
IEEE division outside the guarded range), restated on the host in
tests/division_check.c and checked against IEEE division on ~24 M numerators
over 73 divisors: random numerators over and beyond the guarded exponent
range, quotients within ~2^-104 relative of a rounding midpoint, signed zeros,
subnormals, infinities and NaN. CPU only; the device's own self-check of the
same cases is tests/test_gpu_parity.py::test_verified_division_matches_ieee."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_division_restatement_matches_ieee(tmp_path):
    exe = tmp_path / "division_check"
    subprocess.run(["gcc", "-O2", "-std=gnu11", "-o", str(exe), str(HERE / "division_check.c"), "-lm"],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe), "300000", "11"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    checked, mism, fallbacks, hard = (int(w) for w in r.stdout.split()[1::2])
    assert mism == 0 and checked > 20_000_000 and hard > 500_000, r.stdout
