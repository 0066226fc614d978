"""The oracle against the committed golden fixtures (generated from the
unmodified reference by tests/golden/make_golden.py): every field hash and the
budget of the reference's regression-matrix shape, 2D and 3D. Runs anywhere;
the reference itself is not needed at test time."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import Oracle, make_config
from golden_cases import regression_inputs

GOLD = Path(__file__).resolve().parent / "golden"


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def replay_oracle(cfg):
    orc = Oracle(cfg)
    inj = regression_inputs(cfg)
    orc.set_fields(inj["o"], inj["cr"], inj["p"], np.array(inj["eta"]) if inj["eta"] else None)
    stamp = (12, 1, 1) if cfg.dim == 3 else (12, 1, 0)
    orc.stamp(*stamp)
    for n in range(24):
        if n in (3, 14):
            orc.nucleate()
        if n == 10 and orc.neta:
            orc.scale_eta(0, 12, 7, 6 if cfg.dim == 3 else 0, 0.95)
        assert orc.step() == 0, orc.error()
    orc.refresh()
    return orc


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_reproduces_reference_regression_fixtures(dim):
    cases = json.loads((GOLD / f"regression_{dim}d.json").read_text())
    assert len(cases) == 48
    for case in cases:
        cfg = make_config(dim, **case["config"])
        orc = replay_oracle(cfg)
        for name, want in case["fields"].items():
            assert sha(orc.get(name)) == want, (case["name"], name)
        b = orc.budget()
        for n, (hi, lo) in case["budget"].items():
            assert b[n][0] + b[n][1] == hi + lo, (case["name"], n)
        assert (b["nuclei"], b["clipped"]) == (case["nuclei"], case["clipped"]), case["name"]


def test_example_center_fixture_is_the_stored_reference_example():
    d = json.loads((GOLD / "example_center_2d.json").read_text())
    assert "fields_500.vtk" in d["sha256"] and "diagnostics.csv" in d["text"]
