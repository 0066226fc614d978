#!/usr/bin/env python3
"""Generates the golden fixtures in this directory from the unmodified reference.

Run in a checkout where the reference sources are present and oracle/_ref is
built (`make -C oracle`). It writes:

* regression_3d.json / regression_2d.json: the shape of the reference's own
  regression matrix (mpi3d-slab/tests/verify.py:54-114, regression_driver.cpp):
  {single crystal, static Voronoi, evolving eta, frozen eta} x {closed, mu,
  concentration} x O on/off x Ck legacy/off on 25x15(x13), seeded inputs with
  phi = 0, a stamp across both periodic seams, Ksp scans before steps 3 and 14,
  an eta edit before step 10, 24 steps. Per case: SHA-256 of every field after
  the last step and the budget.
* example_center_2d.json: the reference's stored example
  (mpi2d/example_center): command line, SHA-256 of the VTK/CSV files and the
  diagnostics rows.
* cli_3d.json: two 3D program runs (VTK frames every 20 steps, diagnostics, and
  hashes of the last frame's arrays cast to Float32/Float64 for the VTI payload).
* verify_mpi_2d.json: the five cases of mpi2d/tests/verify_mpi.py:57-75 with the
  SHA-256 of every VTK frame (output every 250 steps) and the diagnostics rows.
* long_runs.json: the specification's workloads run on the reference's run()
  schedule (golden_cases.LONG_CASES): 128^3 with 32 static grains for 2000
  steps (plain and supersaturated), and 256^3 with 8 evolving eta for one
  nucleation period. Per case: SHA-256 of every field, the budget, nuclei and
  clipped cells. The thread-per-rank reference build (oracle/_ref/*_threads)
  runs them on all host cores; its fields equal the single-process build's.

Usage: make_golden.py --ref <reference source dir> [--only NAME ...]
(the reference sources are needed for the stored example; oracle/_ref must
be built with `make -C oracle REF=<dir>`).

Inputs are drawn from numpy's PCG64 (bit-reproducible), so tests regenerate
them instead of storing them.
"""
import hashlib
import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))
from oracle import make_config, run_reference, REF_DIR  # noqa: E402
from golden_cases import (MODES, LONG_CASES, long_inputs, regression_cases, regression_inputs,  # noqa: E402
                          regression_commands)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def regression(dim: int):
    out = []
    for case in regression_cases(dim):
        cfg = make_config(dim, **case["config"])
        inj = regression_inputs(cfg)
        res = run_reference(cfg, regression_commands(dim, ref_driver=True) + ["dump"], inject=inj)
        d = res["dumps"][-1]
        fields = {k: sha(d[k]) for k in ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb") if len(d[k])}
        for g in range(int(d["n_eta"][0])):
            fields[f"eta{g + 1}"] = sha(d[f"eta{g + 1}"])
        if len(d["eta_s2"]) and int(d["n_eta"][0]):
            fields["eta_s2"] = sha(d["eta_s2"])
        names = ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")
        out.append({"name": case["name"], "config": case["config"], "fields": fields,
                    "budget": {n: [float(x) for x in d["budget"][q]] for q, n in enumerate(names)},
                    "nuclei": int(d["counts"][0]), "clipped": int(d["counts"][1]),
                    "stdout": res["stdout"].strip().splitlines()})
    return out


def file_sha(p: Path) -> str:
    return hashlib.sha256(p.read_bytes()).hexdigest()


def example_center(reference: Path):
    src = reference / "mpi2d" / "example_center"
    args = ["--nx", "61", "--ny", "61", "--grain-evolution", "on", "--eta-output", "all", "--seed", "2001",
            "--left-edge-sites", "2", "--nucleation", "center", "--radius-grid", "5.5", "--bc", "closed",
            "--ck", "off", "--bounds", "legacy", "--dt", "1e-12", "--steps", "500", "--output-every", "500"]
    files = {p.name: file_sha(p) for p in sorted(src.iterdir()) if p.name != "parameters.txt"}
    text = {n: (src / n).read_text() for n in ("diagnostics.csv", "grain_diagnostics.csv", "grain_history.csv", "grains.csv")}
    return {"args": args, "sha256": files, "text": text,
            "source": "mpi2d/example_center (stored with the reference; reproduced byte-for-byte by oracle/_ref/ref2d)"}


def verify_mpi_2d():
    common = ["--nx", "61", "--ny", "31", "--grain-diameter-grid", "30", "--seed", "2001", "--grain-evolution", "on",
              "--eta-output", "all", "--bounds", "legacy", "--dt", "1e-12", "--output-every", "250"]
    cases = {
        "mu": ["--bc", "mu", "--ck", "off", "--steps", "1000"],
        "anchored": ["--bc", "mu", "--ck", "off", "--left-edge-sites", "2", "--steps", "1000"],
        "center": ["--bc", "closed", "--ck", "off", "--nucleation", "center", "--steps", "500"],
        "O_off": ["--bc", "closed", "--ck", "off", "--nucleation", "center", "--oxygen-diffusion", "off", "--steps", "500"],
        "legacy_Ck": ["--bc", "closed", "--ck", "legacy", "--nucleation", "center", "--steps", "500"],
    }
    out = {}
    for name, extra in cases.items():
        args = common + extra
        steps = int(extra[extra.index("--steps") + 1])
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            cmds = ["vtk", str(td / "fields_0.vtk"), "log", str(td / "diag.csv"), "0"]
            for n in range(250, steps + 1, 250):
                cmds += ["run", "250", "vtk", str(td / f"fields_{n}.vtk"), "log", str(td / "diag.csv"), str(n)]
            r = subprocess.run([str(REF_DIR / "ref2d")] + args + ["--"] + cmds, capture_output=True, text=True,
                               timeout=600, cwd=td)
            if r.returncode:
                raise RuntimeError(r.stderr)
            frames = {p.name: file_sha(p) for p in sorted(td.glob("fields_*.vtk"))}
            out[name] = {"args": args, "vtk_sha256": frames, "diagnostics": (td / "diag.csv").read_text(),
                         "grain_diagnostics": (td / "diag.csv.grain").read_text(),
                         "grain_history": (td / "diag.csv.history").read_text()}
    return out


def vti_hashes(vtk_text):
    """SHA-256 of each array of a legacy VTK frame cast to Float32 and Float64:
    the payload a VTI of the same state must decode to (verify.py:96-101)."""
    import re
    out = {"float32": {}, "float64": {}}
    for name, payload in re.findall(r"SCALARS (\S+) double 1\nLOOKUP_TABLE default\n(.*?)(?=SCALARS|\Z)", vtk_text, re.S):
        vals = np.array([float(v) for v in payload.split()])
        out["float32"][name] = hashlib.sha256(vals.astype("<f4").tobytes()).hexdigest()
        out["float64"][name] = hashlib.sha256(vals.astype("<f8").tobytes()).hexdigest()
    return out


def cli_3d():
    """3D program runs: VTK frames every 20 steps (static grains with the mu
    inlet and Ksp; evolving eta with the concentration inlet)."""
    cases = {
        "static_mu": ["--nx", "25", "--ny", "15", "--nz", "13", "--grain-diameter-grid", "12", "--bc", "mu",
                      "--ck", "legacy", "--bounds", "legacy", "--dt", "1e-12", "--nucleation", "ksp",
                      "--nucleation-period", "5e-12", "--steps", "40", "--output-every", "20"],
        "eta_concentration": ["--nx", "21", "--ny", "13", "--nz", "11", "--grain-diameter-grid", "8",
                              "--grain-evolution", "on", "--bc", "concentration", "--ck", "legacy",
                              "--bounds", "legacy", "--dt", "1e-12", "--nucleation", "center", "--radius-grid", "3",
                              "--steps", "40", "--output-every", "20"],
    }
    out = {}
    for name, args in cases.items():
        steps = int(args[args.index("--steps") + 1])
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            cmds = ["vtk", str(td / "fields_0.vtk"), "log", str(td / "diag.csv"), "0"]
            for n in range(20, steps + 1, 20):
                cmds += ["run", "20", "vtk", str(td / f"fields_{n}.vtk"), "log", str(td / "diag.csv"), str(n)]
            r = subprocess.run([str(REF_DIR / "ref3d")] + args + ["--"] + cmds, capture_output=True, text=True,
                               timeout=600, cwd=td)
            if r.returncode:
                raise RuntimeError(r.stderr)
            out[name] = {"args": args, "vtk_sha256": {p.name: file_sha(p) for p in sorted(td.glob("fields_*.vtk"))},
                         "diagnostics": (td / "diag.csv").read_text(),
                         "grain_diagnostics": (td / "diag.csv.grain").read_text() if (td / "diag.csv.grain").exists() else "",
                         "vti_payload_sha256": vti_hashes((td / f"fields_{steps}.vtk").read_text())}
    return out


def long_runs(names, threads):
    import os
    path = HERE / "long_runs.json"
    out = json.loads(path.read_text()) if path.exists() else {}
    for name in names:
        case = LONG_CASES[name]
        cfg = make_config(3, **case["config"])
        d0 = run_reference(cfg, ["dump"], threads=threads, timeout=3600)["dumps"][0]
        shape = (cfg.nx, cfg.ny, cfg.nz)
        o, cr, p = long_inputs(case, d0["o"].reshape(shape), d0["cr"].reshape(shape), d0["p"].reshape(shape))
        n_eta = int(d0["n_eta"][0])
        inj = {"o": o, "cr": cr, "p": p, "eta": [d0[f"eta{g + 1}"].reshape(shape) for g in range(n_eta)]}
        cmds = ["reset_inventory"]
        if case["stamp"]:
            cmds.append(["stamp"] + list(case["stamp"]))
        cmds += [["time_run", case["steps"]], "dump"]
        res = run_reference(cfg, cmds, inject=inj, threads=threads, timeout=4 * 3600)
        if "REJECTED" in res["stdout"]:
            raise RuntimeError(f"{name}: the reference rejected a step: {res['stdout']}")
        d = res["dumps"][-1]
        fields = {k: sha(d[k]) for k in ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb")}
        for g in range(n_eta):
            fields[f"eta{g + 1}"] = sha(d[f"eta{g + 1}"])
        if n_eta:
            fields["eta_s2"] = sha(d["eta_s2"])
        names_b = ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")
        out[name] = {"config": case["config"], "steps": case["steps"], "fields": fields,
                     "budget": {n: [float(x) for x in d["budget"][q]] for q, n in enumerate(names_b)},
                     "nuclei": int(d["counts"][0]), "clipped": int(d["counts"][1]),
                     "reference_ranks": threads or 1, "stdout": res["stdout"].strip().splitlines()}
        path.write_text(json.dumps(out, indent=1) + "\n")
        print(name, "nuclei", out[name]["nuclei"], "clipped", out[name]["clipped"], res["stdout"].strip())


def main():
    import argparse
    import os
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", type=Path, required=True, help="directory holding the reference sources")
    ap.add_argument("--only", nargs="*", help="fixture groups: regression example verify cli or a LONG_CASES name")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1, help="reference ranks for the long runs")
    a = ap.parse_args()
    if not (REF_DIR / "ref3d").exists():
        raise SystemExit("oracle/_ref is not built (make -C oracle REF=<dir>)")
    want = set(a.only or ["regression", "example", "verify", "cli"] + list(LONG_CASES))
    if "regression" in want:
        (HERE / "regression_3d.json").write_text(json.dumps(regression(3), indent=1) + "\n")
        (HERE / "regression_2d.json").write_text(json.dumps(regression(2), indent=1) + "\n")
    if "example" in want:
        (HERE / "example_center_2d.json").write_text(json.dumps(example_center(a.ref), indent=1) + "\n")
    if "verify" in want:
        (HERE / "verify_mpi_2d.json").write_text(json.dumps(verify_mpi_2d(), indent=1) + "\n")
    if "cli" in want:
        (HERE / "cli_3d.json").write_text(json.dumps(cli_3d(), indent=1) + "\n")
    long_names = [n for n in LONG_CASES if n in want]
    if long_names:
        long_runs(long_names, a.threads if a.threads > 1 else 0)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
