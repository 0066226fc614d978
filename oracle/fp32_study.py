#!/usr/bin/env python3
"""Measurement, not product: what an FP32 state would do to the solution.

Runs the oracle (the C restatement of the reference step, FP64) on a C3-shaped
grid three ways from the same initial state and compares the final fields:

* fp64: the plain FP64 step (the reference's arithmetic);
* fp32: after every step o, cr, phi and every eta are rounded to FP32, i.e.
  the state is stored in FP32 while the step itself computes in FP64 (an FP32
  state can do no better than this);
* fp32-reproject: as fp32, and after the rounding the O and Cr lost by it
  (the FP64 sum of the unrounded values minus the FP64 sum of the rounded
  ones) is put back in proportion to each cell's own step increment, then
  rounded again: a per-step re-projection of total O and Cr onto the FP64
  budget.

Grid: n^3, 8 Voronoi seeds of seed 2 with one evolving eta each (the
reference's own form of the 8-field work), Cr 0.25 +- 0.01 (PCG64 seed 2, the
inlet plane keeps its value), O supplied at x = 0, Ksp scans on the run()
schedule, legacy Ck and bounds, default dt. Per field: relative L-inf
(max |a - b| / max |b|) and L2 against fp64, and the oxide-front position
(leading X planes with phi >= 0.5 per column) difference in cells.

Usage: fp32_study.py --size 64 --steps 5000  (the three runs go in parallel)
"""
import argparse
import json
import math
import multiprocessing as mp
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))


def config(n):
    from oracle import make_config
    d = (6.0 * n ** 3 / (math.pi * 8)) ** (1.0 / 3.0)
    return make_config(3, nx=n, ny=n, nz=n, grains=1, grain_evolution=1, random_seed=2, bc="concentration",
                       ck="legacy", bounds="legacy", nucleation="ksp", grain_diameter_grid=d)


def f32(a):
    return a.astype(np.float32).astype(np.float64)


def run(args):
    mode, n, steps, out = args
    from oracle import Oracle
    cfg = config(n)
    orc = Oracle(cfg)
    shape = orc.shape
    cr = orc.get("cr")
    noise = 0.25 + np.random.default_rng(2).uniform(-0.01, 0.01, size=shape)
    noise[0] = cr[0]
    eta = np.array([orc.get(f"eta{g + 1}") for g in range(orc.neta)])
    o, p = orc.get("o"), orc.get("p")
    if mode != "fp64":
        o, noise, p, eta = f32(o), f32(noise), f32(p), f32(eta)
    orc.set_fields(o, noise, p, eta)
    orc.reset_inventory()
    period, dt, nxt = cfg.nucleation_period, cfg.dt, cfg.nucleation_period
    for s in range(1, steps + 1):
        if s * dt + 1e-12 * period >= nxt:
            orc.nucleate()
            nxt += period
        if mode != "fp64":
            before = {"o": orc.get("o"), "cr": orc.get("cr")}
        rc = orc.step()
        if rc:
            raise SystemExit(f"{mode}: step {s} rejected: {orc.error()}")
        if mode == "fp64":
            continue
        fields = {"o": orc.get("o"), "cr": orc.get("cr"), "p": orc.get("p")}
        eta = np.array([orc.get(f"eta{g + 1}") for g in range(orc.neta)])
        rounded = {k: f32(v) for k, v in fields.items()}
        if mode == "fp32-reproject":
            for k in ("o", "cr"):
                lost = math.fsum(fields[k].ravel()) - math.fsum(rounded[k].ravel())
                w = np.abs(fields[k] - before[k])
                tot = math.fsum(w.ravel())
                if tot > 0.0:
                    rounded[k] = f32(rounded[k] + lost * w / tot)
        orc.set_fields(rounded["o"], rounded["cr"], rounded["p"], f32(eta))
    res = {f: orc.get(f) for f in ("o", "cr", "p")}
    for g in range(orc.neta):
        res[f"eta{g + 1}"] = orc.get(f"eta{g + 1}")
    np.savez(out, **res)


def front(ph):
    ox = ph >= 0.5
    return np.where(ox.all(axis=0), ph.shape[0], np.argmin(ox, axis=0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--out", default="/tmp/fp32_study")
    a = ap.parse_args()
    Path(a.out).mkdir(parents=True, exist_ok=True)
    modes = ["fp64", "fp32", "fp32-reproject"]
    jobs = [(m, a.size, a.steps, f"{a.out}/{m}_{a.size}.npz") for m in modes]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        pool.map(run, jobs)
    ref = dict(np.load(jobs[0][3]))
    shape = (a.size,) * 3
    summary = {"size": a.size, "steps": a.steps, "fields": {}}
    for m, _, _, path in jobs[1:]:
        got = dict(np.load(path))
        per = {}
        for f, b in ref.items():
            x = got[f]
            per[f] = {"linf_rel": float(np.max(np.abs(x - b)) / max(np.max(np.abs(b)), 1e-300)),
                      "l2_rel": float(np.sqrt(np.mean((x - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))}
        per["oxide_front_max_cells"] = int(np.max(np.abs(front(got["p"].reshape(shape)) - front(ref["p"].reshape(shape)))))
        per["total_O_rel"] = float(abs(got["o"].sum() - ref["o"].sum()) / ref["o"].sum())
        per["total_Cr_rel"] = float(abs(got["cr"].sum() - ref["cr"].sum()) / ref["cr"].sum())
        summary["fields"][m] = per
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
