"""Parameter sweeps over many independent domains (the batched form).

A sweep is a list of domain configurations; on one GPU they run as one
nicr_batch, on N GPUs (one process per GPU) each rank runs the batch of its
share of the domains and only the per-domain results are gathered at the end.
Domains are independent, so the data path has no collective.
"""
from __future__ import annotations

import math

import numpy as np

from ._abi import NicrConfig, make_config

LAYER_O = 0.0023      # Physics::layerO (3S:77)
KSP = 1.28e-7         # Physics::ksp (3S:76)


def diameter_for_grains(n_grains: int, shape) -> float:
    """Grain diameter (grid units) whose seed count round(6V/(pi d^3)) is
    n_grains (3S:416-418: n = max(1, round(V / (pi d^3 / 6))))."""
    v = float(np.prod(shape))
    return (6.0 * v / (math.pi * n_grains)) ** (1.0 / 3.0)


def sweep_configs(n_domains: int = 64, seed: int = 3, edges=(32, 48, 64, 80, 96), precision: int = 0,
                  **common) -> list[NicrConfig]:
    """Seeded sweep of uneven 3D domains: each edge drawn from `edges`, Cr in
    U[0.15, 0.30], O supply U[0.5, 1.0] x layerO, Ksp log-uniform in
    [Ksp/10, 10 Ksp], 8..32 static Voronoi grains, Ksp nucleation, legacy
    bounds. `common` overrides any config field for every domain."""
    rng = np.random.default_rng(seed)
    cfgs = []
    for i in range(n_domains):
        nx, ny, nz = (int(e) for e in rng.choice(edges, size=3))
        cr = float(rng.uniform(0.15, 0.30))
        supply = float(rng.uniform(0.5, 1.0))
        ksp = float(KSP * 10.0 ** rng.uniform(-1.0, 1.0))
        grains = int(rng.integers(8, 33))
        kw = dict(nx=nx, ny=ny, nz=nz, grains=1, grain_evolution=0, random_seed=seed * 1000 + i,
                  grain_diameter_grid=diameter_for_grains(grains, (nx, ny, nz)), bulk_cr=cr,
                  layer_o=supply * LAYER_O, ksp=ksp, bc="concentration", ck="legacy", bounds="legacy",
                  nucleation="ksp", precision=precision)
        kw.update(common)
        cfgs.append(make_config(3, **kw))
    return cfgs


def cells(cfg: NicrConfig) -> int:
    return cfg.nx * cfg.ny * (cfg.nz if cfg.dim == 3 else 1)


def partition_domains(sizes, world: int) -> list[list[int]]:
    """Greedy longest-processing-time bin packing of domains (by cell count)
    onto `world` ranks: largest domain first, each to the least-loaded rank
    (lowest rank on ties). Deterministic, so every rank computes the same
    plan without communication. Returns the sorted domain indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def gather_results(local: dict, n_domains: int, world: int) -> list:
    """All-gather of per-domain results {domain index: result} from every rank
    into one list ordered by domain index (torch.distributed, any backend).
    The only collective of a sharded sweep, after the last step."""
    if world == 1:
        return [local.get(i) for i in range(n_domains)]
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, local)
    out = [None] * n_domains
    for p in parts:
        for i, v in p.items():
            if out[i] is not None:
                raise RuntimeError(f"domain {i} reported by two ranks")
            out[i] = v
    return out


def run_sweep(cfgs, steps: int, rank: int = 0, world: int = 1, schedule: bool = True):
    """Runs this rank's share of the sweep as one batch and gathers per-domain
    summaries (accepted steps, budget residuals, diagnostics) on every rank."""
    from . import Batch
    part = partition_domains([cells(c) for c in cfgs], world)[rank]
    local = {}
    if part:
        with Batch([cfgs[i] for i in part]) as b:
            done, rc = (b.run if schedule else b.step)(steps, check=False)
            for k, i in enumerate(part):
                d = b.domains[k]
                local[i] = {"completed": done[k], "status": rc if done[k] < steps else 0,
                            "budget": d.budget(), "diagnostics": d.diagnostics()}
    return gather_results(local, len(cfgs), world)
