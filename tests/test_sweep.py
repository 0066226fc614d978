"""Host logic of sharded sweeps (no GPU): the seeded sweep generator, the
deterministic domain partition, and the end-of-run gather across ranks
(world_size 2 over gloo on CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from nicr.sweep import cells, diameter_for_grains, gather_results, partition_domains, sweep_configs


def test_sweep_configs_are_seeded_and_in_range():
    a, b = sweep_configs(64, seed=3), sweep_configs(64, seed=3)
    assert [(c.nx, c.ny, c.nz, c.bulk_cr, c.ksp) for c in a] == [(c.nx, c.ny, c.nz, c.bulk_cr, c.ksp) for c in b]
    assert len({(c.nx, c.ny, c.nz) for c in a}) > 20
    for c in a:
        assert {c.nx, c.ny, c.nz} <= {32, 48, 64, 80, 96}
        assert 0.15 <= c.bulk_cr <= 0.30
        assert 0.5 * 0.0023 <= c.layer_o <= 0.0023
        assert 1.28e-8 <= c.ksp <= 1.28e-6
        assert c.grains == 1 and c.grain_evolution == 0
        import math
        v = c.nx * c.ny * c.nz
        n = round(v / (math.pi * c.grain_diameter_grid ** 3 / 6.0))
        assert 8 <= n <= 32
    assert diameter_for_grains(32, (128, 128, 128)) == pytest.approx(50.0, rel=0.02)


def test_partition_covers_every_domain_once_and_balances():
    sizes = [cells(c) for c in sweep_configs(64, seed=3)]
    for world in (1, 2, 3, 8):
        parts = partition_domains(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(sizes) / world + max(sizes)
    assert partition_domains([5, 5, 5], 2) == [[0, 2], [1]]
    assert partition_domains([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        partition_domains([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [cells(c) for c in sweep_configs(10, seed=4)]
        mine = partition_domains(sizes, world)[rank]
        local = {i: {"rank": rank, "cells": sizes[i]} for i in mine}
        out = gather_results(local, len(sizes), world)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_gather_results_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sizes = [cells(c) for c in sweep_configs(10, seed=4)]
    parts = partition_domains(sizes, world)
    for r in range(world):
        out = res[r]
        assert len(out) == 10
        for i, v in enumerate(out):
            assert v["cells"] == sizes[i]
            assert i in parts[v["rank"]]
    assert res[0] == res[1]


def test_gather_results_single_rank():
    assert gather_results({1: "b", 0: "a"}, 3, 1) == ["a", "b", None]
