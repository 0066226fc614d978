"""The slab form with one process per GPU (nicr_slab_* and nicr.slab_ranks):
the per-rank protocol (launch, MIN agreement, commit, halo exchange, Ksp scan
chain) run here with every rank in one process on one GPU (LocalComm: the
exchange and the agreement as device copies ordered by events). Across
processes the same protocol runs over torch.distributed (TorchComm); its host
side is tested with gloo on CPU in test_slab_ranks.py. The ranks must evolve
exactly as one handle on the same configuration."""
import numpy as np
import pytest

import nicr
from nicr.slab_ranks import LocalComm, SlabRank, advance, colour_grains, gather_budget, gather_field, scan
from parity import assert_bitexact, assert_budget, smooth_fields

pytestmark = pytest.mark.gpu


def cfg_for(**kw):
    base = dict(nx=40, ny=24, nz=32, grains=1, grain_evolution=1, grain_diameter_grid=11., random_seed=3,
                bc="concentration", ck="legacy", bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5,
                nucleation_period=5e-12)
    base.update(kw)
    return nicr.make_config(3, **base)


def make(cfg, world):
    ranks = [SlabRank(cfg, world, i) for i in range(world)]
    comm = LocalComm(ranks)
    if cfg.eta_colours:
        colour_grains(comm)
    return ranks, comm


def inject(ranks, solo, seed):
    o, cr, p, eta = smooth_fields(solo.shape, solo.n_eta, seed=seed)
    for name, arr in (("o", o), ("cr", cr), ("p", p)):
        solo.set(name, arr)
        for r in ranks:
            r.set_domain(name, arr)
    for g, e in enumerate(eta):
        solo.set("eta", e, g)
        for r in ranks:
            r.set_domain("eta", e, g)
    solo.reset_inventory()
    for r in ranks:
        r.reset_inventory()


def assert_same(comm, solo, label):
    for f in ("o", "cr", "p", "gb"):
        assert_bitexact(f"{label} {f}", gather_field(comm, f), solo.get(f))
    for g in range(solo.n_eta):
        assert_bitexact(f"{label} eta{g + 1}", gather_field(comm, "eta", g), solo.get("eta", g))
    assert_budget(gather_budget(comm), solo.budget())


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("mode", ["run", "step"])
def test_ranks_match_single_handle(require_gpu, world, mode):
    cfg = cfg_for()
    solo = nicr.Solver(cfg)
    ranks, comm = make(cfg, world)
    inject(ranks, solo, 5)
    for chunk in (7, 1, 12):
        rc, done, msg = advance(comm, chunk, schedule=(mode == "run"))
        getattr(solo, mode)(chunk)
        assert rc == 0 and done == chunk and msg == ""
    assert_same(comm, solo, f"{world} ranks")
    if mode == "run":
        assert gather_budget(comm)["nuclei"] > 3
        assert scan(comm) == solo.nucleate()
        assert_same(comm, solo, "after a scan")
    for r in ranks:
        r.close()
    solo.close()


def test_ranks_coloured_init(require_gpu):
    cfg = cfg_for(eta_colours=6)
    solo = nicr.Solver(cfg)
    ranks, comm = make(cfg, 3)
    for g in range(6):
        assert_bitexact(f"eta{g + 1} initial", gather_field(comm, "eta", g), solo.get("eta", g))
    advance(comm, 9)
    solo.run(9)
    assert_same(comm, solo, "coloured")
    for r in ranks:
        r.close()
    solo.close()


def test_ranks_rejected_trial(require_gpu):
    cfg = cfg_for(bounds="stop", grain_evolution=0)
    solo = nicr.Solver(cfg)
    ranks, comm = make(cfg, 3)
    inject(ranks, solo, 4)
    advance(comm, 6)
    solo.run(6)
    cr = solo.get("cr")
    cr[14, 5, 4] = -0.1
    solo.set("cr", cr)
    for r in ranks:
        r.set_domain("cr", cr)
    before = gather_field(comm, "o")
    rc, done, msg = advance(comm, 8)
    rc1, done1 = solo.run(8, check=False)
    assert rc == rc1 == nicr._abi.ERR_TRIAL_BOUNDS and done == done1 == 0
    assert msg == solo.last_error
    assert_bitexact("o after rejection", gather_field(comm, "o"), before)
    cr[14, 5, 4] = 0.19
    solo.set("cr", cr)
    for r in ranks:
        r.set_domain("cr", cr)
    advance(comm, 9)
    solo.run(9)
    assert_same(comm, solo, "after recovery")
    for r in ranks:
        r.close()
    solo.close()


def _nccl_rank(port, q):
    import os
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "ni-cr_oxidation_phase-field_simulation_b200"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import nicr
    from nicr.slab_ranks import SlabRank, TorchComm, advance, gather_budget, gather_field
    from parity import smooth_fields
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        cfg = cfg_for()
        r = SlabRank(cfg, 1, 0)
        solo = nicr.Solver(cfg)
        o, cr, p, eta = smooth_fields(solo.shape, solo.n_eta, seed=5)
        for name, arr in (("o", o), ("cr", cr), ("p", p)):
            solo.set(name, arr)
            r.set_domain(name, arr)
        for g, e in enumerate(eta):
            solo.set("eta", e, g)
            r.set_domain("eta", e, g)
        solo.reset_inventory()
        r.reset_inventory()
        comm = TorchComm(r)
        out = [advance(comm, n) for n in (7, 6)]
        for n in (7, 6):
            solo.run(n)
        same = all(np.array_equal(gather_field(comm, f).view(np.int64), solo.get(f).view(np.int64))
                   for f in ("o", "cr", "p", "gb"))
        q.put((out, same, gather_budget(comm)["nuclei"], solo.budget()["nuclei"]))
        r.close()
        solo.close()
    finally:
        dist.destroy_process_group()


def test_torchcomm_over_nccl_single_rank(require_gpu):
    """TorchComm over NCCL (a world of one rank on this GPU): the MIN
    all-reduce on the library's agreement word and the stream ordering of
    the collectives with the library's kernels."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_rank, args=(port, q))
    p.start()
    out, same, n1, n2 = q.get(timeout=300)
    p.join(timeout=120)
    assert p.exitcode == 0
    assert [o[:2] for o in out] == [(0, 7), (0, 6)] and same and n1 == n2 > 0
