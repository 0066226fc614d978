"""The learned surrogate end to end on one GPU: trajectories from the solver
(32^3 static Voronoi, Ksp, parameters drawn per seed), a 3D U-Net trained by
the library's BF16 convolution kernels, its K-step prediction on a held-out
seed against persistence and linear extrapolation, and JumpStepper against
the plain solver (the plain run is the oracle that reports the surrogate's
error)."""
import time

import numpy as np
import pytest

import nicr
from nicr import surrogate

pytestmark = pytest.mark.gpu

SIZE, STEPS, EVERY, KS = 32, 256, 8, 2   # K = KS x EVERY = 16 steps


@pytest.fixture(scope="module")
def trained(require_gpu):
    import torch
    cfgs = surrogate.trajectory_configs(5, SIZE, first_seed=100)
    t0 = time.perf_counter()
    x, r = surrogate.trajectories(cfgs, STEPS, EVERY)
    t1 = time.perf_counter()
    torch.manual_seed(0)
    net = surrogate.unet(4, 16).cuda()
    norm, losses = surrogate.train(net, x[:4], r[:4], KS, KS * EVERY, iters=800, batch=4)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    print(f"\ntrajectories {t1 - t0:.1f} s, training {t2 - t1:.1f} s, loss {np.mean(losses[:20]):.4g} -> "
          f"{np.mean(losses[-20:]):.4g}")
    return net, norm, losses, (x, r), cfgs


def test_training_reduces_loss(trained):
    _, _, losses, _, _ = trained
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:20])


def test_network_gain_on_held_out_seed(trained):
    """The network's K-step prediction against what the jump would be
    without it (x + K x rate, its zero output), persistence and linear
    extrapolation of the previous K steps."""
    net, norm, _, (x, r), _ = trained
    e = surrogate.relative_errors(net, norm, x[4:], r[4:], KS)
    print("\nheld-out relative L2 error of the K-step change:", e)
    assert e["persistence"] == pytest.approx(1.0)
    assert e["network"] < min(e["rate"], e["linear"], 0.7)


def test_stepper_without_network_is_the_plain_run(require_gpu):
    """Plain stepping with the stepper's own Ksp clock reproduces nicr_run
    bit for bit across several scans."""
    cfg = surrogate.trajectory_configs(1, 24, first_seed=7, nucleation_period=4e-9)[0]
    a, b = nicr.Solver(cfg), nicr.Solver(cfg)
    st = surrogate.JumpStepper(a, None, None, 16)
    st.advance(37)
    st.advance(60)
    b.run(97)
    assert st.counts["scans"] == 4 and st.counts["plain_steps"] == 97
    for f in ("o", "cr", "p"):
        assert np.array_equal(a.get(f).view(np.int64), b.get(f).view(np.int64)), f
    assert a.budget()["nuclei"] == b.budget()["nuclei"]
    st.close()
    a.close()
    b.close()


def test_jumps_against_plain_solver(trained):
    net, norm, _, _, cfgs = trained
    cfg = cfgs[4]
    jump, plain = nicr.Solver(cfg), nicr.Solver(cfg)
    jump.run(32)
    plain.run(32)
    st = surrogate.JumpStepper(jump, net, norm, KS * EVERY)
    t0 = time.perf_counter()
    counts = st.advance(192)
    t1 = time.perf_counter()
    plain.run(192)
    err = {f: float(np.abs(jump.get(f) - plain.get(f)).max() / max(np.abs(plain.get(f)).max(), 1e-300))
           for f in ("o", "cr", "p")}
    print(f"\njump stepper: {counts}, {t1 - t0:.2f} s; relative Linf error vs the plain run: {err}; "
          f"ledger {st.ledger}")
    tried = counts["accepted"] + counts["rejected_mass"] + counts["rejected_recheck"]
    assert tried >= 1
    assert counts["plain_steps"] + counts["jumped_steps"] == 192
    if counts["accepted"] == 0:
        for f in ("o", "cr", "p"):
            assert np.array_equal(jump.get(f).view(np.int64), plain.get(f).view(np.int64)), f
    else:
        assert max(err.values()) < 0.05
    st.close()
    jump.close()
    plain.close()


@pytest.mark.parametrize("gate", ["mass", "recheck"])
def test_rejected_jumps_leave_the_plain_run(trained, gate):
    """Every jump rejected (mass_tol < 0, or recheck_factor 0): the state is
    the plain run's bit for bit, and the ledger takes back the budget of the
    rolled-back re-check steps."""
    net, norm, _, _, cfgs = trained
    cfg = cfgs[4]
    jump, plain = nicr.Solver(cfg), nicr.Solver(cfg)
    jump.run(32)
    plain.run(32)
    # every trial fails the chosen gate (the mass gate wide open for the re-check case)
    kw = {"mass_tol": -1.0} if gate == "mass" else {"recheck_factor": 0.0, "mass_tol": 1e9}
    st = surrogate.JumpStepper(jump, net, norm, KS * EVERY, **kw)
    counts = st.advance(100)
    plain.run(100)
    assert counts["accepted"] == 0 and counts["plain_steps"] == 100 and counts[f"rejected_{gate}"] >= 4
    for f in ("o", "cr", "p"):
        assert np.array_equal(jump.get(f).view(np.int64), plain.get(f).view(np.int64)), f
    a, b = st._budget_total(), surrogate.JumpStepper(plain, None, None, KS * EVERY)._budget_total()
    for f in ("o", "cr"):
        assert a[f] + st.ledger[f] == pytest.approx(b[f], rel=1e-12, abs=1e-18)
    jump.close()
    plain.close()


def test_device_view_round_trip(require_gpu):
    """Solver.device_view reads the state in place and a write through a
    writable view is what the next step sees (as nicr_set_field)."""
    import torch
    cfg = surrogate.trajectory_configs(1, 24, first_seed=9)[0]
    a, b = nicr.Solver(cfg), nicr.Solver(cfg)
    a.run(5)
    b.run(5)
    for f in ("o", "cr", "p", "gb"):
        assert np.array_equal(a.device_view(f).cpu().numpy(), a.get(f))
    o = a.get("o")
    o[3:6, 4:9, 2:7] *= 1.01
    a.device_view("o", writable=True).copy_(torch.from_numpy(o).cuda())
    torch.cuda.synchronize()
    b.set("o", o)
    a.step(7)
    b.step(7)
    for f in ("o", "cr", "p"):
        assert np.array_equal(a.get(f).view(np.int64), b.get(f).view(np.int64)), f
    a.close()
    b.close()


def _nccl_train(port, q):
    import os
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "ni-cr_oxidation_phase-field_simulation_b200"))
    from nicr import surrogate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        x, r = surrogate.trajectories(surrogate.trajectory_configs(2, 16, first_seed=100), 64, 8)
        torch.manual_seed(0)
        net = surrogate.unet(4, 16).cuda()
        norm, losses = surrogate.train(net, x, r, 2, 16, iters=20, batch=2, group=dist.group.WORLD)
        ok = all(torch.isfinite(p).all() for p in net.parameters())
        q.put((ok, losses[0], losses[-1], surrogate.conv_error()))
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_over_nccl_single_rank(require_gpu):
    """train() with an NCCL group (a world of one rank on this GPU): the
    broadcast, the moment and gradient all-reduces on the library's kernels'
    stream order; the multi-rank host logic is tested over gloo on the CPU."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_train, args=(port, q))
    p.start()
    ok, first, last, err = q.get(timeout=300)
    p.join(timeout=120)
    assert p.exitcode == 0 and ok and err == 0 and last < first


def test_graph_predictor_matches_eager(trained):
    """The proposal replayed as a CUDA graph equals the eager one bit for bit,
    for new inputs written into its static buffers."""
    import torch
    net, norm, _, (x, r), _ = trained
    gp = surrogate.GraphPredictor(net, norm, (1,) + tuple(x.shape[2:]), x.device)
    for i in (3, 7):
        x0, r0 = x[4:, i].contiguous(), r[4:, i].contiguous()
        eager = surrogate.predict(net, norm, x0, r0)
        assert torch.equal(gp(x0, r0), eager)
    assert surrogate.conv_error() == 0


def test_stepper_with_graph_proposals_matches_eager(trained):
    """JumpStepper(graphs=True) replays its proposals as a CUDA graph: same
    gates, same counts and the same fields bit for bit as eager proposals."""
    net, norm, _, _, cfgs = trained
    runs = []
    for graphs in (False, True):
        s = nicr.Solver(cfgs[4])
        s.run(32)
        st = surrogate.JumpStepper(s, net, norm, KS * EVERY, mass_tol=0.25, graphs=graphs)
        counts = st.advance(96)
        runs.append((counts, st.gates, [s.get(f) for f in ("o", "cr", "p")]))
        s.close()
    (c0, g0, f0), (c1, g1, f1) = runs
    assert c0 == c1 and g0 == g1
    for a, b in zip(f0, f1):
        assert np.array_equal(a.view(np.int64), b.view(np.int64))


def test_device_view_2d(require_gpu):
    """2D handles: the view is (nx, ny), equal to get(), and a write is what
    the next step sees."""
    import torch
    cfg = nicr.make_config(2, nx=48, ny=40, grains=0, nucleation="center", radius_grid=4.0, bc="concentration",
                           ck="legacy", bounds="legacy")
    a, b = nicr.Solver(cfg), nicr.Solver(cfg)
    a.run(3)
    b.run(3)
    for f in ("o", "cr", "p"):
        v = a.device_view(f)
        assert tuple(v.shape) == a.get(f).shape and np.array_equal(v.cpu().numpy(), a.get(f))
    cr = a.get("cr")
    cr[10:20, 5:15] += 1e-3
    a.device_view("cr", writable=True).copy_(torch.from_numpy(cr).cuda())
    torch.cuda.synchronize()
    b.set("cr", cr)
    a.step(5)
    b.step(5)
    for f in ("o", "cr", "p"):
        assert np.array_equal(a.get(f).view(np.int64), b.get(f).view(np.int64)), f
    a.close()
    b.close()


def test_reloaded_model_predicts_alike(trained, tmp_path):
    """A trained surrogate saved and loaded on the GPU proposes the same
    states bit for bit."""
    import torch
    net, norm, _, (x, r), _ = trained
    surrogate.save_model(tmp_path / "s.pt", net, norm)
    net2, norm2, _ = surrogate.load_model(tmp_path / "s.pt", device="cuda")
    x0, r0 = x[4:, 5].contiguous(), r[4:, 5].contiguous()
    assert torch.equal(surrogate.predict(net, norm, x0, r0), surrogate.predict(net2, norm2, x0, r0))
