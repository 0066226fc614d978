"""Data-parallel training of the surrogate (nicr.surrogate.train with a
process group) on the CPU: two gloo ranks with different trajectories. The
library's CUDA convolutions are replaced, in these processes only, by torch's
own conv3d on the CPU (tests/conv_ref.py), so that the host logic runs here:
the broadcast of rank 0's weights, the all-reduced normaliser moments, the
one-bucket gradient all-reduce, and identical weights on every rank after
training. The same code runs over NCCL on GPUs (test_gpu_surrogate.py runs a
one-rank NCCL group)."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cpu_convolutions(surrogate):
    import conv_ref

    def fwd(x, w, form="tcgen05"):
        return conv_ref.conv3d(x.float(), w.float()).float()

    def wgrad(x, dy, form="tcgen05"):
        x, dy = x.detach().double(), dy.detach().double()
        n, d, h, w, ci = x.shape
        xp = torch.nn.functional.pad(x, (0, 0, 1, 1, 1, 1, 1, 1))
        out = torch.zeros(dy.shape[-1], 27, ci, dtype=torch.float64)
        for tap in range(27):
            a, b, c = tap // 9, tap // 3 % 3, tap % 3
            out[:, tap] = torch.einsum("ndhwo,ndhwi->oi", dy, xp[:, a:a + d, b:b + h, c:c + w])
        return out.float()

    surrogate.conv3d_raw = fwd
    surrogate.conv3d_wgrad_raw = wgrad
    surrogate.conv3d_act_raw = lambda *a: None   # the unfused path over the stand-ins


def _data(rank):
    g = torch.Generator().manual_seed(100 + rank)
    x = torch.randn((1, 5, 8, 8, 8, 4), generator=g)
    r = torch.randn((1, 5, 8, 8, 8, 4), generator=g) * 0.1
    return x, r


def _rank(rank, world, port, q):
    import torch.distributed as dist
    from nicr import surrogate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        _cpu_convolutions(surrogate)
        torch.manual_seed(rank)                      # different initial weights on every rank
        net = surrogate.unet(4, 16)
        init0 = [p.detach().clone() for p in net.parameters()]
        x, r = _data(rank)
        norm, losses = surrogate.train(net, x, r, 2, 8, iters=3, batch=1, group=dist.group.WORLD)
        flat = torch.cat([p.detach().reshape(-1) for p in net.parameters()])
        every = [torch.zeros_like(flat) for _ in range(world)]
        dist.all_gather(every, flat)
        # one more backward: the all-reduced gradient is the mean of the ranks' own
        xa, ra, xb = surrogate._pairs(x, r, 2)
        net.zero_grad()
        torch.mean((net(norm.inputs(xa[:1], ra[:1])) - norm.target(xa[:1], ra[:1], xb[:1])) ** 2).backward()
        own = torch.cat([p.grad.reshape(-1) for p in net.parameters()])
        grads = [torch.zeros_like(own) for _ in range(world)]
        dist.all_gather(grads, own)
        surrogate.allreduce_gradients(net, dist.group.WORLD)
        reduced = torch.cat([p.grad.reshape(-1) for p in net.parameters()])
        if rank == 0:
            whole_x = torch.cat([_data(i)[0] for i in range(world)])
            whole_r = torch.cat([_data(i)[1] for i in range(world)])
            single = surrogate.Normaliser(whole_x, whole_r, 2, 8)
            torch.manual_seed(0)
            q.put({
                "same_weights": all(torch.equal(e, every[0]) for e in every),
                "moved": any(not torch.equal(a, p.detach()) for a, p in zip(init0, net.parameters())),
                "mean_grad": float((reduced - sum(grads) / world).abs().max() / own.abs().max()),
                "norm": max(float((getattr(norm, n) - getattr(single, n)).abs().max() / getattr(single, n).abs().max())
                            for n in ("mu", "sd", "rsd", "csd", "dsd")),
                "losses": losses,
            })
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out["same_weights"] and out["moved"]
    assert out["mean_grad"] < 1e-6
    assert out["norm"] < 1e-6
    assert len(out["losses"]) == 3 and all(l == l for l in out["losses"])
