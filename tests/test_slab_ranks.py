"""Host side of the slab form with one process per GPU (nicr.slab_ranks), on
CPU: the protocol (exchange geometry and depths, MIN agreement and rollback,
the Ksp scan chain in X order, gathers) driven over host-array stand-ins of
the slabs, in one process and across two gloo processes (TorchComm), against
the same stand-in run on the whole domain. The stand-in steps o and cr with a
radius-2 stencil along X (so the two-plane halos matter), phi with radius 1,
rejects a step when o exceeds a limit (first failing cell in whole-domain
order), and runs a toy ordered nucleation scan with exclusion."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from nicr.slab_ranks import AGREE_NONE, SlabRank, TorchComm, advance, gather_budget, gather_field

NX, NY, NZ = 23, 6, 5
PERIOD, LIMIT, THR = 4, 0.9, 0.35
R_STAMP, R_EXCL = 1, 2


class FakeSlab(SlabRank):
    def __init__(self, world, index, halo=3):
        base, rem = NX // world, NX % world
        x0 = index * base + min(index, rem)
        x1 = x0 + base + (1 if index < rem else 0)
        hlo, hhi = (halo if x0 > 0 else 0), (halo if x1 < NX else 0)
        self.world, self.index, self.halo = world, index, halo
        self.x0, self.x1, self.x_lo, self.x_hi = x0, x1, hlo, hlo + (x1 - x0)
        self.stored = x1 - x0 + hlo + hhi
        self.n_eta, self.advance_eta = 0, False
        self.device = torch.device("cpu")
        self.agree = torch.full((1,), AGREE_NONE, dtype=torch.int64)
        self.box_half = R_STAMP + R_EXCL
        self.buf = {f: [np.zeros((self.stored, NY, NZ)), np.zeros((self.stored, NY, NZ))] for f in ("o", "cr", "p")}
        self.cur, self.steps_done, self.nuclei = 0, 0, 0
        self.failed_flag, self.key, self.fail_step = False, None, -1

    # planes
    def region(self, name, index, which, width):
        first = {0: self.x_lo, 1: self.x_hi - width, 2: self.x_lo - width, 3: self.x_hi}[which]
        assert 0 <= first and first + width <= self.stored
        return torch.from_numpy(self.buf[name][self.cur][first:first + width].reshape(-1))

    def _local(self, g):
        return int(np.clip(g, 0, NX - 1)) - (self.x0 - self.x_lo)

    # steps
    def begin(self, nsteps, schedule):
        self.before, self.schedule = self.steps_done, schedule
        self.failed_flag, self.key = False, None

    def scan_due(self, s):
        return self.schedule and (self.before + s + 1) % PERIOD == 0

    def note(self, s, scanned):
        pass

    def failed(self):
        return self.failed_flag

    def launch(self):
        if self.failed_flag:
            self.agree[0] = AGREE_NONE
            return
        cur, nxt = self.buf, 1 - self.cur
        key = AGREE_NONE
        for xl in range(self.x_lo, self.x_hi):
            g = self.x0 + (xl - self.x_lo)
            pl = {d: self._local(g + d) for d in (-2, -1, 1, 2)}
            o, cr, p = (cur[f][self.cur] for f in ("o", "cr", "p"))
            oc = o[xl]
            lat = np.roll(oc, 1, 0) + np.roll(oc, -1, 0) + np.roll(oc, 1, 1) + np.roll(oc, -1, 1) - 4 * oc
            on = oc + .05 * (o[pl[-2]] - 2 * oc + o[pl[2]]) + .1 * (o[pl[-1]] - 2 * oc + o[pl[1]]) + .02 * lat
            crc = cr[xl]
            crn = crc + .07 * (cr[pl[-2]] - 2 * crc + cr[pl[2]]) + .01 * oc
            pn = p[xl] + .1 * (p[pl[-1]] - 2 * p[xl] + p[pl[1]]) + .0005 * oc
            cur["o"][nxt][xl], cur["cr"][nxt][xl], cur["p"][nxt][xl] = on, crn, pn
            bad = np.argwhere(on > LIMIT)
            if len(bad):
                y, z = bad[0]
                key = min(key, (g * NY + int(y)) * NZ + int(z))
        self.agree[0] = key

    def commit(self):
        if self.failed_flag:
            return
        k = int(self.agree[0])
        if k != AGREE_NONE:
            self.failed_flag, self.key, self.fail_step = True, k, self.steps_done
            return
        self.cur, self.steps_done = 1 - self.cur, self.steps_done + 1

    def end(self, enqueued):
        if not self.failed_flag:
            return 0, enqueued, ""
        g = self.key // (NY * NZ)
        mine = self.x0 <= g < self.x1
        return 3, self.fail_step - self.before, (f"trial fails at cell {self.key}" if mine else "")

    # toy ordered nucleation: candidates with o > THR and phi < .01 in (x, y, z)
    # order; a candidate is taken unless an earlier nucleus lies within R_EXCL
    # (Chebyshev, periodic in y, z) or stamped it; a stamp sets phi = 1 within R_STAMP
    def _stamp(self, x1, y1, z1):
        for dx in range(-R_STAMP, R_STAMP + 1):
            g = x1 - 1 + dx
            lo, hi = self.x0 - self.x_lo, self.x0 - self.x_lo + self.stored
            if 0 <= g < NX and lo <= g < hi:
                for dy in range(-R_STAMP, R_STAMP + 1):
                    for dz in range(-R_STAMP, R_STAMP + 1):
                        self.buf["p"][self.cur][g - lo, (y1 - 1 + dy) % NY, (z1 - 1 + dz) % NZ] = 1.0

    def scan_candidates(self):
        o, p = self.buf["o"][self.cur], self.buf["p"][self.cur]
        own = (o[self.x_lo:self.x_hi] > THR) & (p[self.x_lo:self.x_hi] < .01)
        self.cand = [(self.x0 + int(i), int(j), int(k)) for i, j, k in np.argwhere(own)]

    @staticmethod
    def _near(a, b):
        dy, dz = abs(a[1] - b[1]) % NY, abs(a[2] - b[2]) % NZ
        return max(abs(a[0] - b[0]), min(dy, NY - dy), min(dz, NZ - dz)) <= R_EXCL

    def scan_resolve(self, pre):
        taken = [tuple(int(v) - 1 for v in row[:3]) for row in np.asarray(pre).reshape(-1, 4)]
        for t in taken:
            self._stamp(t[0] + 1, t[1] + 1, t[2] + 1)
        rows = []
        for c in self.cand:
            if self.buf["p"][self.cur][self._local(c[0]), c[1], c[2]] >= .01 or any(self._near(c, t) for t in taken):
                continue
            taken.append(c)
            self._stamp(c[0] + 1, c[1] + 1, c[2] + 1)
            rows.append([c[0] + 1, c[1] + 1, c[2] + 1, 1])
        self.nuclei += len(rows)
        return np.array(rows, dtype=np.int32).reshape(-1, 4), len(rows)

    def scan_apply(self, later):
        for row in np.asarray(later).reshape(-1, 4):
            self._stamp(int(row[0]), int(row[1]), int(row[2]))

    # data
    def own(self, name, index=0):
        return self.buf[name][self.cur][self.x_lo:self.x_hi].copy()

    def set_domain(self, name, whole, index=0):
        lo, hi = self.stored_range()
        self.buf[name][self.cur][:] = whole[lo:hi]

    def reset_inventory(self):
        pass

    def budget(self):
        return {"sum_o": (float(self.own("o").sum()), 0.0), "nuclei": self.nuclei}


class HostComm:
    """Every stand-in rank in this process."""

    def __init__(self, ranks):
        self.local = list(ranks)

    def agree(self):
        k = min(int(r.agree[0]) for r in self.local)
        for r in self.local:
            r.agree[0] = k

    def exchange(self, plans):
        by_rank = {r.index: p for r, p in zip(self.local, plans)}
        for r, plan in zip(self.local, plans):
            for (peer, f, i), (_, recv) in plan.items():
                recv.copy_(by_rank[peer][(r.index, f, i)][0])

    def any(self, flags):
        return any(flags)

    def broadcast(self, obj, src):
        return obj

    def gather(self, objs):
        return list(objs)


def initial():
    rng = np.random.default_rng(7)
    o = rng.uniform(0, .6, size=(NX, NY, NZ))
    cr = rng.uniform(.1, .3, size=(NX, NY, NZ))
    p = np.zeros((NX, NY, NZ))
    return o, cr, p


def run_ranks(ranks, comm, steps=(5, 3, 7), spike=None):
    o, cr, p = initial()
    if spike is not None:
        o[spike] = 2.0
    for r in comm.local:
        for name, a in (("o", o), ("cr", cr), ("p", p)):
            r.set_domain(name, a)
    results = [advance(comm, n, schedule=True) for n in steps]
    fields = {f: gather_field(comm, f) for f in ("o", "cr", "p")}
    return results, fields, gather_budget(comm)


def test_whole_domain_stand_in_nucleates_and_steps():
    whole = FakeSlab(1, 0)
    results, fields, budget = run_ranks([whole], HostComm([whole]))
    assert [r[0] for r in results] == [0, 0, 0]
    assert budget["nuclei"] > 2 and (fields["p"] > 0.5).sum() > 9   # stamped cells (phi diffuses after)


@pytest.mark.parametrize("world", [2, 3, 4])
def test_host_ranks_match_whole_domain(world):
    whole = FakeSlab(1, 0)
    want = run_ranks([whole], HostComm([whole]))
    ranks = [FakeSlab(world, i) for i in range(world)]
    got = run_ranks(ranks, HostComm(ranks))
    assert got[0] == want[0]
    for f in ("o", "cr", "p"):
        assert np.array_equal(got[1][f], want[1][f]), f
    assert got[2]["nuclei"] == want[2]["nuclei"]
    assert abs(got[2]["sum_o"][0] + got[2]["sum_o"][1] - want[2]["sum_o"][0]) < 1e-12


@pytest.mark.parametrize("spike", [(7, 2, 2), (8, 0, 4), (15, 3, 1)])
def test_host_ranks_reject_like_whole_domain(spike):
    whole = FakeSlab(1, 0)
    want = run_ranks([whole], HostComm([whole]), spike=spike)
    assert want[0][0][0] == 3                      # the spike fails the first batch
    ranks = [FakeSlab(3, i) for i in range(3)]
    got = run_ranks(ranks, HostComm(ranks), spike=spike)
    assert got[0] == want[0]
    for f in ("o", "cr", "p"):
        assert np.array_equal(got[1][f], want[1][f]), f


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q, spike):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slab = FakeSlab(world, rank)
        results, fields, budget = run_ranks([slab], TorchComm(slab), spike=spike)
        if rank == 0:
            q.put((results, {k: v.tolist() for k, v in fields.items()}, budget["nuclei"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spike", [None, (8, 0, 4)])
def test_gloo_ranks_match_whole_domain(spike):
    whole = FakeSlab(1, 0)
    want = run_ranks([whole], HostComm([whole]), spike=spike)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q, spike)) for r in range(2)]
    for p in procs:
        p.start()
    results, fields, nuclei = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [tuple(r) for r in results] == [tuple(r) for r in want[0]]
    for f in ("o", "cr", "p"):
        assert np.array_equal(np.array(fields[f]), want[1][f]), f
    assert nuclei == want[2]["nuclei"]
