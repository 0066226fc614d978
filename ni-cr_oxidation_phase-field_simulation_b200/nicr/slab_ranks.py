"""The slab form with one process per GPU: one domain split along X over the
ranks of a torch.distributed group (mpi3d-slab's decomposition, 3S:146-191,
with ranks on GPUs), each rank holding one slab (nicr_slab_* in
include/nicr.h). Per step, on the library's stream and without host
synchronisation:

    launch       every rank: step kernels into its trial buffers, then this
                 step's agreement word (int64: INT64_MAX or the first failing
                 cell's key in whole-domain order)
    agreement    MIN all-reduce of the agreement words
    commit       every rank: accept or reject alike, flip parity
    exchange     each rank sends its boundary planes of the new state to its
                 neighbours' halo planes (o, cr two planes deep; phi, and
                 with evolving grains gb and every eta, one)

A Ksp scan (every nucleation period) refreshes phi `halo` planes deep, flags
candidates on every rank, resolves rank after rank in X order (each rank gets
the nuclei the lower ranks accepted, broadcast by their owners), then stamps
the nuclei of the higher ranks. The protocol is written once, SPMD over the
ranks this process holds (`comm.local`): TorchComm runs one rank per process
over torch.distributed (NCCL between GPUs, gloo on CPU); LocalComm holds
every rank in one process (any GPUs) and moves the planes with device copies
ordered by CUDA events. The slab objects only need the methods SlabRank
defines, so the protocol also runs over host-array stand-ins.
"""
from __future__ import annotations

import ctypes

import numpy as np

AGREE_NONE = (1 << 63) - 1
# planes each field is exchanged with after a step: (field name, depth)
STEP_FIELDS = (("o", 2), ("cr", 2), ("p", 1))
ETA_FIELDS = (("gb", 1),)


class _DeviceBuffer:
    """A device allocation as __cuda_array_interface__ (zero-copy to torch)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 2}


class SlabRank:
    """Slab `index` of `world` slabs of the domain `cfg`, on GPU cfg.device."""

    def __init__(self, cfg, world: int, index: int):
        import torch
        from . import NicrError, lib
        self.cfg, self.world, self.index = cfg, world, index
        L = lib()
        self._lib = L
        self.h = ctypes.c_void_p()
        rc = L.nicr_slab_create(ctypes.byref(cfg), world, index, ctypes.byref(self.h))
        if rc != 0:
            raise NicrError(rc, L.nicr_last_error(None).decode())
        v = [ctypes.c_int(0) for _ in range(6)]
        self._check(L.nicr_slab_info(self.h, *[ctypes.byref(q) for q in v]))
        self.x0, self.x1, self.x_lo, self.x_hi, self.stored, self.halo = (q.value for q in v)
        from . import NicrInfo
        info = NicrInfo()
        self._check(L.nicr_get_info(self.h, ctypes.byref(info)))
        self.n_eta = info.n_eta
        self.advance_eta = bool(cfg.grains and cfg.grain_evolution and cfg.eta_L > 0 and self.n_eta)
        self.device = torch.device("cuda", cfg.device)
        self.stream = torch.cuda.ExternalStream(L.nicr_stream(self.h), device=self.device)
        self.agree = self._tensor(L.nicr_slab_agree_word(self.h), 1, "<i8")
        self.box_half = L.nicr_slab_box_half(self.h)

    # -------------------------------------------------------------- helpers
    def _check(self, rc: int):
        from . import NicrError
        if rc != 0:
            raise NicrError(rc, self._lib.nicr_last_error(self.h).decode())
        return rc

    def _tensor(self, ptr: int, n: int, typestr: str):
        import torch
        return torch.as_tensor(_DeviceBuffer(ptr, n, typestr), device=self.device)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self._lib.nicr_destroy(self.h)
            self.h = ctypes.c_void_p()

    # -------------------------------------------------------------- planes
    def region(self, name: str, index: int, which: int, width: int):
        """Device planes of a field: which 0/1 = the own planes next to the
        rank below/above, 2/3 = the halo planes below/above."""
        from . import FIELD
        ptr, count = ctypes.c_void_p(), ctypes.c_longlong(0)
        self._check(self._lib.nicr_slab_region(self.h, FIELD[name], index, which, width, ctypes.byref(ptr),
                                               ctypes.byref(count)))
        return self._tensor(ptr.value, count.value, "<f8")

    def exchange_plan(self, phi_only: bool = False):
        """{(peer, field, index): (send tensor, receive tensor)} of this rank."""
        fields = [("p", 0, self.halo)] if phi_only else \
            [(f, 0, w) for f, w in STEP_FIELDS] + \
            ([(f, 0, w) for f, w in ETA_FIELDS] + [("eta", g, 1) for g in range(self.n_eta)] if self.advance_eta else [])
        plan = {}
        for peer, send_which, recv_which in ((self.index - 1, 0, 2), (self.index + 1, 1, 3)):
            if 0 <= peer < self.world:
                for f, i, w in fields:
                    plan[(peer, f, i)] = (self.region(f, i, send_which, w), self.region(f, i, recv_which, w))
        return plan

    # -------------------------------------------------------------- steps
    def begin(self, nsteps: int, schedule: bool):
        self._check(self._lib.nicr_slab_begin(self.h, nsteps, 1 if schedule else 0))

    def scan_due(self, s: int) -> bool:
        return bool(self._lib.nicr_slab_scan_due(self.h, s))

    def note(self, s: int, scanned: bool):
        self._check(self._lib.nicr_slab_note_step(self.h, s, 1 if scanned else 0))

    def failed(self) -> bool:
        f = ctypes.c_int(0)
        self._check(self._lib.nicr_slab_failed(self.h, ctypes.byref(f)))
        return bool(f.value)

    def launch(self):
        self._check(self._lib.nicr_slab_launch(self.h))

    def commit(self):
        self._check(self._lib.nicr_slab_commit(self.h))

    def end(self, enqueued: int):
        """(status, accepted steps, message): the message only on the rank
        owning the failing cell."""
        done = ctypes.c_int(0)
        rc = self._lib.nicr_slab_end(self.h, enqueued, ctypes.byref(done))
        msg = self._lib.nicr_last_error(self.h).decode() if rc != 0 else ""
        return rc, done.value, msg

    # -------------------------------------------------------------- Ksp scan
    def scan_candidates(self):
        self._check(self._lib.nicr_slab_scan_candidates(self.h))

    def scan_resolve(self, pre):
        """Resolves this rank's candidates after the nuclei `pre` (x, y, z,
        full rows) of the lower ranks; returns (accepted rows, nuclei)."""
        pre = np.ascontiguousarray(np.asarray(pre, dtype=np.int32).reshape(-1, 4))
        cap = 1 << 16
        out = np.zeros((cap, 4), dtype=np.int32)
        n, k = ctypes.c_int(0), ctypes.c_int(0)
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(self._lib.nicr_slab_scan_resolve(self.h, pre.ctypes.data_as(ip), len(pre), out.ctypes.data_as(ip),
                                                     cap, ctypes.byref(n), ctypes.byref(k)))
        return out[: n.value].copy(), k.value

    def scan_apply(self, later):
        later = np.ascontiguousarray(np.asarray(later, dtype=np.int32).reshape(-1, 4))
        self._check(self._lib.nicr_slab_scan_apply(self.h, later.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                   len(later)))

    # -------------------------------------------------------------- data
    def stored_range(self):
        """Domain planes [lo, hi) this rank stores (own planes and halos)."""
        lo = self.x0 - self.x_lo
        return lo, lo + self.stored

    def own(self, name: str, index: int = 0) -> np.ndarray:
        """The field on this rank's own planes, (x1 - x0, ny, nz)."""
        from . import FIELD, _dp
        c = self.cfg
        a = np.empty(self.stored * c.ny * c.nz)
        self._check(self._lib.nicr_get_field(self.h, FIELD[name], index, _dp(a)))
        return a.reshape(self.stored, c.ny, c.nz)[self.x_lo:self.x_hi]

    def set_domain(self, name: str, whole: np.ndarray, index: int = 0):
        """Sets a state field from the whole-domain array (every stored plane)."""
        from . import FIELD, _dp
        lo, hi = self.stored_range()
        a = np.ascontiguousarray(np.asarray(whole, dtype=np.float64)[lo:hi]).ravel()
        self._check(self._lib.nicr_set_field(self.h, FIELD[name], index, _dp(a)))

    def reset_inventory(self):
        self._check(self._lib.nicr_reset_inventory(self.h))

    def budget(self) -> dict:
        from . import NicrBudget
        b = NicrBudget()
        self._check(self._lib.nicr_get_budget(self.h, ctypes.byref(b)))
        d = {n: (getattr(b, n)[0], getattr(b, n)[1]) for n in
             ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr", "initialO", "initialCr")}
        d["nuclei"], d["clipped"] = int(b.nuclei), int(b.clipped)
        return d

    def adjacency(self) -> np.ndarray:
        """This slab's part of the grains' face adjacency (ng x ng bytes)."""
        ng = len(self._seeds())
        adj = np.zeros(ng * ng, dtype=np.uint8)
        self._check(self._lib.nicr_slab_adjacency(self.h, adj.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))))
        return adj

    def set_colours(self, adj: np.ndarray):
        """Colours the grains from the domain's adjacency and fills eta."""
        ng = len(self._seeds())
        colours = np.zeros(ng, dtype=np.int32)
        a = np.ascontiguousarray(adj, dtype=np.uint8)
        self._check(self._lib.nicr_colour_grains(a.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), ng,
                                                 self.cfg.eta_colours, colours.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self._check(self._lib.nicr_slab_set_colours(self.h, colours.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def _seeds(self):
        from . import NicrInfo, _dp
        info = NicrInfo()
        self._check(self._lib.nicr_get_info(self.h, ctypes.byref(info)))
        xyz = np.zeros(info.n_seeds * 3)
        vol = np.zeros(info.n_seeds, dtype=np.int64)
        self._check(self._lib.nicr_get_seeds(self.h, _dp(xyz), vol.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return xyz.reshape(-1, 3)


# ------------------------------------------------------------------ communicators
class TorchComm:
    """This process's rank (one slab) of a torch.distributed group: NCCL for
    slabs on GPUs, gloo for host-array slabs."""

    def __init__(self, rank_obj, group=None):
        self.local = [rank_obj]
        self.group = group

    def _stream(self):
        import contextlib
        import torch
        r = self.local[0]
        return torch.cuda.stream(r.stream) if r.device.type == "cuda" else contextlib.nullcontext()

    def agree(self):
        import torch.distributed as dist
        with self._stream():
            dist.all_reduce(self.local[0].agree, op=dist.ReduceOp.MIN, group=self.group)

    def exchange(self, plans):
        import torch.distributed as dist
        (plan,) = plans
        with self._stream():
            ops = []
            for (peer, f, i), (send, recv) in sorted(plan.items()):
                ops.append(dist.P2POp(dist.isend, send, peer, group=self.group))
                ops.append(dist.P2POp(dist.irecv, recv, peer, group=self.group))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()

    def any(self, flags) -> bool:
        import torch
        import torch.distributed as dist
        r = self.local[0]
        t = torch.tensor([1 if any(flags) else 0], dtype=torch.int64, device=r.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=self.group)
        return bool(t.item())

    def broadcast(self, obj, src: int):
        import torch.distributed as dist
        box = [obj]
        dist.broadcast_object_list(box, src=src, group=self.group)
        return box[0]

    def gather(self, obj) -> list:
        import torch.distributed as dist
        out = [None] * dist.get_world_size(self.group)
        dist.all_gather_object(out, obj, group=self.group)
        return out

    def reduce_or(self, arrays) -> np.ndarray:
        return np.bitwise_or.reduce(np.stack([a for part in self.gather(arrays) for a in part]), axis=0)


class LocalComm:
    """Every rank in this process (slabs on one or several GPUs): the halo
    planes and agreement words move by device copies on the receiving rank's
    stream after a wait on the sending rank's event, so no host
    synchronisation enters a step."""

    def __init__(self, ranks):
        self.local = list(ranks)

    def _events(self):
        import torch
        evs = []
        for r in self.local:
            e = torch.cuda.Event()
            e.record(r.stream)
            evs.append(e)
        return evs

    def _wait_all(self, evs):
        for r in self.local:
            for e in evs:
                r.stream.wait_event(e)

    def agree(self):
        import torch
        ready = self._events()
        self._wait_all(ready)
        for r in self.local:
            with torch.cuda.stream(r.stream):
                words = torch.cat([q.agree.to(r.device) for q in self.local])
                r.agree.copy_(words.min().view(1))
        self._wait_all(self._events())   # nobody rewrites its word before every rank has read it

    def exchange(self, plans):
        import torch
        by_rank = {r.index: p for r, p in zip(self.local, plans)}
        self._wait_all(self._events())
        for r, plan in zip(self.local, plans):
            with torch.cuda.stream(r.stream):
                for (peer, f, i), (_, recv) in plan.items():
                    send, _ = by_rank[peer][(r.index, f, i)]
                    recv.copy_(send.to(r.device))
        self._wait_all(self._events())   # the sources stay untouched until every copy is done

    def any(self, flags) -> bool:
        return any(flags)

    def broadcast(self, obj, src: int):
        return obj

    def gather(self, objs) -> list:
        return list(objs)

    def reduce_or(self, arrays) -> np.ndarray:
        return np.bitwise_or.reduce(np.stack(arrays), axis=0)


# ------------------------------------------------------------------ the protocol
def colour_grains(comm):
    """The coloured eta initialisation (eta_colours > 0) of every rank: the
    union of the slabs' adjacencies is the domain's (every face between two
    planes lies in some slab's stored planes)."""
    adj = comm.reduce_or([r.adjacency() for r in comm.local])
    for r in comm.local:
        r.set_colours(adj)


def _near(nuclei, r):
    """The nuclei whose stamp or exclusion marks reach rank r's stored planes."""
    lo, hi = r.stored_range()
    if len(nuclei) == 0:
        return np.zeros((0, 4), dtype=np.int32)
    a = np.asarray(nuclei, dtype=np.int32).reshape(-1, 4)
    x = a[:, 0]
    return a[(x + r.box_half >= lo + 1) & (x - r.box_half <= hi)]


def scan(comm) -> int:
    """One Ksp scan of the whole domain (Model::nucleate, 3S:752-759)."""
    ranks = comm.local
    comm.exchange([r.exchange_plan(phi_only=True) for r in ranks])
    for r in ranks:
        r.scan_candidates()
    world = ranks[0].world
    mine = {r.index: r for r in ranks}
    accepted, per_rank, nuclei = np.zeros((0, 4), dtype=np.int32), [], 0
    for s in range(world):
        out = None
        if s in mine:
            rows, k = mine[s].scan_resolve(_near(accepted, mine[s]))
            out = (rows, k)
        rows, k = comm.broadcast(out, src=s)
        per_rank.append(rows)
        accepted = np.concatenate([accepted, rows])
        nuclei += k
    for r in ranks:
        later = np.concatenate([np.zeros((0, 4), dtype=np.int32)] + per_rank[r.index + 1:])
        r.scan_apply(_near(later, r))
    return nuclei


def advance(comm, nsteps: int, schedule: bool = True):
    """nsteps steps of the domain (nicr_run when schedule, else nicr_step).
    Returns (status, accepted steps, message) on every rank."""
    ranks = comm.local
    for r in ranks:
        r.begin(nsteps, schedule)
    enqueued = 0
    for s in range(nsteps):
        if schedule:
            scanned = False
            if ranks[0].scan_due(s):
                if comm.any([r.failed() for r in ranks]):
                    break                      # a rejected step ends the batch
                scan(comm)
                scanned = True
            for r in ranks:
                r.note(s, scanned)
        for r in ranks:
            r.launch()
        comm.agree()
        for r in ranks:
            r.commit()
        comm.exchange([r.exchange_plan() for r in ranks])
        enqueued += 1
    results = [r.end(enqueued) for r in ranks]
    msgs = [m for res in comm.gather([res[2] for res in results]) for m in (res if isinstance(res, list) else [res])]
    msg = next((m for m in msgs if m), "")
    rc, done, _ = results[0]
    return rc, done, msg


def gather_field(comm, name: str, index: int = 0) -> np.ndarray:
    """The whole-domain field on every rank."""
    parts = comm.gather([(r.x0, r.own(name, index)) for r in comm.local])
    flat = [p for part in parts for p in (part if isinstance(part, list) else [part])]
    flat.sort(key=lambda t: t[0])
    return np.concatenate([a for _, a in flat])


def gather_budget(comm) -> dict:
    """The domain budget: the ranks' double-double sums added in rank order."""
    parts = comm.gather([(r.index, r.budget()) for r in comm.local])
    flat = sorted((p for part in parts for p in (part if isinstance(part, list) else [part])), key=lambda t: t[0])
    out = {}
    for k in flat[0][1]:
        if isinstance(flat[0][1][k], tuple):
            hi, lo = 0.0, 0.0
            for _, b in flat:
                for v in b[k]:
                    s = hi + v                      # two-sum of hi + v, error folded into lo
                    bb = s - hi
                    lo += (hi - (s - bb)) + (v - bb)
                    hi = s
            out[k] = (hi, lo)
        else:
            out[k] = sum(b[k] for _, b in flat)
    return out
