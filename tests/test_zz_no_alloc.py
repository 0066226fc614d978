"""nicr_step_noalloc: the allocation-free step for callers that cannot call
cudaMalloc (they own all device memory, or run where the CUDA memory API may
not be used). The test allocates the caller-side arrays itself (as such a
caller would, from its own pool) and checks two calls in a row against the
handle API's nicr_step: fields bit-identical, budget increments within the
suite's budget tolerance (1e-13 relative). Covered: the drop-in and the
reciprocal form, no grains, static grains and evolving eta (the caller passes
gb and eta_s2 of the current eta), and a grid with long X and small planes
whose default X chunk would exceed the scratch array (the call lengthens the
chunk). Collected last on purpose."""
import ctypes

import numpy as np
import pytest

import nicr
from parity import assert_bitexact, smooth_fields, ld

pytestmark = pytest.mark.gpu


class StepResult(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double * 2) for n in ("ckO", "ckCr", "clipO", "clipCr", "bcO")] + \
               [("clipped", ctypes.c_longlong), ("trial_key", ctypes.c_ulonglong)]


def entry():
    L = nicr.lib()
    f = L.nicr_step_noalloc
    f.argtypes = [ctypes.POINTER(nicr.NicrConfig)] + [ctypes.c_void_p] * 10
    f.restype = ctypes.c_int
    return f


CASES = [
    # dim, grain mode, bc, precision, shape
    (3, "static", "mu", 0, (37, 21, 45)),
    (3, "single", "concentration", 0, (37, 21, 45)),
    (2, "static", "concentration", 0, (53, 70)),
    (3, "evolving", "mu", 0, (29, 24, 33)),
    (3, "evolving", "concentration", 1, (29, 24, 33)),
    (3, "static", "mu", 1, (37, 21, 45)),
    (2, "evolving", "mu", 1, (53, 70)),
    # 120 x 320 planes are 150 step tiles; the default chunk of 16 planes gives
    # 8250 CTAs, more than the scratch array holds
    (3, "static", "concentration", 0, (872, 120, 320)),
]


@pytest.mark.parametrize("dim,mode,bc,precision,shape", CASES)
def test_noalloc_matches_handle_step_twice(require_gpu, dim, mode, bc, precision, shape):
    import torch
    # ~300 grains on the long grid (the Voronoi initialisation is O(cells x grains))
    diameter = 12. if np.prod(shape) < 1e6 else 60.
    kw = dict(nx=shape[0], ny=shape[1], grains=0 if mode == "single" else 1, grain_diameter_grid=diameter,
              grain_evolution=1 if mode == "evolving" else 0, bc=bc, ck="legacy", bounds="legacy",
              nucleation="off", dt=1e-12, precision=precision)
    if dim == 3:
        kw["nz"] = shape[2]
    cfg = nicr.make_config(dim, **kw)
    sol = nicr.Solver(cfg)
    neta = sol.n_eta if mode == "evolving" else 0
    o, cr, p, eta = smooth_fields(shape, neta, seed=5)
    p = 0.02 * (1 + np.cos(np.indices(shape).sum(axis=0) * 0.3))   # some interface cells
    sol.set_fields(o, cr, p, eta if neta else None)
    dev = torch.device("cuda", 0)
    f = entry()
    res = torch.zeros(ctypes.sizeof(StepResult), dtype=torch.uint8, device=dev)
    b0 = sol.budget()
    totals = {n: 0.0 for n in ("ckO", "ckCr", "clipO", "clipCr", "bcO")}
    clipped = 0
    cur = [torch.from_numpy(np.ascontiguousarray(sol.get(n))).to(dev) for n in ("o", "cr", "p")]
    nxt = [torch.empty_like(t) for t in cur]
    for call in range(2):
        # the caller's mask inputs of this step: gb, and eta_s2 when eta evolves
        gb = torch.from_numpy(np.ascontiguousarray(sol.get("gb"))).to(dev)
        s2 = torch.from_numpy(np.ascontiguousarray(sol.get("eta_s2"))).to(dev) if neta else None
        torch.cuda.synchronize()
        rc = f(ctypes.byref(cfg), *(t.data_ptr() for t in cur), gb.data_ptr(), s2.data_ptr() if neta else None,
               *(t.data_ptr() for t in nxt), res.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        r = StepResult.from_buffer_copy(res.cpu().numpy().tobytes())
        assert r.trial_key == 2 ** 64 - 1
        sol.step(1)
        for name, t in zip(("o", "cr", "p"), nxt):
            assert_bitexact(f"{name} (call {call + 1})", t.cpu().numpy(), sol.get(name))
        for n in totals:
            totals[n] += getattr(r, n)[0] + getattr(r, n)[1]
        clipped += r.clipped
        b = sol.budget()
        for n in totals:
            want = ld(b[n]) - ld(b0[n])
            assert abs(totals[n] - want) <= 1e-13 * (1.0 + abs(want)), (n, totals[n], want)
        assert clipped == b["clipped"] - b0["clipped"]
        cur, nxt = nxt, cur
    sol.close()


def test_noalloc_rejects_grids_beyond_its_scratch(require_gpu):
    cfg = nicr.make_config(3, nx=64, ny=4096, nz=4096 * 64, grains=0, nucleation="off")
    rc = entry()(ctypes.byref(cfg), *([None] * 10))
    assert rc == nicr._abi.ERR_INVALID_ARG
