"""nicr_step_noalloc: the allocation-free step for callers that cannot call
cudaMalloc (they own all device memory, or run where the CUDA memory API may
not be used). The test allocates the caller-side arrays itself (as such a
caller would, from its own pool) and checks two calls in a row against the
handle API's nicr_step: fields bit-identical, budget increments within the
suite's budget tolerance (1e-13 relative). Collected last on purpose."""
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


@pytest.mark.parametrize("dim,mode,bc", [(3, "static", "mu"), (3, "single", "concentration"), (2, "static", "concentration")])
def test_noalloc_matches_handle_step_twice(require_gpu, dim, mode, bc):
    import torch
    shape = (37, 21, 45) if dim == 3 else (53, 70)
    kw = dict(nx=shape[0], ny=shape[1], grains=1 if mode == "static" else 0, grain_diameter_grid=12.,
              bc=bc, ck="legacy", bounds="legacy", nucleation="off", dt=1e-12)
    if dim == 3:
        kw["nz"] = shape[2]
    cfg = nicr.make_config(dim, **kw)
    sol = nicr.Solver(cfg)
    o, cr, p, _ = smooth_fields(shape, 0, seed=5)
    p = 0.02 * (1 + np.cos(np.indices(shape).sum(axis=0) * 0.3))   # some interface cells
    sol.set_fields(o, cr, p)
    dev = torch.device("cuda", 0)
    cur = [torch.from_numpy(np.ascontiguousarray(sol.get(f))).to(dev) for f in ("o", "cr", "p")]
    gb = torch.from_numpy(np.ascontiguousarray(sol.get("gb"))).to(dev)
    nxt = [torch.empty_like(t) for t in cur]
    res = torch.zeros(ctypes.sizeof(StepResult), dtype=torch.uint8, device=dev)
    f = entry()
    b0 = sol.budget()
    totals = {n: 0.0 for n in ("ckO", "ckCr", "clipO", "clipCr", "bcO")}
    clipped = 0
    for call in range(2):
        torch.cuda.synchronize()
        rc = f(ctypes.byref(cfg), *(t.data_ptr() for t in cur), gb.data_ptr(), None,
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
    cfg = nicr.make_config(3, nx=64, ny=4096, nz=4096, grains=0, nucleation="off")
    rc = entry()(ctypes.byref(cfg), *([None] * 10))
    assert rc == nicr._abi.ERR_INVALID_ARG
