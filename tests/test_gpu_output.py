"""VTI output built on the GPU (arrays in file order and type, parallel zlib
blocks): files byte-identical to the unmodified reference's own write_vti
(oracle/_ref driver, same state, same zlib), the asynchronous writer equal
to the synchronous one while stepping continues, and the reference's
out-of-range refusal."""
import os

import numpy as np
import pytest

import nicr
from oracle import make_config, reference_available, run_reference
from parity import smooth_fields

pytestmark = pytest.mark.gpu

BASE = dict(grain_diameter_grid=12., bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5,
            nucleation_period=5e-12, bc="mu")


def cfg_for(shape, **kw):
    d = dict(BASE, nx=shape[0], ny=shape[1], nz=shape[2])
    d.update(kw)
    return make_config(3, **d)


def inputs(shape, neta, seed):
    o, cr, p, eta = smooth_fields(shape, neta, seed=seed)
    p = 0.3 * (1 + np.cos(np.indices(shape).sum(axis=0) * 0.37)) ** 2   # phi over its range: h(phi) matters
    return o, cr, np.clip(p, 0, 1), eta


@pytest.mark.skipif(not reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("shape,mode,f64,level", [
    ((25, 15, 13), "static", 0, 1),
    ((70, 21, 40), "static", 1, 6),
    ((70, 21, 40), "evolving", 0, 1),
    ((33, 40, 29), "evolving", 1, 0),
])
def test_vti_bytes_equal_the_reference(require_gpu, tmp_path, shape, mode, f64, level):
    cfg = cfg_for(shape, grains=1, grain_evolution=1 if mode == "evolving" else 0, output_float64=f64,
                  compression_level=level)
    sol = nicr.Solver(cfg)
    o, cr, p, eta = inputs(shape, sol.n_eta, seed=shape[0])
    sol.set_fields(o, cr, p, eta if eta else None)
    sol.reset_inventory()
    sol.run(7)
    ours = tmp_path / "ours.vti"
    sol.write_vti(ours)
    theirs = tmp_path / "ref.vti"
    inj = {"o": o, "cr": cr, "p": p, "eta": eta}
    run_reference(cfg, ["reset_inventory", ("run", 7), ("vti", str(theirs))], inject=inj)
    a, b = ours.read_bytes(), theirs.read_bytes()
    assert len(a) == len(b) and a == b
    sol.close()


def test_async_frame_equals_sync_frame_while_stepping(require_gpu, tmp_path):
    cfg = cfg_for((70, 21, 40), grains=1, grain_evolution=1)
    sol = nicr.Solver(cfg)
    o, cr, p, eta = inputs((70, 21, 40), sol.n_eta, seed=3)
    sol.set_fields(o, cr, p, eta)
    sol.run(3)
    sol.write_vti(tmp_path / "sync.vti")
    sol.write_vti_async(tmp_path / "async.vti")
    sol.run(5)                                    # the state changes while the frame is written
    sol.write_vti_async(tmp_path / "async2.vti")  # completes the first frame before starting
    sol.output_wait()
    assert (tmp_path / "async.vti").read_bytes() == (tmp_path / "sync.vti").read_bytes()
    sol.write_vti(tmp_path / "sync2.vti")
    assert (tmp_path / "async2.vti").read_bytes() == (tmp_path / "sync2.vti").read_bytes()
    assert not any(f.name.endswith(".tmp") for f in tmp_path.iterdir())
    sol.close()


def test_out_of_range_float32_frame_is_refused(require_gpu, tmp_path):
    cfg = cfg_for((25, 15, 13), grains=1)
    sol = nicr.Solver(cfg)
    cr = sol.get("cr")
    cr[3, 4, 5] = 1e39
    sol.set("cr", cr)
    with pytest.raises(nicr.NicrError) as e:
        sol.write_vti(tmp_path / "x.vti")
    assert "VTI conc_Cr exceeds output type range; use --output-precision float64." in str(e.value)
    sol.write_vti_async(tmp_path / "y.vti")
    with pytest.raises(nicr.NicrError) as e:
        sol.output_wait()
    assert "conc_Cr" in str(e.value)
    assert os.listdir(tmp_path) == []
    sol.close()
