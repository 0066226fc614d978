"""Checkpoint / restart (nicr_save_state, nicr_load_state): a run interrupted
by a checkpoint and resumed in a fresh handle must continue bit for bit as
the uninterrupted run; the file's field section must be the reference's
snapshot_state layout (mpi3d-slab/tests/regression_driver.cpp:17-32) of the
same state, checked against the oracle; bad files and foreign configurations
are rejected before the handle is touched."""
import struct

import numpy as np
import pytest

import nicr
from oracle import Oracle, make_config
from parity import assert_bitexact, smooth_fields

pytestmark = pytest.mark.gpu

BASE = dict(grain_diameter_grid=12., bounds="legacy", nucleation="ksp", dt=1e-12, radius_grid=2.5,
            nucleation_period=5e-12)
CASES = {
    "3d-static-mu": (3, (31, 21, 19), dict(grains=1, bc="mu")),
    "3d-evolving": (3, (25, 15, 13), dict(grains=1, grain_evolution=1, bc="concentration")),
    "2d-evolving": (2, (40, 33), dict(grains=1, grain_evolution=1, bc="closed")),
    "2d-center": (2, (31, 25), dict(grains=0, nucleation="center", radius_grid=4.0, bc="concentration")),
}


def cfg_of(name):
    dim, shape, kw = CASES[name]
    base = dict(BASE, nx=shape[0], ny=shape[1])
    if dim == 3:
        base["nz"] = shape[2]
    base.update(kw)
    return make_config(dim, **base)


def prepared(cfg):
    s = nicr.Solver(cfg)
    o, cr, p, eta = smooth_fields(s.shape, s.n_eta, seed=cfg.nx)
    if cfg.nucleation != nicr._abi.NUCLEATION["center"]:
        s.set_fields(o, cr, p, eta if eta else None)
        s.reset_inventory()
    return s


def state(s):
    d = {f: s.get(f) for f in ("o", "cr", "p", "gb")}
    for g in range(s.n_eta):
        d[f"eta{g + 1}"] = s.get("eta", g)
    return d


def assert_same(a, b):
    sa, sb = state(a), state(b)
    for k in sa:
        assert_bitexact(k, sa[k], sb[k])
    assert a.budget() == b.budget()
    assert a.info().steps_done == b.info().steps_done


@pytest.mark.parametrize("name", list(CASES))
def test_resume_continues_bit_for_bit(require_gpu, tmp_path, name):
    cfg = cfg_of(name)
    straight = prepared(cfg)
    straight.run(9)
    straight.run(13)
    a = prepared(cfg)
    a.run(9)
    a.save(tmp_path / "ck.bin")
    a.run(13)
    b = nicr.Solver(cfg)          # fresh handle, own initialisation, then the checkpoint
    b.load(tmp_path / "ck.bin")
    assert b.info().steps_done == 9
    b.run(13)
    assert_same(b, a)
    assert_same(a, straight)      # writing a checkpoint does not disturb the run
    if name == "3d-static-mu":
        assert a.budget()["nuclei"] > 0   # the Ksp schedule fired after the restart
    for s in (straight, a, b):
        s.close()


def test_field_section_is_the_reference_snapshot_layout(require_gpu, tmp_path):
    cfg = cfg_of("3d-evolving")
    s = prepared(cfg)
    orc = Oracle(cfg)
    o, cr, p, eta = smooth_fields(orc.shape, orc.neta, seed=cfg.nx)
    orc.set_fields(o, cr, p, np.array(eta))
    orc.reset_inventory()
    assert orc.run(5) == (0, 5)
    s.run(5)
    s.save(tmp_path / "ck.bin")
    orc.refresh()
    want = b"".join(np.ascontiguousarray(orc.get(f), dtype="<f8").tobytes()
                    for f in ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb", "eta_s2"))
    want += b"".join(np.ascontiguousarray(orc.get(f"eta{g + 1}"), dtype="<f8").tobytes() for g in range(orc.neta))
    raw = (tmp_path / "ck.bin").read_bytes()
    header_bytes = struct.unpack_from("<I", raw, 12)[0]
    info = s.info()
    start = header_bytes + info.n_seeds * 3 * 8 + info.n_seeds * 8
    assert raw[start:start + len(want)] == want
    s.close()


def test_rejections_leave_the_handle_untouched(require_gpu, tmp_path):
    cfg = cfg_of("3d-static-mu")
    a = prepared(cfg)
    a.run(4)
    a.save(tmp_path / "ck.bin")
    b = prepared(cfg)
    before = state(b)
    raw = bytearray((tmp_path / "ck.bin").read_bytes())
    raw[len(raw) // 2] ^= 0x40
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    (tmp_path / "short.bin").write_bytes(bytes(raw[: len(raw) // 3]))
    (tmp_path / "junk.bin").write_bytes(b"not a checkpoint" * 8)
    for f, msg in (("bad.bin", "checksum"), ("short.bin", "Truncated"), ("junk.bin", "Not a checkpoint"),
                   ("missing.bin", "Cannot open")):
        with pytest.raises(nicr.NicrError) as e:
            b.load(tmp_path / f)
        assert msg in str(e.value), str(e.value)
    other = make_config(3, **dict(BASE, nx=31, ny=21, nz=19, grains=1, bc="mu", dt=2e-12))
    c = nicr.Solver(other)
    with pytest.raises(nicr.NicrError) as e:
        c.load(tmp_path / "ck.bin")
    assert "dt differs" in str(e.value)
    after = state(b)
    for k in before:
        assert_bitexact(k, after[k], before[k])
    # the arithmetic form may change on restart
    fast = make_config(3, **dict(BASE, nx=31, ny=21, nz=19, grains=1, bc="mu", precision=1))
    d = nicr.Solver(fast)
    d.load(tmp_path / "ck.bin")
    assert d.info().steps_done == 4
    for s in (a, b, c, d):
        s.close()


def test_program_checkpoint_and_restart(require_gpu, tmp_path):
    """bin/nicr3d --checkpoint-every / --restart: a run stopped at step 20 and
    restarted from its checkpoint writes the same step-30 frame and
    diagnostics row as the uninterrupted run."""
    args = ["--nx", "31", "--ny", "21", "--nz", "19", "--dt", "1e-12", "--nucleation-period", "5e-12",
            "--radius-grid", "2.5", "--grain-diameter-grid", "12", "--bc", "mu", "--bounds", "legacy",
            "--output-every", "10"]
    full, first, second = tmp_path / "full", tmp_path / "first", tmp_path / "second"
    assert nicr.main(3, args + ["--steps", "30", "--out", str(full)]) == 0
    assert nicr.main(3, args + ["--steps", "20", "--checkpoint-every", "10", "--out", str(first)]) == 0
    assert (first / "checkpoint.bin").exists() and not (first / "checkpoint.bin.tmp").exists()
    assert nicr.main(3, args + ["--steps", "30", "--restart", str(first / "checkpoint.bin"), "--out", str(second)]) == 0
    assert (second / "fields_30.vti").read_bytes() == (full / "fields_30.vti").read_bytes()
    assert (second / "fields_20.vti").read_bytes() == (full / "fields_20.vti").read_bytes()
    last = lambda d: (d / "diagnostics.csv").read_text().strip().splitlines()[-1]
    assert last(second) == last(full)
    assert nicr.main(3, args + ["--steps", "30", "--restart", str(tmp_path / "none.bin"),
                                "--out", str(tmp_path / "x")]) == 1
