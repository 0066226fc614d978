"""Shared parity helpers: seeded inputs and bit-exact comparisons of the CUDA
path (nicr.Solver) against the oracle (oracle.Oracle)."""
import numpy as np

FIELDS = ("o", "cr", "p", "muO", "muCr", "mo", "mc", "gb")
BUDGET = ("nucO", "nucCr", "ckO", "ckCr", "clipO", "clipCr", "bcO", "bcCr")


def smooth_fields(shape, n_eta, seed=0):
    """Regression-driver-like inputs (mpi3d-slab/tests/regression_driver.cpp:44-45
    fills fill_smooth and zeroes phi): supersaturated O, smooth Cr, eta near 0.2."""
    rng = np.random.default_rng(seed)
    idx = np.indices(shape).astype(float) + 1.0
    i, j = idx[0], idx[1]
    k = idx[2] if len(shape) == 3 else 0.0
    o = .001 * (1. + .08 * np.sin(.3 * i + .5 * j - .4 * k)) * (1 + 1e-3 * rng.random(shape))
    cr = .19 + .001 * np.cos(.2 * i - .3 * j + .6 * k)
    p = np.zeros(shape)
    eta = [.2 + .02 * np.cos(.2 * i - .3 * j + .7 * g + .5 * k) for g in range(n_eta)]
    return o, cr, p, eta


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def assert_bitexact(name, got, want):
    got, want = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    if not np.array_equal(bits(got), bits(want)):
        diff = np.abs(got - want)
        bad = np.argwhere(bits(got) != bits(want))
        raise AssertionError(f"{name}: {len(bad)} cells differ; first {bad[0].tolist()} got {got[tuple(bad[0])]!r} "
                             f"want {want[tuple(bad[0])]!r}; max |diff| {np.nanmax(diff):.3e}")


def ld(pair):
    return float(pair[0]) + float(pair[1])


def assert_budget(got, want, rtol=1e-13):
    for n in BUDGET + ("initialO", "initialCr"):
        a, b = ld(got[n]), ld(want[n])
        assert abs(a - b) <= rtol * (1.0 + abs(b)), (n, a, b)
    assert got["nuclei"] == want["nuclei"], (got["nuclei"], want["nuclei"])
    assert got["clipped"] == want["clipped"], (got["clipped"], want["clipped"])


def compare_state(sol, orc, with_refresh=True):
    orc.refresh()
    names = FIELDS if with_refresh else ("o", "cr", "p")
    for f in names:
        assert_bitexact(f, sol.get(f), orc.get(f))
    for g in range(orc.neta):
        assert_bitexact(f"eta{g + 1}", sol.get("eta", g), orc.get(f"eta{g + 1}"))
    if orc.neta:
        assert_bitexact("eta_s2", sol.get("eta_s2"), orc.get("eta_s2"))
    assert_budget(sol.budget(), orc.budget())
