"""Host logic of the surrogate's JumpStepper on the CPU, over a fake solver
(torch CPU tensors with a deterministic toy update and a toy inlet budget)
and a network whose output is zero, so that a proposal is the rate
extrapolation x + K r: the Ksp scan schedule of nicr_run, the gates'
accounting, accepted jumps where the toy dynamics are exactly linear, and
rollbacks that leave the plain run bit for bit with the ledger taking back
the budget of the undone re-check steps."""
import types

import pytest
import torch

from nicr import NUCLEATION
from nicr import surrogate

SHAPE = (4, 5, 6)


class FakeSolver:
    """o grows by a constant inflow per step (exactly linear), cr relaxes
    towards 0.2 (decaying), p stays; the inlet budget counts the inflow."""

    def __init__(self, linear_cr=False, period_steps=40):
        self.cfg = types.SimpleNamespace(dt=1e-3, nucleation_period=period_steps * 1e-3, nucleation=NUCLEATION["ksp"],
                                         grain_evolution=0)
        g = torch.Generator().manual_seed(3)
        self.f = {"o": torch.rand(SHAPE, generator=g, dtype=torch.float64) * 0.01,
                  "cr": 0.2 + 0.05 * torch.rand(SHAPE, generator=g, dtype=torch.float64),
                  "p": torch.zeros(SHAPE, dtype=torch.float64), "gb": torch.rand(SHAPE, generator=g, dtype=torch.float64)}
        self.linear_cr = linear_cr
        self.steps, self.scans, self.bc = 0, [], 0.0

    def info(self):
        return types.SimpleNamespace(steps_done=self.steps)

    def step(self, m):
        for _ in range(m):
            self.f["o"] += 1e-4
            self.bc += 1e-4 * self.f["o"].numel()
            self.f["cr"] += -1e-5 if self.linear_cr else 0.01 * (0.2 - self.f["cr"])
            self.steps += 1
        return 0, m

    def run(self, m):
        """nicr_run's schedule: a scan before the step whose time reaches the next scan time."""
        for _ in range(m):
            n = self.steps + 1
            if n * self.cfg.dt + 1e-12 * self.cfg.nucleation_period >= self.next_scan:
                self.nucleate()
                self.next_scan += self.cfg.nucleation_period
            self.step(1)

    def nucleate(self):
        self.scans.append(self.steps)
        return 0

    def device_view(self, name, index=0, writable=False):
        return self.f[name]

    def budget(self):
        z = (0.0, 0.0)
        return {"bcO": (self.bc, 0.0), "nucO": z, "ckO": z, "clipO": z, "bcCr": z, "nucCr": z, "ckCr": z,
                "clipCr": z}


def norm_for(solver, k):
    x = torch.stack([solver.f[n] for n in ("o", "cr", "p", "gb")], dim=-1).float()
    xs = torch.stack([x, x + 1e-3, x + 2e-3])[None]          # (runs, samples, ..., 4)
    return surrogate.Normaliser(xs, torch.full_like(xs, 1e-4), 1, k)


def zero_model(inp):
    return torch.zeros(inp.shape[:-1] + (4,))


def test_scan_schedule_matches_run():
    a, b = FakeSolver(), FakeSolver()
    b.next_scan = b.cfg.nucleation_period
    st = surrogate.JumpStepper(a, None, None, 8)
    st.advance(37)
    st.advance(90)
    b.run(127)
    assert a.scans == b.scans == [39, 79, 119] and st.counts["scans"] == 3 and a.steps == b.steps == 127
    assert torch.equal(a.f["o"], b.f["o"]) and torch.equal(a.f["cr"], b.f["cr"])


def test_linear_dynamics_jump_exactly():
    """With o and cr exactly linear in time, rate extrapolation is exact: every
    trial passes both gates (re-check ratio 1) and the jumped state matches
    the plain run up to the FP32 rounding of the proposal."""
    k = 8
    a, b = FakeSolver(linear_cr=True, period_steps=10 ** 6), FakeSolver(linear_cr=True, period_steps=10 ** 6)
    st = surrogate.JumpStepper(a, zero_model, norm_for(a, k), k)
    counts = st.advance(60)
    b.step(60)
    assert counts["accepted"] >= 4 and counts["rejected_mass"] == 0 and counts["rejected_recheck"] == 0
    assert counts["plain_steps"] + counts["jumped_steps"] == 60
    # proposals are computed in FP32 (the network's precision): FP32 rounding of values up to 0.25
    for n in ("o", "cr"):
        assert torch.allclose(a.f[n], b.f[n], rtol=0, atol=2e-8), n
    # the jumps' O is in the ledger, not in the fake solver's inlet count
    assert st.ledger["o"] + a.bc == pytest.approx(b.bc, rel=1e-9)


@pytest.mark.parametrize("gate", ["mass", "recheck"])
def test_rejections_leave_the_plain_run(gate):
    k = 8
    a, b = FakeSolver(period_steps=10 ** 6), FakeSolver(period_steps=10 ** 6)
    kw = {"mass_tol": -1.0} if gate == "mass" else {"recheck_factor": 0.0, "mass_tol": 1e9}
    st = surrogate.JumpStepper(a, zero_model, norm_for(a, k), k, **kw)
    counts = st.advance(50)
    b.step(50)
    assert counts["accepted"] == 0 and counts[f"rejected_{gate}"] >= 3 and counts["plain_steps"] == 50
    for n in ("o", "cr", "p"):
        assert torch.equal(a.f[n], b.f[n]), n
    # undone re-check steps ran through the fake budget: the ledger takes them back
    assert a.bc + st.ledger["o"] == pytest.approx(b.bc, rel=1e-12)


def test_expected_change_models():
    a = FakeSolver()
    st = surrogate.JumpStepper(a, None, None, 10, budget="geometric")
    assert st._expected_change([0.0, 1.0, 1.5]) == pytest.approx(0.5 * 0.5 * (1 - 0.5 ** 10) / 0.5)
    assert st._expected_change([0.0, 1.0, 2.0]) == pytest.approx(10.0)   # no decay: linear
    st.budget = "linear"
    assert st._expected_change([0.0, 1.0, 1.5]) == pytest.approx(7.5)
    with pytest.raises(ValueError):
        surrogate.JumpStepper(a, None, None, 10, budget="cubic")


def test_save_and_load_model(tmp_path):
    """save_model / load_model: the U-Net's shape and weights, the normaliser
    and the metadata round-trip exactly (on the CPU)."""
    torch.manual_seed(1)
    net = surrogate.unet(4, 16)
    x = torch.randn((1, 4, 8, 8, 8, 4))
    norm = surrogate.Normaliser(x, torch.randn_like(x) * 0.1, 2, 16)
    surrogate.save_model(tmp_path / "s.pt", net, norm, seeds=[100, 101])
    net2, norm2, meta = surrogate.load_model(tmp_path / "s.pt", device="cpu")
    assert meta == {"seeds": [100, 101]} and net2.base == 16 and net2.fields == 4 and norm2.steps_k == 16
    for (k, a), (k2, b) in zip(net.state_dict().items(), net2.state_dict().items()):
        assert k == k2 and torch.equal(a, b)
    for k in ("mu", "sd", "rsd", "csd", "dsd"):
        assert torch.equal(getattr(norm, k), getattr(norm2, k))
    xi, ri = x[0, :1], x[0, :1] * 0.1
    assert torch.equal(norm.inputs(xi, ri), norm2.inputs(xi, ri))


def test_argument_checks():
    x = torch.zeros((1, 3, 4, 4, 4, 4))
    net = surrogate.unet(4, 16)
    with pytest.raises(ValueError):
        surrogate.train(net, x, x, 3, 16)          # k must leave pairs
    with pytest.raises(ValueError):
        surrogate.train(net, x, x[:, :2], 1, 16)   # rates shaped like the states
    with pytest.raises(ValueError):
        surrogate.trajectories([], 64, 2, probe=2)
    a = FakeSolver()
    with pytest.raises(ValueError):
        surrogate.JumpStepper(a, None, None, 8, probe=1)
    with pytest.raises(ValueError):
        surrogate.JumpStepper(a, zero_model, norm_for(a, 8), 16)   # K of the network
