"""The learned surrogate: a 3-level 3D U-Net over the fields (c_O, c_Cr,
phi, GB indicator) and their per-step rates that predicts the state K steps
ahead, trained on trajectories the solver itself generates. Every
convolution runs on the library's BF16 tcgen05 kernels with FP32
accumulation: nicr_conv3d_fwd_act for the forward pass (bias, ReLU and the
BF16 store in its epilogue) and the data gradient, nicr_conv3d_wgrad for the
weight gradient. Pooling, upsampling, skip concatenation, the loss and the
optimiser are torch operations on the same stream. Activations are
channels-last (NDHWC) BF16; the weights' master copy is FP32. train() runs
data parallel over a process group (NCCL). JumpStepper applies the trained
network to a Solver: each jump is accepted only if the FP64 mass budget
holds and a short plain re-check agrees, otherwise the plain steps run.
"""
from __future__ import annotations

import math

import numpy as np

FIELDS = ("o", "cr", "p", "gb")
PAD = 16   # channels are padded to a multiple of 16 for the tensor-core tiles


def _lib():
    import ctypes
    from . import lib
    L = lib()
    if not getattr(L, "_conv_bound", False):
        vp, i = ctypes.c_void_p, ctypes.c_int
        for f in ("nicr_conv3d_fwd", "nicr_conv3d_fwd_tma", "nicr_conv3d_fwd_gather", "nicr_conv3d_fwd_mma_sync",
                  "nicr_conv3d_wgrad", "nicr_conv3d_wgrad_tma", "nicr_conv3d_wgrad_mma_sync"):
            getattr(L, f).argtypes = [vp, vp, vp, i, i, i, i, i, i, vp]
        L.nicr_conv3d_fwd_act.argtypes = [vp, vp, vp, i, vp, i, i, i, i, i, i, vp]
        L.nicr_conv3d_fwd_halo.argtypes = [vp, vp, vp, i, vp, i, i, i, i, i, i, vp]
        L.nicr_conv3d_fwd_march.argtypes = [vp, vp, vp, i, vp, i, i, i, i, i, i, vp]
        L.nicr_conv3d_error.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L._conv_bound = True
    return L


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} failed with status {rc}")


def conv3d_raw(x, w_bf16, form: str = "tcgen05"):
    """y = conv(x, w): x (n, d, h, w, cin) BF16, w (cout, 27, cin) BF16 -> FP32.
    form: "tcgen05" (nicr_conv3d_fwd: y-march, halo block, TMA-staged or
    gathered as the shapes allow), "march", "halo", "tma", "gather" (the
    tcgen05 forms alone) or "mma_sync"."""
    import torch
    n, d, h, wd, cin = x.shape
    cout = w_bf16.shape[0]
    y = torch.empty((n, d, h, wd, cout), dtype=torch.float32, device=x.device)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    if form in ("halo", "march"):
        f = f"nicr_conv3d_fwd_{form}"
        _check(getattr(_lib(), f)(x.data_ptr(), w_bf16.data_ptr(), None, 0, y.data_ptr(), n, d, h, wd, cin, cout,
                                  stream), f)
        return y
    f = {"tcgen05": "nicr_conv3d_fwd", "tma": "nicr_conv3d_fwd_tma", "gather": "nicr_conv3d_fwd_gather",
         "mma_sync": "nicr_conv3d_fwd_mma_sync"}[form]
    _check(getattr(_lib(), f)(x.data_ptr(), w_bf16.data_ptr(), y.data_ptr(), n, d, h, wd, cin, cout, stream), f)
    return y


def conv3d_act_raw(x, w_bf16, bias, relu: bool, out_bf16: bool):
    """act(conv(x, w) + bias) in the TMA forward's epilogue (nicr_conv3d_fwd_act):
    BF16 when out_bf16 else FP32; None where the TMA form is unavailable."""
    import torch
    n, d, h, wd, cin = x.shape
    cout = w_bf16.shape[0]
    y = torch.empty((n, d, h, wd, cout), dtype=torch.bfloat16 if out_bf16 else torch.float32, device=x.device)
    rc = _lib().nicr_conv3d_fwd_act(x.data_ptr(), w_bf16.data_ptr(), bias.data_ptr() if bias is not None else None,
                                    (1 if relu else 0) | (2 if out_bf16 else 0), y.data_ptr(), n, d, h, wd, cin, cout,
                                    torch.cuda.current_stream(x.device).cuda_stream)
    if rc == 1:   # NICR_ERR_INVALID_ARG: shapes valid (checked by the caller's layer sizes) but no tensor map
        return None
    _check(rc, "nicr_conv3d_fwd_act")
    return y


def conv_error() -> int:
    """The tcgen05 kernel's timeout flag (synchronous; cleared by the read)."""
    import ctypes
    flag = ctypes.c_int(0)
    _check(_lib().nicr_conv3d_error(ctypes.byref(flag)), "nicr_conv3d_error")
    return flag.value


def conv3d_wgrad_raw(x, dy, form: str = "tcgen05"):
    """dw[co][tap][ci] = sum_v dy[v][co] x[v + off(tap)][ci] (FP32). form:
    "tcgen05" (nicr_conv3d_wgrad: TMA-staged where Cout allows, else WMMA),
    "tma" or "mma_sync" alone."""
    import torch
    n, d, h, wd, cin = x.shape
    cout = dy.shape[-1]
    dw = torch.empty((cout, 27, cin), dtype=torch.float32, device=x.device)
    f = {"tcgen05": "nicr_conv3d_wgrad", "tma": "nicr_conv3d_wgrad_tma", "mma_sync": "nicr_conv3d_wgrad_mma_sync"}[form]
    _check(getattr(_lib(), f)(x.data_ptr(), dy.data_ptr(), dw.data_ptr(), n, d, h, wd, cin, cout,
                              torch.cuda.current_stream(x.device).cuda_stream), f)
    return dw


def _data_gradient(gyb, wt, dtype):
    """dx = conv(dy, w'), stored by the epilogue in the input's BF16 where it can."""
    import torch
    if dtype == torch.bfloat16:
        gx = conv3d_act_raw(gyb, wt, None, False, True)
        if gx is not None:
            return gx
    return conv3d_raw(gyb, wt).to(dtype)


def _make_fn():
    import torch

    class Conv3dFn(torch.autograd.Function):
        """3x3x3 convolution on the library's kernels; x BF16 NDHWC, w FP32
        master weights (cast to BF16 for the tensor cores)."""

        @staticmethod
        def forward(ctx, x, w):
            xb = x.contiguous()
            wb = w.to(torch.bfloat16).contiguous()
            ctx.save_for_backward(xb, wb)
            return conv3d_raw(xb, wb)

        @staticmethod
        def backward(ctx, gy):
            xb, wb = ctx.saved_tensors
            gyb = gy.to(torch.bfloat16).contiguous()
            # data gradient: the forward convolution of dy with w'[ci][tap][co] = w[co][26 - tap][ci]
            wt = wb.flip(1).permute(2, 1, 0).contiguous()
            gx = _data_gradient(gyb, wt, xb.dtype)
            gw = conv3d_wgrad_raw(xb, gyb)
            return gx, gw

    class ConvActFn(torch.autograd.Function):
        """act(conv(x, w) + b) with the bias, the ReLU and the BF16 store in
        the convolution's epilogue; the backward masks the gradient with the
        stored activation (y > 0), sums it for the bias and runs the data and
        weight gradients on the library's kernels."""

        @staticmethod
        def forward(ctx, x, w, b, relu, out_bf16):
            xb = x.contiguous()
            wb = w.to(torch.bfloat16).contiguous()
            bf = b.float().contiguous()
            y = conv3d_act_raw(xb, wb, bf, relu, out_bf16)
            if y is None:
                y = conv3d_raw(xb, wb) + bf
                y = torch.relu(y) if relu else y
                y = y.to(torch.bfloat16) if out_bf16 else y
            ctx.relu = relu
            ctx.save_for_backward(xb, wb, y if relu else None)
            return y

        @staticmethod
        def backward(ctx, gy):
            xb, wb, y = ctx.saved_tensors
            g = gy.float()
            if ctx.relu:
                g = g * (y > 0)
            gb = g.sum(dim=tuple(range(g.dim() - 1)))
            gyb = g.to(torch.bfloat16).contiguous()
            wt = wb.flip(1).permute(2, 1, 0).contiguous()
            gx = _data_gradient(gyb, wt, xb.dtype)
            gw = conv3d_wgrad_raw(xb, gyb)
            return gx, gw, gb, None, None

    return Conv3dFn, ConvActFn


_FN = None


def _fns():
    global _FN
    if _FN is None:
        _FN = _make_fn()
    return _FN


def conv3d(x, w):
    return _fns()[0].apply(x, w)


def conv3d_act(x, w, b, relu: bool = True, out_bf16: bool = True):
    """act(conv(x, w) + b): x BF16 NDHWC, w FP32 [Cout][27][Cin], b FP32
    [Cout]; BF16 result when out_bf16, else FP32."""
    return _fns()[1].apply(x, w, b, relu, out_bf16)


def _module_classes():
    import torch
    import torch.nn as nn

    class Conv(nn.Module):
        def __init__(self, cin, cout, relu=True):
            super().__init__()
            self.w = nn.Parameter(torch.randn(cout, 27, cin) * math.sqrt(2.0 / (27 * cin)))
            self.b = nn.Parameter(torch.zeros(cout))
            self.relu = relu

        def forward(self, x):
            # hidden layers: ReLU, BF16 activations; the head: FP32 output
            return conv3d_act(x, self.w, self.b, self.relu, out_bf16=self.relu)

    def pool(x):   # 2x2x2 average, NDHWC
        n, d, h, w, c = x.shape
        return x.float().view(n, d // 2, 2, h // 2, 2, w // 2, 2, c).mean(dim=(2, 4, 6)).to(torch.bfloat16)

    def up(x):     # nearest 2x, NDHWC
        return x.repeat_interleave(2, 1).repeat_interleave(2, 2).repeat_interleave(2, 3)

    class UNet3d(nn.Module):
        """3 levels, `base` channels at full resolution (x2 per level)."""

        def __init__(self, fields: int = 4, base: int = 32):
            super().__init__()
            c1, c2, c3 = base, 2 * base, 4 * base
            self.fields, self.base = fields, base
            self.enc1 = nn.Sequential(Conv(PAD, c1), Conv(c1, c1))
            self.enc2 = nn.Sequential(Conv(c1, c2), Conv(c2, c2))
            self.mid = nn.Sequential(Conv(c2, c3), Conv(c3, c3))
            self.dec2 = nn.Sequential(Conv(c3 + c2, c2), Conv(c2, c2))
            self.dec1 = nn.Sequential(Conv(c2 + c1, c1), Conv(c1, c1))
            self.head = Conv(c1, PAD, relu=False)

        def forward(self, x):
            """x: (n, d, h, w, fields) FP32, normalised -> the predicted change (same shape)."""
            pad = torch.zeros(x.shape[:-1] + (PAD - x.shape[-1],), dtype=x.dtype, device=x.device)
            h0 = torch.cat([x, pad], dim=-1).to(torch.bfloat16)
            e1 = self.enc1(h0)
            e2 = self.enc2(pool(e1))
            m = self.mid(pool(e2))
            d2 = self.dec2(torch.cat([up(m), e2], dim=-1))
            d1 = self.dec1(torch.cat([up(d2), e1], dim=-1))
            return self.head(d1).float()[..., : self.fields]

    return Conv, UNet3d


def unet(fields: int = 4, base: int = 32):
    return _module_classes()[1](fields, base)


_NORM_KEYS = ("mu", "sd", "rsd", "csd", "dsd")


def save_model(path, model, norm, **meta):
    """A trained surrogate in one file: the U-Net's shape and weights, the
    normaliser (K in steps and the per-field scales) and caller metadata
    (e.g. the training configurations), for JumpStepper runs in other
    processes."""
    import torch
    torch.save({"fields": model.fields, "base": model.base,
                "weights": {k: v.detach().cpu() for k, v in model.state_dict().items()},
                "steps_k": norm.steps_k, "norm": {k: getattr(norm, k).detach().cpu() for k in _NORM_KEYS},
                "meta": meta}, str(path))


def load_model(path, device="cuda"):
    """(model, normaliser, metadata) from save_model, on `device`."""
    import torch
    d = torch.load(str(path), map_location="cpu", weights_only=True)
    model = unet(d["fields"], d["base"])
    model.load_state_dict(d["weights"])
    model.to(device)
    norm = Normaliser.__new__(Normaliser)
    for k in _NORM_KEYS:
        setattr(norm, k, d["norm"][k].to(device))
    norm.steps_k = int(d["steps_k"])
    return model, norm, d["meta"]


# ------------------------------------------------------------------ data
def trajectory_configs(n: int, size: int, first_seed: int = 100, **kw):
    """Static-Voronoi runs with the batching form's parameter draws (bulk Cr
    U[0.15, 0.30], O supply U[0.5, 1.0] x the default layerO, Ksp log-uniform
    over a decade around the default, 8-32 grains), one seed per run; kw
    overrides other configuration fields."""
    from . import default_config, make_config
    d0 = default_config(3)
    out = []
    for k in range(n):
        rng = np.random.default_rng(first_seed + k)
        grains = int(rng.integers(8, 33))
        d = (6.0 * size ** 3 / (math.pi * grains)) ** (1.0 / 3.0)
        out.append(make_config(3, nx=size, ny=size, nz=size, grains=1, grain_evolution=0,
                               grain_diameter_grid=d, random_seed=first_seed + k, bc="concentration",
                               bounds="legacy", nucleation="ksp", bulk_cr=float(rng.uniform(0.15, 0.30)),
                               layer_o=d0.layer_o * float(rng.uniform(0.5, 1.0)),
                               ksp=d0.ksp * 10.0 ** float(rng.uniform(-1.0, 1.0)), **kw))
    return out


def trajectories(cfgs, steps: int, every: int, probe: int = 2, device: int = 0):
    """States (fields o, cr, p, gb) of each run at steps every, 2 every, ...,
    and their per-step rates over the `probe` steps before each: tensors
    x, r of shape (runs, steps // every, size, size, size, 4), FP32 on the
    GPU (read in place through Solver.device_view)."""
    import torch
    from . import Solver
    if every <= probe or probe < 1 or steps < every:
        raise ValueError(f"need 1 <= probe < every <= steps (probe {probe}, every {every}, steps {steps})")
    xs, rs = [], []
    for c in cfgs:
        c.device = device
        s = Solver(c)
        state = lambda: torch.stack([s.device_view(f) for f in FIELDS], dim=-1)
        x, r = [], []
        for _ in range(steps // every):
            s.run(every - probe)
            a = state()
            s.run(probe)
            b = state()
            x.append(b.float())
            r.append(((b - a) / probe).float())
        s.close()
        xs.append(torch.stack(x))
        rs.append(torch.stack(r))
    return torch.stack(xs), torch.stack(rs)


def pair_samples(cfgs, steps: int, k_steps: int, per_run: int = 2, probe: int = 2, seed: int = 0,
                 device: int = 0):
    """Training pairs from long runs: for each configuration, `per_run`
    times t drawn uniformly (seeded) in [4 * k_steps, steps - k_steps], the
    state at t with its per-step rates over the `probe` steps before, and the
    state k_steps later. Returns x, r of shape (runs * per_run, 2, size,
    size, size, 4) FP32 on the GPU, sample 0 at t and sample 1 at t + k_steps,
    for train(..., k=1, steps_k=k_steps)."""
    import torch
    from . import Solver
    rng = np.random.default_rng(seed)
    xs, rs = [], []
    for c in cfgs:
        c.device = device
        s = Solver(c)
        state = lambda: torch.stack([s.device_view(f) for f in FIELDS], dim=-1)
        times = sorted(int(t) for t in rng.integers(4 * k_steps, steps - k_steps + 1, size=per_run))
        done = 0
        for t in times:
            if t - probe > done:
                s.run(t - probe - done)
            a = state().float()
            s.run(probe)
            b = state().float()
            rate = (b - a) / probe
            s.run(k_steps)
            c1 = state().float()
            s.run(probe)
            rate1 = (state().float() - c1) / probe
            done = t + k_steps + probe
            xs.append(torch.stack([b, c1]))
            rs.append(torch.stack([rate, rate1]))
            del a
        s.close()
    return torch.stack(xs), torch.stack(rs)


def _moments(v, group):
    """(mean, std) per field of v (..., fields) over every rank of group
    (sums of v and v^2 in FP64 all-reduced; population std). Summed in
    slices of the leading dimension, so large sample sets need no FP64 copy."""
    import torch
    f = v.shape[-1]
    m = torch.zeros((3, f), dtype=torch.float64, device=v.device)
    for i in range(v.shape[0]):
        flat = v[i].reshape(-1, f).double()
        m[0] += flat.sum(0)
        m[1] += (flat * flat).sum(0)
        m[2] += float(flat.shape[0])
    if group is not None:
        import torch.distributed as dist
        dist.all_reduce(m, group=group)
    mean = m[0] / m[2]
    var = (m[1] / m[2] - mean * mean).clamp_min(0.0)
    return mean.to(v.dtype), var.sqrt().to(v.dtype)


class Normaliser:
    """Per-field scales: of the states (mu, sd), of the per-step rates (rsd),
    of the K-step changes (csd) and of the network's target, the K-step
    change minus K x the rate (dsd). K counts steps; k counts samples. With
    a process group the moments are those of every rank's samples."""

    def __init__(self, x, r, k: int, steps_k: int, group=None):
        d = x[:, k:] - x[:, :-k]
        self.mu, sd = _moments(x, group)
        self.sd = sd.clamp_min(1e-12)
        self.rsd = _moments(r, group)[1].clamp_min(1e-30)
        self.csd = _moments(d, group)[1].clamp_min(1e-30)
        self.dsd = _moments(d - steps_k * r[:, :-k], group)[1].clamp_min(1e-30)
        self.steps_k = steps_k

    def inputs(self, x, r):
        import torch
        return torch.cat([(x - self.mu) / self.sd, r / self.rsd], dim=-1)

    def target(self, x0, r0, x1):
        return (x1 - x0 - self.steps_k * r0) / self.dsd

    def apply(self, x0, r0, pred):
        return x0 + self.steps_k * r0 + pred * self.dsd


def _pairs(x, r, k):
    f = x.shape[2:]
    return x[:, :-k].reshape((-1,) + f), r[:, :-k].reshape((-1,) + f), x[:, k:].reshape((-1,) + f)


def allreduce_gradients(model, group):
    """Averages the gradients over the ranks of group: one flat bucket, one
    all-reduce (NCCL on GPUs, gloo on the CPU)."""
    import torch
    import torch.distributed as dist
    grads = [p.grad for p in model.parameters() if p.grad is not None]
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, group=group)
    flat /= dist.get_world_size(group)
    o = 0
    for g in grads:
        g.copy_(flat[o:o + g.numel()].view_as(g))
        o += g.numel()


def train(model, x, r, k: int, steps_k: int, iters: int = 200, batch: int = 2, lr: float = 2e-3, seed: int = 0,
          group=None):
    """Adam (cosine-decayed rate) on the MSE of the normalised target over
    sample pairs k apart (steps_k steps); returns (normaliser, losses).

    Data parallel with a process group: each rank passes its own
    trajectories (its share of the seeds), draws its own batches, and the
    gradients are averaged over the ranks before every optimiser step
    (allreduce_gradients), after rank 0's initial weights were broadcast; all
    ranks then hold the same weights. The losses are each rank's own."""
    import torch
    if not 1 <= k < x.shape[1] or tuple(r.shape) != tuple(x.shape):
        raise ValueError(f"need 1 <= k < samples per run ({x.shape[1]}) and rates shaped like the states")
    torch.manual_seed(seed)
    rank = 0
    if group is not None:
        import torch.distributed as dist
        rank = dist.get_rank(group)
        for p in model.parameters():
            dist.broadcast(p.data, src=dist.get_global_rank(group, 0), group=group)
    norm = Normaliser(x, r, k, steps_k, group)
    x0, r0, x1 = _pairs(x, r, k)
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, iters)
    g = torch.Generator(device="cpu").manual_seed(seed + 1000003 * rank)
    losses = []
    for _ in range(iters):
        idx = torch.randint(0, x0.shape[0], (batch,), generator=g)
        a, ra, b = x0[idx], r0[idx], x1[idx]
        loss = torch.mean((model(norm.inputs(a, ra)) - norm.target(a, ra, b)) ** 2)
        opt.zero_grad()
        loss.backward()
        if group is not None:
            allreduce_gradients(model, group)
        opt.step()
        sched.step()
        losses.append(loss.item())
    return norm, losses


def predict(model, norm, x0, r0, chunk: int = 4):
    """The network's state K steps after x0 with rates r0 (n, d, h, w, fields)."""
    import torch
    out = []
    with torch.no_grad():
        for i in range(0, x0.shape[0], chunk):
            a, ra = x0[i:i + chunk], r0[i:i + chunk]
            out.append(norm.apply(a, ra, model(norm.inputs(a, ra))))
    return torch.cat(out)


class GraphPredictor:
    """predict() for one input shape as a CUDA graph: the normalisation, every
    launch of the U-Net (convolutions included, with their tensor maps fixed
    at capture) and the un-normalisation replay as one graph from static
    input buffers. The model's weights are read in place, so training after
    capture is seen by later replays; a new shape needs a new predictor."""

    def __init__(self, model, norm, shape, device=None):
        import torch
        self.x = torch.zeros(shape, dtype=torch.float32, device=device or "cuda")
        self.r = torch.zeros_like(self.x)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side), torch.no_grad():
            for _ in range(2):   # warm-up: the library's one-time setup runs outside the capture
                norm.apply(self.x, self.r, model(norm.inputs(self.x, self.r)))
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph), torch.no_grad():
            self.out = norm.apply(self.x, self.r, model(norm.inputs(self.x, self.r)))

    def __call__(self, x0, r0):
        self.x.copy_(x0)
        self.r.copy_(r0)
        self.graph.replay()
        return self.out


def relative_errors(model, norm, x, r, k: int):
    """Relative L2 error of the K-step change (each field scaled by the
    spread of its change; c_O, c_Cr and phi) predicted by the network, by
    persistence (no change: 1 by definition), by extrapolation of the
    current rate (x + K r: the network's starting point) and by linear
    extrapolation of the previous K steps (2 x_t - x_{t-K})."""
    import torch
    f = x.shape[2:]
    x0 = x[:, k:-k].reshape((-1,) + f)
    r0 = r[:, k:-k].reshape((-1,) + f)
    xm = x[:, :-2 * k].reshape((-1,) + f)
    x1 = x[:, 2 * k:].reshape((-1,) + f)
    c = slice(0, 3)
    ref = torch.linalg.vector_norm(((x1 - x0) / norm.csd)[..., c])
    e = lambda y: float(torch.linalg.vector_norm(((y - x1) / norm.csd)[..., c]) / ref)
    return {"network": e(predict(model, norm, x0, r0)), "persistence": e(x0), "rate": e(x0 + norm.steps_k * r0),
            "linear": e(2 * x0 - xm)}


# ------------------------------------------------------------------ jumps
class JumpStepper:
    """Advances a Solver by plain steps and surrogate jumps of K steps, with
    the state read and written in place on the GPU (Solver.device_view).

    A jump is tried only where no Ksp scan falls inside it. It runs: `probe`
    plain steps (which measure the per-step rate of every field and the FP64
    rate of change of total O and Cr), the network's proposal for K steps
    ahead, the mass-budget gate, and `probe` plain re-check steps from the
    proposal.

    Mass budget: the proposal's change of total O and of total Cr must equal
    the change extrapolated from the probe steps' FP64 totals (K x their mean
    rate, or with budget="geometric" a decaying rate summed over K steps) up
    to a correction c x |change| per cell with |c| <= mass_tol; the
    correction is then applied, so the accepted state carries exactly the
    extrapolated budget (summed in FP64). Re-check: the
    per-step change of the re-check steps may be at most recheck_factor x
    that of the probe steps (an off-manifold proposal relaxes fast in its
    first plain steps). A jump failing either gate is rolled back to the
    state before it (device copies of c_O, c_Cr, phi) and K plain steps run
    instead. `ledger` holds what the solver's budget does not see: the
    amounts of accepted jumps, less the budget increments of re-check steps
    that were rolled back.

    With backoff, f consecutive rejections are followed by min(2^(f-1), 8)
    spans of plain steps before the next trial (the inlet transient, where
    the mass gate fails, costs fewer proposals).

    The stepper keeps the simulated clock itself: the solver's own step
    counter does not see jumps, so plain stepping uses nicr_step and the Ksp
    scans fire here (before the step whose physical time reaches the next
    scan time, as nicr_run fires them). Grains must be static (the jump
    leaves eta as it is).
    """

    def __init__(self, solver, model, norm, k: int, probe: int = 2, mass_tol: float = 0.05,
                 recheck_factor: float = 4.0, backoff: bool = False, graphs: bool = False,
                 budget: str = "linear"):
        from . import NUCLEATION
        if k < 1 or probe < 2:
            raise ValueError("need K >= 1 and at least 2 probe steps")
        if norm is not None and norm.steps_k != k:
            raise ValueError(f"the network predicts {norm.steps_k} steps ahead, not {k}")
        if model is not None and solver.cfg.grain_evolution:
            raise ValueError("jumps leave eta unchanged: static grains only")
        self.s, self.model, self.norm, self.k, self.probe = solver, model, norm, k, probe
        self.mass_tol, self.recheck_factor = mass_tol, recheck_factor
        if budget not in ("linear", "geometric"):
            raise ValueError(budget)
        self.budget = budget
        c = solver.cfg
        self.dt, self.period = c.dt, c.nucleation_period
        self.ksp = c.nucleation == NUCLEATION["ksp"]
        self.t = int(solver.info().steps_done)
        self.next_scan = self.period
        while self._due(self.t):
            self.next_scan += self.period
        self.ledger = {"o": 0.0, "cr": 0.0}
        self.counts = {"accepted": 0, "rejected_mass": 0, "rejected_recheck": 0, "plain_steps": 0,
                       "jumped_steps": 0, "scans": 0}
        self.gates = []   # per trial: (c for O, c for Cr, re-check ratio post / pre or None)
        # backoff: after f consecutive rejections, min(2^(f-1), 8) spans of plain steps before the next trial
        self.backoff, self.fails, self.skip = backoff, 0, 0
        # graphs: proposals replayed as a CUDA graph (GraphPredictor), captured at the first trial;
        # at 128^3 a replay takes 2.65 ms against 2.74 eager (the proposal is GPU-bound)
        self.graphs, self._graph = graphs, None

    def _predict(self, x0, r0):
        if not self.graphs:
            return predict(self.model, self.norm, x0, r0)
        if self._graph is None:
            self._graph = GraphPredictor(self.model, self.norm, tuple(x0.shape), x0.device)
        return self._graph(x0, r0)

    def _due(self, t: int) -> bool:
        """A scan fires before step t + 1."""
        return self.ksp and (t + 1) * self.dt + 1e-12 * self.period >= self.next_scan

    def _steps_free(self) -> int:
        """Steps that can run before the next scan."""
        if not self.ksp:
            return 1 << 60
        m = 0
        while not self._due(self.t + m):
            m += 1
        return m

    def plain(self, n: int):
        while n > 0:
            if self._due(self.t):
                self.s.nucleate()
                self.counts["scans"] += 1
                self.next_scan += self.period
                self._step(1)
                n -= 1
                continue
            m = min(n, self._steps_free())
            self._step(m)
            n -= m

    def _step(self, m: int):
        self.s.step(m)
        self.t += m
        self.counts["plain_steps"] += m

    def _state(self):
        """(nx, ny, nz, 4) FP64 copy of o, cr, p, gb on the GPU."""
        import torch
        return torch.stack([self.s.device_view(f) for f in FIELDS], dim=-1)

    def _write(self, x):
        import torch
        for i, f in enumerate(("o", "cr", "p")):
            self.s.device_view(f, writable=True).copy_(x[..., i])
        if x.is_cuda:   # the next library call runs on the solver's stream
            torch.cuda.current_stream(x.device).synchronize()

    def _totals(self, x):
        """FP64 totals of O and Cr (of x, or of the solver's current state)."""
        if x is None:
            return tuple(float(self.s.device_view(f).sum()) for f in ("o", "cr"))
        return float(x[..., 0].sum()), float(x[..., 1].sum())

    def _expected_change(self, t):
        """The change of a total over the next K steps from its values over
        the probe steps: K x the mean rate (budget="linear"), or, with
        budget="geometric" and a rate that keeps its sign and decays between
        the last two probe steps (ratio q), r q + r q^2 + ... + r q^K."""
        r = [b - a for a, b in zip(t, t[1:])]
        mean = (t[-1] - t[0]) / (len(t) - 1)
        if self.budget != "geometric" or len(r) < 2 or r[-2] == 0.0:
            return self.k * mean
        q = r[-1] / r[-2]
        if not 0.0 < q < 1.0:
            return self.k * mean
        return r[-1] * q * (1.0 - q ** self.k) / (1.0 - q)

    def _change(self, a, b):
        import torch
        return float(torch.linalg.vector_norm(((b - a) / self.norm.csd.double())[..., :3]))

    def _budget_total(self):
        """Amounts of O and Cr the solver's budget has recorded (inlet,
        nucleation, Ck and clipping terms)."""
        b = self.s.budget()
        species = {"o": "O", "cr": "Cr"}
        return {f: sum(b[n + sp][0] + b[n + sp][1] for n in ("bc", "nuc", "ck", "clip")) for f, sp in species.items()}

    def advance(self, n: int):
        """n simulated steps; returns the counts."""
        end = self.t + n
        span = self.k + 2 * self.probe
        while self.t < end:
            left = end - self.t
            free = self._steps_free()
            if self.model is None or left < span or free < span:
                self.plain(left if self.model is None else min(left, free + 1))
                continue
            if self.skip > 0:
                self.skip -= 1
                self.plain(span)
                continue
            t0, counts0 = self.t, dict(self.counts)
            xa = self._state()
            totals = [self._totals(xa)]
            for _ in range(self.probe):
                self.plain(1)
                totals.append(self._totals(None))
            xb = self._state()
            rb = (xb - xa) / self.probe
            pre = self._change(xa, xb) / self.probe
            prop = self._predict(xb[None].float(), rb[None].float())[0].double()
            prop[..., 3] = xb[..., 3]
            cs = []
            for i, f in ((0, "o"), (1, "cr")):
                d = prop[..., i] - xb[..., i]
                want = self._expected_change([t[i] for t in totals])
                mag = float(d.abs().sum())
                cs.append((want - float(d.sum())) / mag if mag > 0 else 0.0)
            if max(abs(c) for c in cs) > self.mass_tol:
                self.gates.append((cs[0], cs[1], None))
                self.counts["rejected_mass"] += 1
                self._rejected()
                self.plain(self.k + self.probe)
                continue
            for i, c in enumerate(cs):
                d = prop[..., i] - xb[..., i]
                prop[..., i] = xb[..., i] + d + c * d.abs()
            jumped = {f: float((prop[..., i] - xb[..., i]).sum()) for i, f in ((0, "o"), (1, "cr"))}
            self._write(prop)
            b0 = self._budget_total()
            self.t += self.k
            self.plain(self.probe)
            post = self._change(prop, self._state()) / self.probe
            self.gates.append((cs[0], cs[1], post / pre if pre > 0 else float("inf")))
            if post <= self.recheck_factor * pre:
                self.fails = 0
                self.counts["accepted"] += 1
                self.counts["jumped_steps"] += self.k
                for f in ("o", "cr"):
                    self.ledger[f] += jumped[f]
                continue
            b1 = self._budget_total()
            self._write(xb)
            for f in ("o", "cr"):
                self.ledger[f] -= b1[f] - b0[f]
            self.t, self.counts = t0 + self.probe, counts0
            self.counts["plain_steps"] += self.probe
            self.counts["rejected_recheck"] += 1
            self._rejected()
            self.plain(self.k + self.probe)
        return dict(self.counts)

    def _rejected(self):
        self.fails += 1
        if self.backoff:
            self.skip = min(2 ** (self.fails - 1), 8)

    def close(self):
        pass
