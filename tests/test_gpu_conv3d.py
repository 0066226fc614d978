"""The surrogate's BF16 tensor-core convolutions (nicr_conv3d_fwd,
nicr_conv3d_wgrad) and their autograd wrapper against torch's conv3d in FP64
on the CPU, on BF16-representable inputs. Bound: FP32 accumulation, so each
output may differ from the FP64 value by at most 1e-4 x the same sum taken
over absolute values (a wrong tap, channel or voxel gives errors of order 1)."""
import pytest
import torch

import conv_ref
from nicr import surrogate

pytestmark = pytest.mark.gpu

# (n, d, h, w, cin, cout): chunks of 64/48/32/16 channels, a partial
# 128-voxel tile (64 voxels), two output-channel tiles (cout 272 = 256 + 16)
# and rows of 128 voxels or more (the halo-block form: one x tile, a partial
# second x tile, 1 to 4 chunks of 16 input channels)
SHAPES = [(2, 4, 8, 8, 16, 48), (1, 8, 8, 8, 32, 64), (1, 6, 4, 16, 48, 16), (2, 16, 16, 16, 16, 32),
          (1, 8, 8, 8, 96, 128), (1, 4, 4, 4, 16, 16), (1, 4, 8, 8, 32, 272), (1, 4, 4, 8, 80, 32),
          (1, 8, 8, 8, 64, 256), (1, 3, 4, 128, 16, 16), (1, 2, 3, 160, 48, 32), (1, 2, 4, 136, 64, 48),
          (1, 3, 20, 128, 16, 16), (2, 2, 16, 200, 32, 32), (1, 2, 1, 128, 48, 16)]
HALO = lambda shape: shape[3] >= 128 and shape[5] <= 64
# the y-march form: Cin <= 48, Cout <= 32, rows >= 128, and its shared memory (27 x Cin x Cout x 2 B of
# weights beside 4 x Cin/8 input planes) within a CTA's
MARCH = lambda shape: (shape[3] >= 128 and shape[4] <= 48 and shape[5] <= 32 and
                       4 * (shape[4] // 8) * 6272 + 27 * shape[4] * shape[5] * 2 + 1080 <= 227 * 1024)
TOL = 1e-4


def inputs(shape, seed):
    n, d, h, w, ci, co = shape
    g = torch.Generator().manual_seed(seed)
    x = conv_ref.bf16_rounded((n, d, h, w, ci), g)
    wt = conv_ref.bf16_rounded((co, 27, ci), g, 0.2)
    dy = conv_ref.bf16_rounded((n, d, h, w, co), g)
    return x, wt, dy


def within(got, ref, bound, label):
    err = (got.double().cpu() - ref).abs()
    worst = float((err / (bound + 1e-300)).max())
    assert worst <= TOL, f"{label}: error {worst:.3g} x the absolute-value bound"


@pytest.mark.parametrize("form", ["tcgen05", "march", "halo", "tma", "gather", "mma_sync"])
@pytest.mark.parametrize("shape", SHAPES)
def test_forward(require_gpu, shape, form):
    x, wt, _ = inputs(shape, 1)
    if (form == "halo" and not HALO(shape)) or (form == "march" and not MARCH(shape)):
        with pytest.raises(RuntimeError):
            surrogate.conv3d_raw(x.cuda().bfloat16(), wt.cuda().bfloat16(), form)
        return
    y = surrogate.conv3d_raw(x.cuda().bfloat16(), wt.cuda().bfloat16(), form)
    torch.cuda.synchronize()
    within(y, conv_ref.conv3d(x, wt), conv_ref.conv3d(x.abs(), wt.abs()), f"forward ({form})")
    assert surrogate.conv_error() == 0


@pytest.mark.parametrize("shape", SHAPES)
def test_data_gradient(require_gpu, shape):
    x, wt, dy = inputs(shape, 2)
    dx_ref, _ = conv_ref.grads(x, wt, dy)
    wf = conv_ref.dgrad_weights(wt)
    dx = surrogate.conv3d_raw(dy.cuda().bfloat16(), wf.cuda().bfloat16())
    within(dx, dx_ref, conv_ref.conv3d(dy.abs(), wf.abs()), "data gradient")


TMA_WGRAD_COUT = (16, 32, 64, 128, 256)


@pytest.mark.parametrize("form", ["tcgen05", "tma", "mma_sync"])
@pytest.mark.parametrize("shape", SHAPES)
def test_weight_gradient(require_gpu, shape, form):
    x, wt, dy = inputs(shape, 3)
    xb, dyb = x.cuda().bfloat16(), dy.cuda().bfloat16()
    if form == "tma" and shape[-1] not in TMA_WGRAD_COUT:
        with pytest.raises(RuntimeError):
            surrogate.conv3d_wgrad_raw(xb, dyb, form)
        return
    _, dw_ref = conv_ref.grads(x, wt, dy)
    _, dw_abs = conv_ref.grads(x.abs(), wt, dy.abs())
    dw = surrogate.conv3d_wgrad_raw(xb, dyb, form)
    within(dw, dw_ref, dw_abs, f"weight gradient ({form})")
    assert surrogate.conv_error() == 0


def test_autograd_wrapper(require_gpu):
    """Conv3dFn's gradients: dw in FP32, dx rounded to the input's BF16."""
    x, wt, dy = inputs((1, 8, 8, 8, 32, 48), 4)
    dx_ref, dw_ref = conv_ref.grads(x, wt, dy)
    xg = x.cuda().bfloat16().requires_grad_(True)
    wg = wt.cuda().requires_grad_(True)
    y = surrogate.conv3d(xg, wg)
    (y * dy.cuda()).sum().backward()
    _, dw_abs = conv_ref.grads(x.abs(), wt, dy.abs())
    within(wg.grad, dw_ref, dw_abs, "autograd dw")
    rel = float((xg.grad.double().cpu() - dx_ref).abs().max() / dx_ref.abs().max())
    assert rel < 8e-3


@pytest.mark.parametrize("shape", [(1, 8, 8, 8, 32, 48), (1, 2, 3, 128, 32, 48), (1, 2, 12, 128, 32, 32)])
@pytest.mark.parametrize("relu,out_bf16", [(True, True), (False, False), (True, False)])
def test_fused_bias_activation(require_gpu, relu, out_bf16, shape):
    """conv3d_act: y = act(conv(x, w) + b) from the epilogue (TMA form at W = 8,
    halo-block form at W = 128 with Cout 48, y-march with Cout 32), and its gradients (ReLU mask from the stored
    activation, bias = sum of dy) against torch's FP64 autograd on the CPU."""
    x, wt, dy = inputs(shape, 5)
    b = conv_ref.bf16_rounded((shape[5],), torch.Generator().manual_seed(6), 0.3)
    xd, wd, bd = x.double().requires_grad_(True), wt.double().requires_grad_(True), b.double().requires_grad_(True)
    yd = conv_ref.conv3d(xd, wd) + bd
    yd = torch.relu(yd) if relu else yd
    (yd * dy.double()).sum().backward()
    xg = x.cuda().bfloat16().requires_grad_(True)
    wg = wt.cuda().requires_grad_(True)
    bg = b.cuda().requires_grad_(True)
    y = surrogate.conv3d_act(xg, wg, bg, relu, out_bf16)
    assert y.dtype == (torch.bfloat16 if out_bf16 else torch.float32)
    bound = conv_ref.conv3d(x.abs(), wt.abs()) + b.abs().double()
    err = (y.double().cpu() - yd.detach()).abs()
    # FP32 accumulation, then (BF16 output) one rounding to 8 significant bits
    tol = 1e-4 * bound + (yd.detach().abs() * 2.0 ** -8 * 1.01 if out_bf16 else 0.0)
    assert bool((err <= tol).all())
    (y.float() * dy.cuda()).sum().backward()
    assert surrogate.conv_error() == 0
    for got, ref, name in ((wg.grad, wd.grad, "w"), (bg.grad, bd.grad, "b")):
        rel = float((got.double().cpu() - ref).abs().max() / ref.abs().max())
        assert rel < 2e-2, name   # the masked gradient is rounded to BF16 before the kernels
    rel = float((xg.grad.double().cpu() - xd.grad).abs().max() / xd.grad.abs().max())
    assert rel < 2e-2


def test_rejects_misaligned_shapes(require_gpu):
    x = torch.zeros((1, 3, 3, 3, 16), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((16, 27, 16), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(RuntimeError):
        surrogate.conv3d_raw(x, w)


def test_unet_gradients_finite_and_descend(require_gpu):
    """One U-Net on random inputs: every parameter receives a finite gradient
    from the library's kernels, and a few Adam steps reduce the loss."""
    torch.manual_seed(0)
    net = surrogate.unet(4, 16).cuda()
    x = torch.randn(2, 16, 16, 16, 4, device="cuda")
    target = torch.tanh(x.roll(1, 1)) * 0.5
    opt = torch.optim.Adam(net.parameters(), lr=2e-3)
    losses = []
    for _ in range(30):
        loss = torch.mean((net(x) - target) ** 2)
        opt.zero_grad()
        loss.backward()
        for p in net.parameters():
            assert p.grad is not None and torch.isfinite(p.grad).all()
        opt.step()
        losses.append(loss.item())
    assert losses[-1] < 0.7 * losses[0]


def _random_shapes(count, seed):
    """Seeded shapes over the forms' cases: batches, degenerate d or h of 1,
    rows below, at and above 128 voxels (not multiples of 128), channel
    counts 16..96 and Cout up to 80; voxel counts multiples of 64."""
    import random
    rnd = random.Random(seed)
    out = []
    while len(out) < count:
        n, d, h = rnd.choice([1, 2]), rnd.choice([1, 2, 3, 5]), rnd.choice([1, 2, 4, 6])
        w = rnd.choice([8, 16, 24, 64, 128, 136, 200, 256])
        ci, co = rnd.choice([16, 32, 48, 64, 96]), rnd.choice([16, 32, 48, 64, 80])
        if (n * d * h * w) % 64 == 0 and n * d * h * w <= 8192:
            out.append((n, d, h, w, ci, co))
    return out


@pytest.mark.parametrize("shape", _random_shapes(14, 11))
def test_random_shapes_every_form(require_gpu, shape):
    x, wt, dy = inputs(shape, 9)
    ref, bound = conv_ref.conv3d(x, wt), conv_ref.conv3d(x.abs(), wt.abs())
    xb, wb, dyb = x.cuda().bfloat16(), wt.cuda().bfloat16(), dy.cuda().bfloat16()
    forms = ["tcgen05", "tma", "gather"] + (["halo"] if HALO(shape) else []) + (["march"] if MARCH(shape) else [])
    for form in forms:
        within(surrogate.conv3d_raw(xb, wb, form), ref, bound, f"forward ({form}) {shape}")
    _, dw_ref = conv_ref.grads(x, wt, dy)
    _, dw_abs = conv_ref.grads(x.abs(), wt, dy.abs())
    within(surrogate.conv3d_wgrad_raw(xb, dyb), dw_ref, dw_abs, f"weight gradient {shape}")
    assert surrogate.conv_error() == 0
