"""CPU oracle of the surrogate's convolutions: torch's own conv3d in FP64 on
the library's layouts (activations NDHWC; weights [Cout][27][Cin], tap =
(dz+1)*9 + (dy+1)*3 + (dx+1))."""
import torch
import torch.nn.functional as F


def to_torch_weight(w):
    """[Cout][27][Cin] -> torch's [Cout][Cin][3][3][3] (kz, ky, kx)."""
    co, _, ci = w.shape
    return w.reshape(co, 3, 3, 3, ci).permute(0, 4, 1, 2, 3)


def conv3d(x, w):
    """y = conv(x, w), stride 1, zero padding 1, in FP64: x (n, d, h, w, cin)."""
    xt = x.double().permute(0, 4, 1, 2, 3)
    y = F.conv3d(xt, to_torch_weight(w.double()), padding=1)
    return y.permute(0, 2, 3, 4, 1)


def dgrad_weights(w):
    """w'[ci][tap][co] = w[co][26 - tap][ci]: dx = conv(dy, w')."""
    return w.flip(1).permute(2, 1, 0).contiguous()


def grads(x, w, dy):
    """(dx, dw) of sum(conv(x, w) * dy) by torch autograd in FP64."""
    xd = x.double().clone().requires_grad_(True)
    wd = w.double().clone().requires_grad_(True)
    (conv3d(xd, wd) * dy.double()).sum().backward()
    return xd.grad, wd.grad


def bf16_rounded(shape, gen, scale=1.0):
    """Seeded normal values already representable in BF16 (as FP32)."""
    return (torch.randn(shape, generator=gen) * scale).to(torch.bfloat16).float()
