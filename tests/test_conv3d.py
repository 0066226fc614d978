"""Host-side checks of the surrogate's convolution layouts (no GPU): the
weight layout maps onto torch's, the data gradient is the forward
convolution with the flipped and transposed weights, and the C-ABI checks
its shape arguments before touching memory."""
import pytest
import torch

import conv_ref


@pytest.mark.parametrize("shape", [(1, 4, 4, 4, 16, 16), (2, 3, 5, 4, 16, 32)])
def test_dgrad_is_flipped_forward(shape):
    n, d, h, w, ci, co = shape
    g = torch.Generator().manual_seed(7)
    x = conv_ref.bf16_rounded((n, d, h, w, ci), g)
    wt = conv_ref.bf16_rounded((co, 27, ci), g, 0.1)
    dy = conv_ref.bf16_rounded((n, d, h, w, co), g)
    dx, dw = conv_ref.grads(x, wt, dy)
    assert torch.allclose(conv_ref.conv3d(dy, conv_ref.dgrad_weights(wt)), dx, rtol=0, atol=1e-12)
    # dw[co][tap][ci] = sum_v dy[v][co] x[v + off(tap)][ci]
    xp = torch.nn.functional.pad(x.double(), (0, 0, 1, 1, 1, 1, 1, 1))
    for tap in (0, 4, 13, 26):
        dz, dyy, dxx = tap // 9, tap // 3 % 3, tap % 3
        xs = xp[:, dz:dz + d, dyy:dyy + h, dxx:dxx + w, :]
        ref = torch.einsum("ndhwo,ndhwi->oi", dy.double(), xs)
        assert torch.allclose(dw[:, tap, :], ref, rtol=0, atol=1e-10)


def test_tap_order():
    """tap 14 = (dz, dy, dx) = (0, 0, +1): y[v] = x[v + 1 along W]."""
    x = torch.arange(2 * 3 * 4 * 16, dtype=torch.float32).reshape(1, 2, 3, 4, 16)
    w = torch.zeros(16, 27, 16)
    w[torch.arange(16), 14, torch.arange(16)] = 1.0
    y = conv_ref.conv3d(x, w)
    assert torch.equal(y[..., :3, :], x[..., 1:, :].double())
    assert torch.equal(y[..., 3, :], torch.zeros_like(y[..., 3, :]))


def test_conv_abi_rejects_shapes():
    """Voxel counts not a multiple of 64 and channels not a multiple of 16
    are refused before any launch (no device memory is touched)."""
    import nicr
    from nicr import surrogate
    L = surrogate._lib()
    err = nicr._abi.ERR_INVALID_ARG
    for n, d, h, w, ci, co in ((1, 3, 3, 3, 16, 16), (1, 4, 4, 4, 8, 16), (1, 4, 4, 4, 16, 24), (0, 4, 4, 4, 16, 16)):
        assert L.nicr_conv3d_fwd(1, 1, 1, n, d, h, w, ci, co, None) == err
        for f in ("nicr_conv3d_fwd_mma_sync", "nicr_conv3d_fwd_tma", "nicr_conv3d_fwd_gather"):
            assert getattr(L, f)(1, 1, 1, n, d, h, w, ci, co, None) == err
        for f in ("nicr_conv3d_wgrad", "nicr_conv3d_wgrad_tma", "nicr_conv3d_wgrad_mma_sync"):
            assert getattr(L, f)(1, 1, 1, n, d, h, w, ci, co, None) == err
    assert L.nicr_conv3d_fwd(None, 1, 1, 1, 4, 4, 4, 16, 16, None) == err
    # the halo-block form: Cout <= 64 and rows of at least 128 voxels
    assert L.nicr_conv3d_fwd_halo(1, 1, None, 0, 1, 1, 4, 4, 64, 16, 16, None) == err
    assert L.nicr_conv3d_fwd_halo(1, 1, None, 0, 1, 1, 1, 1, 128, 16, 128, None) == err
    assert L.nicr_conv3d_fwd_act(1, 1, None, 4, 1, 1, 1, 1, 128, 16, 16, None) == err   # unknown act bit
    # the y-march form: Cin <= 48, Cout <= 32, rows of at least 128 voxels
    assert L.nicr_conv3d_fwd_march(1, 1, None, 0, 1, 1, 1, 1, 128, 64, 16, None) == err
    assert L.nicr_conv3d_fwd_march(1, 1, None, 0, 1, 1, 1, 1, 128, 16, 48, None) == err
    assert L.nicr_conv3d_fwd_march(1, 1, None, 0, 1, 1, 1, 4, 64, 16, 16, None) == err
