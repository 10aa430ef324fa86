"""Learned start density: the BF16 convolution kernels and the network backward against
CPU float64 torch (the checker), and the start-density contract (positive, N electrons).

Tolerances: kernels see BF16-rounded operands (the float64 reference gets the same
rounded values), so only FP32 accumulation differs: 1e-4 relative to the largest output.
The whole-network backward stores BF16 activations between layers: parameter gradients
agree with float64 autograd to 5e-2 in relative norm per layer.
"""
import numpy as np
import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _circ_conv(x, w, b, stride):
    return F.conv3d(F.pad(x, (1, 1, 1, 1, 1, 1), mode="circular"), w, b, stride=stride)


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


@pytest.mark.parametrize("stride,ci,co,d", [(1, 3, 5, 8), (2, 4, 9, 8), (1, 16, 16, 12), (2, 8, 3, 6)])
def test_conv_kernels_match_float64(stride, ci, co, d):
    from amaterasu_b200.learned import conv_bwd, conv_fwd
    g = torch.Generator().manual_seed(ci * 100 + co)
    x = torch.randn((2, ci, d, d, d), generator=g).to(torch.bfloat16)
    w = (torch.randn((co, ci, 3, 3, 3), generator=g) * 0.2).to(torch.bfloat16)
    b = torch.randn(co, generator=g)
    y = conv_fwd(x.cuda(), w.cuda(), b.cuda(), stride).cpu().double()
    xd = x.double().requires_grad_(True)
    wd = w.double().requires_grad_(True)
    bd = b.double().requires_grad_(True)
    yref = _circ_conv(xd, wd, bd, stride)
    assert _rel(y, yref.detach()) < 1e-4
    dy = torch.randn(yref.shape, generator=g)
    yref.backward(dy.double())
    dx, dw, db = conv_bwd(dy.float().cuda().contiguous(), x.cuda(), w.cuda(), stride)
    assert _rel(dx.cpu().double(), xd.grad) < 1e-4
    assert _rel(dw.cpu().double(), wd.grad) < 1e-4
    assert _rel(db.cpu().double(), bd.grad) < 1e-4


def test_silu_and_upsample_match_float64():
    from amaterasu_b200.learned import silu_bwd, silu_fwd, up_bwd, up_fwd
    g = torch.Generator().manual_seed(3)
    z = torch.randn((2, 3, 5, 5, 5), generator=g)
    a = silu_fwd(z.cuda()).cpu().double()
    assert _rel(a, F.silu(z.double())) < 1e-2  # BF16 output
    zd = z.double().requires_grad_(True)
    dy = torch.randn(z.shape, generator=g)
    F.silu(zd).backward(dy.double())
    assert _rel(silu_bwd(z.cuda(), dy.cuda()).cpu().double(), zd.grad) < 1e-5
    x = torch.randn((2, 3, 4, 4, 4), generator=g).to(torch.bfloat16)
    u = up_fwd(x.cuda()).cpu()
    ref = x.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)
    assert torch.equal(u, ref)
    du = torch.randn(u.shape, generator=g)
    dx = up_bwd(du.cuda()).cpu().double()
    ref_dx = du.double().reshape(2, 3, 4, 2, 4, 2, 4, 2).sum(dim=(3, 5, 7))
    assert _rel(dx, ref_dx) < 1e-6


def _reference_net(params, x):
    """float64 torch replica of DensityNet.forward (BF16-rounded weights)."""
    def c(name, inp, stride, act=True):
        w, b = params[name]
        y = _circ_conv(inp, w, b, stride)
        return F.silu(y) if act else y

    def up(t):
        return t.repeat_interleave(2, 2).repeat_interleave(2, 3).repeat_interleave(2, 4)

    e1 = c("e1b", c("e1a", x, 1), 1)
    e2 = c("e2b", c("e2a", e1, 2), 1)
    e3 = c("e3b", c("e3a", e2, 2), 1)
    d2 = c("d2", c("u2", up(e3), 1) + e2, 1)
    d1 = c("d1", c("u1", up(d2), 1) + e1, 1)
    return c("out", d1, 1, act=False)


def test_network_backward_matches_autograd():
    from amaterasu_b200.learned import DensityNet
    net = DensityNet(seed=1)
    g = torch.Generator().manual_seed(2)
    x = torch.randn((1, 8, 36, 36, 36), generator=g) * 0.5
    out, cache = net.forward(x.cuda(), keep=True)
    dout = torch.randn(out.shape, generator=g)
    grads = net.backward(dout.cuda().contiguous(), cache)
    params = {}
    for name, (w, b) in net.params.items():
        params[name] = (w.to(torch.bfloat16).double().cpu().requires_grad_(True), b.double().cpu().requires_grad_(True))
    ref = _reference_net(params, x.to(torch.bfloat16).double())
    assert _rel(out.cpu().double(), ref.detach()) < 5e-2
    ref.backward(dout.double())
    for name, (dw, db) in grads.items():
        rw = params[name][0].grad
        err = float((dw.cpu().double() - rw).norm() / rw.norm().clamp_min(1e-30))
        assert err < 5e-2, (name, err)


def test_learned_start_is_a_valid_density(mini_system):
    from amaterasu_b200.learned import DensityNet, LearnedStart
    s = mini_system
    ls = LearnedStart(DensityNet(seed=0), np.asarray(s.cell))
    d = ls.predict(s)
    assert not ls.stats["fallback"]
    assert d.shape == (1, *s.grid.shape)
    assert np.all(d > 0)
    np.testing.assert_allclose(d.sum() * s.grid.cell_volume_per_point, s.nelectrons, rtol=1e-12)


def test_band_limit_matches_fourier_resample(mini_system):
    """The device band limit (one grid-filter pass) equals the host same-shape Fourier
    resampling the learned start used to run (Nyquist planes of even axes removed), to
    1e-12 of the field's scale."""
    import torch
    from amaterasu_b200.learned import fourier_resample
    from amaterasu_b200.potential import grid_ops
    s = mini_system
    assert all(n % 2 == 0 for n in s.grid.shape)
    rng = np.random.default_rng(11)
    f = s.initial_density()[0] * np.exp(0.3 * rng.normal(size=s.grid.shape))
    ref = fourier_resample(f, tuple(s.grid.shape))
    got = grid_ops(s).band_limit(torch.from_numpy(f)).reshape(s.grid.shape).cpu().numpy()
    assert np.abs(got - ref).max() < 1e-12 * np.abs(ref).max()
