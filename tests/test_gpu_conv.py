"""Learned-denoiser kernels against plain PyTorch fp32 references on the
same bf16-rounded operands: 3x3 convolution forward, input gradient and
weight / bias gradients (tolerance 2 % of the reference's largest value,
the bf16 rounding of the outputs), pool / upsample and their gradients,
the whole network's loss and weight gradients, and a short training run."""
import ctypes

import numpy as np
import pytest

import roxy_native as nat

torch = pytest.importorskip("torch")
F = torch.nn.functional
pytestmark = pytest.mark.gpu


def _ctx():
    return nat.context()


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    # torch's default stream (handle 0) is the legacy default stream, handle 1
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or 1)


def _close(got, ref, frac=2e-2):
    ref = ref.detach()
    scale = float(ref.abs().max()) + 1e-6
    err = float((got.float() - ref.float()).abs().max())
    assert err <= frac * scale, (err, scale)


def _view(t, off, c):
    return t[..., off:off + c]


CASES = [  # N, H, W, Cin, Cout, x_stride, x_off, y_stride, y_off, relu
    (1, 8, 8, 16, 32, 16, 0, 32, 0, 1),
    (2, 17, 23, 32, 64, 48, 16, 64, 0, 0),
    (1, 12, 20, 64, 128, 64, 0, 160, 32, 1),
    (1, 9, 31, 192, 64, 192, 0, 96, 32, 1),
    (2, 16, 16, 96, 16, 96, 0, 16, 0, 0),
    (1, 40, 36, 128, 128, 128, 0, 128, 0, 1),
]


@pytest.fixture(params=[0, 1, 2], ids=["tcgen05", "mma_sync", "tcgen05_streaming"])
def impl(request):
    ctx = _ctx()
    ctx.check(nat.lib().rx_conv_set_impl(ctx.h, request.param))
    yield request.param
    ctx.check(nat.lib().rx_ctx_sync(ctx.h))  # no kernel raised its error flag
    ctx.check(nat.lib().rx_conv_set_impl(ctx.h, 0))


@pytest.mark.parametrize("N,H,W,Cin,Cout,xs,xo,ys,yo,relu", CASES + [(1, 3, 300, 32, 64, 32, 0, 64, 0, 1)])
def test_conv_fwd_and_grads_match_torch(N, H, W, Cin, Cout, xs, xo, ys, yo, relu, impl):
    ctx = _ctx()
    g = torch.Generator(device="cuda").manual_seed(N * 1000 + H)
    dev = "cuda"
    xbuf = torch.randn((N, H, W, xs), generator=g, device=dev).to(torch.bfloat16)
    w = (torch.randn((Cout, 9, Cin), generator=g, device=dev) * (1.0 / np.sqrt(9 * Cin))).to(torch.bfloat16)
    bias = torch.randn(Cout, generator=g, device=dev) * 0.1
    ybuf = torch.zeros((N, H, W, ys), dtype=torch.bfloat16, device=dev)
    d = nat.ConvDesc(N, H, W, Cin, Cout, xs, xo, ys, yo)
    L = nat.lib()
    ctx.check(L.rx_conv_bf16_fwd(ctx.h, ctypes.byref(d), _p(xbuf), _p(w), _p(bias), _p(ybuf), None, relu, _stream()))
    xin = _view(xbuf, xo, Cin).float().permute(0, 3, 1, 2).contiguous().requires_grad_(True)
    wt = w.float().view(Cout, 3, 3, Cin).permute(0, 3, 1, 2).contiguous().requires_grad_(True)
    bt = bias.clone().requires_grad_(True)
    ref = F.conv2d(xin, wt, bt, padding=1)
    if relu:
        ref = F.relu(ref)
    got = _view(ybuf, yo, Cout).float().permute(0, 3, 1, 2)
    torch.cuda.synchronize()
    _close(got, ref)
    # untouched channels of the output view stay zero
    if ys > Cout:
        mask = torch.ones(ys, dtype=torch.bool, device=dev)
        mask[yo:yo + Cout] = False
        assert float(ybuf[..., mask].float().abs().max()) == 0.0
    # gradients for a random output gradient
    dyv = torch.randn((N, H, W, Cout), generator=g, device=dev).to(torch.bfloat16)
    dybuf = torch.zeros((N, H, W, ys), dtype=torch.bfloat16, device=dev)
    dybuf[..., yo:yo + Cout] = dyv
    ref.backward(dyv.float().permute(0, 3, 1, 2))
    dxbuf = torch.zeros((N, H, W, xs), dtype=torch.bfloat16, device=dev)
    rot = torch.empty(Cout * 9 * Cin, dtype=torch.bfloat16, device=dev)
    dw = torch.zeros((Cout, 9, Cin), dtype=torch.float32, device=dev)
    db = torch.zeros(Cout, dtype=torch.float32, device=dev)
    if relu:
        # the kernels take the gradient after the ReLU mask
        op = nat.DnOp(nat.RX_DN_RELU_MASK, N, H, W, Cout, _p(ybuf), ys, yo, _p(dybuf), ys, yo, 0)
        ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(op), _stream()))
    ctx.check(L.rx_conv_bf16_bwd_data(ctx.h, ctypes.byref(d), _p(dybuf), _p(w), _p(rot), _p(dxbuf), _stream()))
    ctx.check(L.rx_conv_bf16_bwd_weight(ctx.h, ctypes.byref(d), _p(dybuf), _p(xbuf), _p(dw), _p(db), _stream()))
    torch.cuda.synchronize()
    _close(_view(dxbuf, xo, Cin).float().permute(0, 3, 1, 2), xin.grad, 3e-2)
    _close(dw.view(Cout, 3, 3, Cin).permute(0, 3, 1, 2), wt.grad, 2e-2)
    _close(db, bt.grad, 2e-2)


def test_conv_rejects_bad_descriptors():
    ctx = _ctx()
    x = torch.zeros((1, 4, 4, 16), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((16, 9, 16), dtype=torch.bfloat16, device="cuda")
    for d in (nat.ConvDesc(1, 4, 4, 12, 16, 16, 0, 16, 0), nat.ConvDesc(1, 4, 4, 16, 16, 16, 4, 16, 0),
              nat.ConvDesc(1, 4, 4, 16, 16, 16, 0, 8, 0)):
        with pytest.raises(ValueError):
            ctx.check(nat.lib().rx_conv_bf16_fwd(ctx.h, ctypes.byref(d), _p(x), _p(w), None, _p(x), None, 0, None))


def test_pool_and_upsample_match_torch():
    ctx = _ctx()
    L = nat.lib()
    N, H, W, C = 2, 12, 20, 32
    x = torch.randn((N, H, W, C), device="cuda").to(torch.bfloat16)
    p = torch.zeros((N, H // 2, W // 2, C), dtype=torch.bfloat16, device="cuda")
    ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_POOL, N, H, W, C, _p(x), C, 0, _p(p), C, 0, 0)),
                            _stream()))
    u = torch.zeros((N, 2 * H, 2 * W, C), dtype=torch.bfloat16, device="cuda")
    ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_UP, N, H, W, C, _p(x), C, 0, _p(u), C, 0, 0)),
                            _stream()))
    xt = x.float().permute(0, 3, 1, 2)
    _close(p.float().permute(0, 3, 1, 2), F.avg_pool2d(xt, 2), 1e-2)
    _close(u.float().permute(0, 3, 1, 2), F.interpolate(xt, scale_factor=2, mode="nearest"), 1e-6)
    # channel views (16-byte chunk kernels) and a stride that is not a
    # multiple of 8 channels (element kernels): the same values
    for stride, off in ((48, 16), (36, 4)):
        wide = torch.zeros((N, H, W, stride), dtype=torch.bfloat16, device="cuda")
        wide[..., off:off + C] = x
        pv = torch.zeros((N, H // 2, W // 2, stride), dtype=torch.bfloat16, device="cuda")
        uv = torch.zeros((N, 2 * H, 2 * W, stride), dtype=torch.bfloat16, device="cuda")
        ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_POOL, N, H, W, C, _p(wide), stride, off,
                                                             _p(pv), stride, off, 0)), _stream()))
        ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_UP, N, H, W, C, _p(wide), stride, off,
                                                             _p(uv), stride, off, 0)), _stream()))
        torch.cuda.synchronize()
        assert torch.equal(pv[..., off:off + C], p) and torch.equal(uv[..., off:off + C], u), (stride, off)
        assert not pv[..., :off].any() and not uv[..., off + C:].any()
    # gradients
    gp = torch.randn((N, H // 2, W // 2, C), device="cuda").to(torch.bfloat16)
    gx = torch.zeros_like(x)
    ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_POOL_BWD, N, H, W, C, _p(gp), C, 0, _p(gx), C, 0,
                                                         0)), _stream()))
    xr = xt.clone().requires_grad_(True)
    F.avg_pool2d(xr, 2).backward(gp.float().permute(0, 3, 1, 2))
    _close(gx.float().permute(0, 3, 1, 2), xr.grad, 1e-2)
    gu = torch.randn((N, 2 * H, 2 * W, C), device="cuda").to(torch.bfloat16)
    gx2 = torch.zeros_like(x)
    ctx.check(L.rx_dn_layer(ctx.h, ctypes.byref(nat.DnOp(nat.RX_DN_UP_BWD, N, H, W, C, _p(gu), C, 0, _p(gx2), C, 0,
                                                         0)), _stream()))
    xr2 = xt.clone().requires_grad_(True)
    F.interpolate(xr2, scale_factor=2, mode="nearest").backward(gu.float().permute(0, 3, 1, 2))
    torch.cuda.synchronize()
    _close(gx2.float().permute(0, 3, 1, 2), xr2.grad, 1e-2)


def _torch_net(net, x16, base, target):
    """fp32 PyTorch replica of the network on the same bf16 weights."""
    from rendering.learned_denoiser import LAYERS
    params = {}
    for name, cin, cout, _ in LAYERS:
        w = net.w16[name].float().view(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous().requires_grad_(True)
        b = net.b32[name].clone().requires_grad_(True)
        params[name] = (w, b)

    def conv(name, t, relu=True):
        w, b = params[name]
        y = F.conv2d(t, w, b, padding=1)
        return F.relu(y) if relu else y

    x = x16.float().permute(0, 3, 1, 2)
    s1 = conv("e1b", conv("e1a", x))
    s2 = conv("e2b", conv("e2a", F.avg_pool2d(s1, 2)))
    e3 = conv("e3b", conv("e3a", F.avg_pool2d(s2, 2)))
    d2 = conv("d2b", conv("d2a", torch.cat([F.interpolate(e3, scale_factor=2), s2], 1)))
    d1 = conv("d1b", conv("d1a", torch.cat([F.interpolate(d2, scale_factor=2), s1], 1)))
    out = conv("head", d1, relu=False)[:, :3].permute(0, 2, 3, 1)
    loss = (out + base - target).abs().sum()
    P = x.shape[0] * x.shape[2] * x.shape[3]
    (loss / (3 * P)).backward()
    return float(loss.detach()), {k: (v[0].grad, v[1].grad) for k, v in params.items()}


def test_tcgen05_and_mma_sync_convolutions_agree():
    """The forward kernels on the same operands (persistent and streaming
    tcgen05, then mma.sync): same values up to the order of their float32
    sums (and the bf16 rounding of the output)."""
    ctx = _ctx()
    L = nat.lib()
    g = torch.Generator(device="cuda").manual_seed(21)
    for (Cin, Cout, H, W) in ((16, 32, 33, 257), (96, 32, 20, 128), (64, 128, 9, 200), (32, 16, 5, 130),
                              (64, 64, 70, 300), (192, 64, 6, 129), (32, 32, 128, 512), (96, 32, 600, 256),
                              (96, 64, 20, 140), (128, 128, 12, 140)):
        x = torch.randn((2, H, W, Cin), generator=g, device="cuda").to(torch.bfloat16)
        w = (torch.randn((Cout, 9, Cin), generator=g, device="cuda") / np.sqrt(9 * Cin)).to(torch.bfloat16)
        b = torch.randn(Cout, generator=g, device="cuda")
        d = nat.ConvDesc(2, H, W, Cin, Cout, Cin, 0, Cout, 0)
        outs = []
        for impl_ in (0, 2, 1):
            ctx.check(L.rx_conv_set_impl(ctx.h, impl_))
            y = torch.zeros((2, H, W, Cout), dtype=torch.bfloat16, device="cuda")
            y32 = torch.zeros((2, H, W, Cout), dtype=torch.float32, device="cuda")
            ctx.check(L.rx_conv_bf16_fwd(ctx.h, ctypes.byref(d), _p(x), _p(w), _p(b), _p(y), _p(y32), 0, _stream()))
            outs.append(y32)
        ctx.check(L.rx_conv_set_impl(ctx.h, 0))
        ctx.check(L.rx_ctx_sync(ctx.h))
        scale = float(outs[2].abs().max())
        assert float((outs[0] - outs[2]).abs().max()) <= 1e-3 * scale, (Cin, Cout)
        assert float((outs[1] - outs[2]).abs().max()) <= 1e-3 * scale, (Cin, Cout)


def test_network_loss_and_gradients_match_torch():
    from rendering.learned_denoiser import LAYERS, Denoiser
    net = Denoiser(seed=3)
    N, H, W = 2, 16, 24
    g = torch.Generator(device="cuda").manual_seed(7)
    rad = torch.rand((N, H, W, 3), generator=g, device="cuda") * 2
    alb = torch.rand((N, H, W, 3), generator=g, device="cuda")
    nrm = torch.randn((N, H, W, 3), generator=g, device="cuda")
    dep = torch.rand((N, H, W, 1), generator=g, device="cuda") * 3
    target = torch.log1p(rad * 0.8 + 0.1)
    net.features(rad, alb, nrm, dep, N, H, W, train=True)
    b = net.forward(N, H, W, train=True)
    loss = float(net.loss(N, H, W, target))
    net.backward(N, H, W)
    torch.cuda.synchronize()
    ref_loss, grads = _torch_net(net, b["x"], b["base"], target)
    assert abs(loss - ref_loss) <= 2e-2 * abs(ref_loss)
    for name, cin, cout, _ in LAYERS:
        gw = net.dw[name].view(cout, 3, 3, cin).permute(0, 3, 1, 2).flatten()
        rw = grads[name][0].flatten()
        cos = float(torch.dot(gw, rw) / (gw.norm() * rw.norm() + 1e-20))
        assert cos > 0.98, (name, cos)
        cb = float(torch.dot(net.db[name], grads[name][1]) / (net.db[name].norm() * grads[name][1].norm() + 1e-20))
        assert cb > 0.98 or float(grads[name][1].norm()) < 1e-6, (name, cb)


def test_training_reduces_the_loss():
    from rendering.learned_denoiser import Denoiser
    net = Denoiser(seed=1)
    N, H, W = 4, 32, 32
    g = torch.Generator(device="cuda").manual_seed(11)
    clean = torch.rand((N, H, W, 3), generator=g, device="cuda")
    clean = F.avg_pool2d(clean.permute(0, 3, 1, 2), 5, 1, 2).permute(0, 2, 3, 1).contiguous()
    noisy = (clean * (1 + 0.6 * torch.randn((N, H, W, 3), generator=g, device="cuda"))).clamp_min(0)
    alb = torch.ones((N, H, W, 3), device="cuda") * 0.5
    nrm = torch.zeros((N, H, W, 3), device="cuda")
    dep = torch.ones((N, H, W, 1), device="cuda")
    target = torch.log1p(clean)
    losses = [float(net.train_step(noisy, alb, nrm, dep, target, lr=3e-3)) for _ in range(60)]
    assert np.mean(losses[-10:]) < 0.7 * np.mean(losses[:5]), (losses[:5], losses[-10:])
    out = net.denoise(noisy, alb, nrm, dep)
    assert out.shape == (N, H, W, 3) and bool(torch.isfinite(out).all())
