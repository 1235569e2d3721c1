"""Learned warm start: the tcgen05 convolution kernels and the U-Net built on
them, checked against plain PyTorch on the CPU (float64) with the same
BF16-rounded inputs and weights."""
import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")


def _padded(x):
    """dense (nb, C, d, h, w) -> padded channels-last (rows, C) BF16 on the GPU"""
    nb, c, d, h, w = x.shape
    p = torch.zeros(nb, d + 2, h + 2, w + 2, c, dtype=torch.bfloat16)
    p[:, 1:-1, 1:-1, 1:-1] = x.permute(0, 2, 3, 4, 1).to(torch.bfloat16)
    return p.reshape(-1, c).cuda()


def _dense(p, nb, d, h, w):
    c = p.shape[1]
    return p.reshape(nb, d + 2, h + 2, w + 2, c)[:, 1:-1, 1:-1, 1:-1].permute(0, 4, 1, 2, 3).double().cpu()


def _bf(x):
    return x.to(torch.bfloat16).double()


def _conv_ref(x, w, b=None):
    """x (nb, cin, d, h, w) float64, w (cout, 27, cin)"""
    import torch.nn.functional as F
    co, _, cin = w.shape
    return F.conv3d(x, w.permute(0, 2, 1).reshape(co, cin, 3, 3, 3), b, padding=1)


@pytest.mark.gpu
@pytest.mark.parametrize("c1,c2,co", [(16, 0, 16), (16, 32, 48), (64, 0, 64), (32, 16, 96)])
def test_conv3_forward(lib, c1, c2, co):
    from yoricktrtt_b200._lib import check
    from yoricktrtt_b200.unet import _p, _stream
    g = torch.Generator().manual_seed(c1 + c2 + co)
    nb, d, h, w = 2, 6, 10, 20
    x1 = _bf(torch.randn(nb, c1, d, h, w, generator=g))
    x2 = _bf(torch.randn(nb, c2, d, h, w, generator=g)) if c2 else None
    cin = c1 + c2
    wt = torch.randn(co, 27, cin, generator=g) / np.sqrt(27 * cin)
    bias = torch.randn(co, generator=g)
    pack = torch.empty(27 * co * cin, dtype=torch.bfloat16, device="cuda")
    check(lib.trtt_b200_conv3_pack(_p(wt.cuda()), co, cin, 0, _p(pack), _stream()), "pack")
    xp1, xp2 = _padded(x1), (_padded(x2) if c2 else None)
    rows = xp1.shape[0]
    ref = _conv_ref(torch.cat([x1, x2], 1) if c2 else x1, _bf(wt), bias.double())
    # FP32 output, identity activation
    y = torch.zeros(rows, co, dtype=torch.float32, device="cuda")
    check(lib.trtt_b200_conv3_forward(_p(xp1), c1, _p(xp2), c2, _p(pack), co, _p(bias.cuda()), 1, 1.0,
                                      _p(y), None, 0, 0, None, nb, d, h, w, _stream()), "conv")
    check(lib.trtt_b200_unet_status(_stream()), "status")
    yd = y.reshape(nb, d + 2, h + 2, w + 2, co)
    assert float(yd[:, 0].abs().max()) == 0.0 and float(yd[:, :, :, 0].abs().max()) == 0.0  # border untouched
    got = yd[:, 1:-1, 1:-1, 1:-1].permute(0, 4, 1, 2, 3).double().cpu()
    assert rel_l2(got.numpy(), ref.numpy()) <= 1e-5
    # BF16 output with leaky ReLU
    yb = torch.zeros(rows, co, dtype=torch.bfloat16, device="cuda")
    check(lib.trtt_b200_conv3_forward(_p(xp1), c1, _p(xp2), c2, _p(pack), co, _p(bias.cuda()), 0, 0.1,
                                      _p(yb), None, 0, 0, None, nb, d, h, w, _stream()), "conv")
    refa = torch.nn.functional.leaky_relu(ref, 0.1)
    assert rel_l2(_dense(yb, nb, d, h, w).numpy(), refa.numpy()) <= 4e-3


@pytest.mark.gpu
@pytest.mark.parametrize("tma", [-1, 0])
@pytest.mark.parametrize("c1,c2,co", [(16, 0, 16), (32, 16, 16), (64, 32, 32), (32, 0, 64)])
def test_conv3_gradients(lib, c1, c2, co, tma):
    """Input gradient (transposed-flipped weights, split into the two input
    tensors, accumulate) and weight/bias gradients against autograd, with
    the default TMA staging and with cp.async staging (set_tma(0))."""
    try:
        lib.trtt_b200_conv3_set_tma(tma)
        _conv3_gradients(lib, c1, c2, co)
    finally:
        lib.trtt_b200_conv3_set_tma(-1)


def _conv3_gradients(lib, c1, c2, co):
    from yoricktrtt_b200._lib import check
    from yoricktrtt_b200.unet import _p, _stream
    g = torch.Generator().manual_seed(7 * co + c1)
    nb, d, h, w = 2, 4, 6, 12
    cin = c1 + c2
    x = _bf(torch.randn(nb, cin, d, h, w, generator=g)).requires_grad_(True)
    wt = _bf(torch.randn(co, 27, cin, generator=g) / np.sqrt(27 * cin)).requires_grad_(True)
    b = torch.zeros(co, dtype=torch.float64, requires_grad=True)
    gy = _bf(torch.randn(nb, co, d, h, w, generator=g))
    (_conv_ref(x, wt, b) * gy).sum().backward()
    pack = torch.empty(27 * cin * co, dtype=torch.bfloat16, device="cuda")
    check(lib.trtt_b200_conv3_pack(_p(wt.detach().float().cuda()), co, cin, 1, _p(pack), _stream()), "pack")
    gyp = _padded(gy)
    g1 = _padded(torch.ones(nb, c1, d, h, w))  # accumulate onto ones
    g2 = _padded(torch.zeros(nb, c2, d, h, w)) if c2 else None
    check(lib.trtt_b200_conv3_forward(_p(gyp), co, None, 0, _p(pack), cin, None, 3, 1.0, _p(g1), _p(g2), c1,
                                      1, None, nb, d, h, w, _stream()), "dx")
    dx = _dense(g1, nb, d, h, w) - 1.0
    if c2:
        dx = torch.cat([dx, _dense(g2, nb, d, h, w)], 1)
    assert rel_l2(dx.numpy(), x.grad.numpy()) <= 1e-2  # BF16 result
    xp1 = _padded(x.detach()[:, :c1])
    xp2 = _padded(x.detach()[:, c1:]) if c2 else None
    need = lib.trtt_b200_conv3_wgrad_scratch(co, cin, nb, d, h, w)
    scratch = torch.empty(need // 4 + 1, dtype=torch.float32, device="cuda")
    dw = torch.zeros(co, 27, cin, device="cuda")
    db = torch.zeros(co, device="cuda")
    check(lib.trtt_b200_conv3_wgrad(_p(gyp), co, _p(xp1), c1, _p(xp2), c2, _p(dw), _p(db), _p(scratch),
                                    scratch.numel() * 4, nb, d, h, w, _stream()), "wgrad")
    check(lib.trtt_b200_unet_status(_stream()), "status")
    assert rel_l2(dw.double().cpu().numpy(), wt.grad.numpy()) <= 1e-5
    assert rel_l2(db.double().cpu().numpy(), b.grad.numpy()) <= 1e-5


@pytest.mark.gpu
def test_resample_ops(lib):
    import torch.nn.functional as F
    from yoricktrtt_b200._lib import check
    from yoricktrtt_b200.unet import _p, _stream
    g = torch.Generator().manual_seed(3)
    nb, c, d, h, w = 2, 16, 4, 6, 8
    fine = _bf(torch.randn(nb, c, d, h, w, generator=g))
    coarse = _bf(torch.randn(nb, c, d // 2, h // 2, w // 2, generator=g))
    fp, cp = _padded(fine), _padded(coarse)
    out_c = _padded(torch.zeros_like(coarse))
    check(lib.trtt_b200_unet_resample(_p(fp), _p(out_c), c, nb, d, h, w, 0, 0, _stream()), "pool")
    assert rel_l2(_dense(out_c, nb, d // 2, h // 2, w // 2).numpy(), F.avg_pool3d(fine, 2).numpy()) <= 4e-3
    out_f = _padded(torch.zeros_like(fine))
    check(lib.trtt_b200_unet_resample(_p(out_f), _p(cp), c, nb, d, h, w, 2, 0, _stream()), "up")
    up = F.interpolate(coarse, scale_factor=2, mode="nearest")
    assert rel_l2(_dense(out_f, nb, d, h, w).numpy(), up.numpy()) == 0.0
    # adjoints: <pool f, c> = <f, pool^T c>, <up c, f> = <c, up^T f>
    pt = _padded(torch.zeros_like(fine))
    check(lib.trtt_b200_unet_resample(_p(pt), _p(cp), c, nb, d, h, w, 1, 0, _stream()), "pool^T")
    assert rel_l2(_dense(pt, nb, d, h, w).numpy(), (up / 8).numpy()) <= 4e-3
    ut = _padded(torch.zeros_like(coarse))
    check(lib.trtt_b200_unet_resample(_p(fp), _p(ut), c, nb, d, h, w, 3, 0, _stream()), "up^T")
    assert rel_l2(_dense(ut, nb, d // 2, h // 2, w // 2).numpy(), (8 * F.avg_pool3d(fine, 2)).numpy()) <= 4e-3


def _random_net(seed=0):
    from yoricktrtt_b200.unet import UNet3D
    net = UNet3D(scale=1.0, seed=seed)
    g = torch.Generator().manual_seed(seed + 100)
    for name, p in net.params.items():
        w = p["w"]
        if name == "head":
            w[:1].copy_((torch.randn(1, 27, 16, generator=g) * 0.05).cuda())
        p["b"].copy_((torch.randn(p["b"].shape, generator=g) * 0.05).cuda())
        if name == "head":
            p["b"][1:] = 0
        if name == "e1a":
            p["w"][:, :, 1:] = 0
    net._pack_all()
    return net


@pytest.mark.gpu
def test_unet_forward_and_gradients_match_cpu(lib):
    """The whole network: output and every parameter gradient against
    autograd of the float64 CPU restatement (BF16 activations on the GPU)."""
    net = _random_net()
    g = torch.Generator().manual_seed(5)
    nb, d, h, w = 2, 8, 12, 16
    x = torch.rand(nb, d, h, w, generator=g)
    t = torch.rand(nb, d, h, w, generator=g)
    y = net.forward(x.cuda())
    net.status()
    ref = net.torch_reference(x)
    assert rel_l2(y.double().cpu().numpy(), ref.numpy()) <= 2e-2
    loss = float(net.backward(x.cuda(), t.cuda()))
    net.status()
    # autograd reference
    params = {}
    for name, p in net.params.items():
        params[name] = (p["w"].detach().cpu().double().requires_grad_(True),
                        p["b"].detach().cpu().double().requires_grad_(True))
    import torch.nn.functional as F
    from yoricktrtt_b200.unet import SLOPE

    def conv(name, tt, act=True):
        wt, bt = params[name]
        co, _, cin = wt.shape
        yy = F.conv3d(tt, wt.permute(0, 2, 1).reshape(co, cin, 3, 3, 3), bt, padding=1)
        return F.leaky_relu(yy, SLOPE) if act else yy

    xin = torch.zeros(nb, 16, d, h, w, dtype=torch.float64)
    xin[:, 0] = x.double()
    e1b = conv("e1b", conv("e1a", xin))
    e2b = conv("e2b", conv("e2a", F.avg_pool3d(e1b, 2)))
    e3b = conv("e3b", conv("e3a", F.avg_pool3d(e2b, 2)))
    d2b = conv("d2b", conv("d2a", torch.cat([F.interpolate(e3b, scale_factor=2), e2b], 1)))
    d1b = conv("d1b", conv("d1a", torch.cat([F.interpolate(d2b, scale_factor=2), e1b], 1)))
    out = x.double() + conv("head", d1b, act=False)[:, 0]
    lref = ((out - t.double()) ** 2).mean()
    lref.backward()
    assert abs(loss - float(lref.detach())) <= 2e-2 * float(lref.detach())
    for name in net.params:
        gw = net._grads[name]["w"].double().cpu()
        gb = net._grads[name]["b"].double().cpu()
        rw, rb = params[name][0].grad, params[name][1].grad
        if name == "e1a":
            gw, rw = gw[:, :, :1], rw[:, :, :1]
        if name == "head":
            gw, rw, gb, rb = gw[:1], rw[:1], gb[:1], rb[:1]
        assert rel_l2(gw.numpy(), rw.numpy()) <= 5e-2, name
        assert rel_l2(gb.numpy(), rb.numpy()) <= 5e-2, name


@pytest.mark.gpu
def test_unet_training_reduces_loss(lib):
    """Adam steps on one fixed pair lower the loss (smoke test of the
    training loop on the tensor-core kernels): the target is the input
    plus a smooth offset field."""
    from yoricktrtt_b200.unet import UNet3D
    g = torch.Generator().manual_seed(11)
    x = torch.rand(1, 16, 16, 16, generator=g)
    zz = torch.linspace(0, 1, 16)
    t = (x + 0.2 + 0.1 * zz[None, :, None, None]).contiguous()
    net = UNet3D(scale=1.0, seed=1, lr=2e-3)
    losses = [float(net.train_step(x.cuda(), t.cuda())) for _ in range(150)]
    net.status()
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.3 * losses[0]


@pytest.mark.gpu
@pytest.mark.parametrize("c1,c2,co,dims", [(16, 0, 16, (2, 6, 10, 20)), (16, 32, 48, (1, 8, 12, 40)),
                                           (64, 0, 64, (1, 4, 6, 130)), (32, 16, 96, (2, 6, 10, 20))])
def test_conv3_forward_tma_staging(lib, c1, c2, co, dims):
    """TMA staging with a producer thread and an MMA thread on an mbarrier
    ring, one tile per CTA (trtt_b200_conv3_set_tma(1)) or persistent CTAs
    with two tensor-memory accumulators and epilogue warps (2), gives the
    same outputs as the cp.async staging: the same MMAs in the same order.
    The widths cover a slab of one partial TMA box (w = 20), of several
    boxes (w = 130: 518 rows, two full boxes of 256 and one of 6); 96
    output channels take the whole tensor memory (2 x 2 x 96 columns)."""
    from yoricktrtt_b200._lib import check
    from yoricktrtt_b200.unet import _p, _stream
    g = torch.Generator().manual_seed(c1 + 3 * c2 + co)
    nb, d, h, w = dims
    x1 = _bf(torch.randn(nb, c1, d, h, w, generator=g))
    x2 = _bf(torch.randn(nb, c2, d, h, w, generator=g)) if c2 else None
    cin = c1 + c2
    wt = torch.randn(co, 27, cin, generator=g) / np.sqrt(27 * cin)
    bias = torch.randn(co, generator=g).cuda()
    pack = torch.empty(27 * co * cin, dtype=torch.bfloat16, device="cuda")
    check(lib.trtt_b200_conv3_pack(_p(wt.cuda()), co, cin, 0, _p(pack), _stream()), "pack")
    xp1, xp2 = _padded(x1), (_padded(x2) if c2 else None)
    rows = xp1.shape[0]
    outs = []
    try:
        for tma in (0, 1, 2):
            check(lib.trtt_b200_conv3_set_tma(tma), "set_tma")
            y = torch.zeros(rows, co, dtype=torch.float32, device="cuda")
            check(lib.trtt_b200_conv3_forward(_p(xp1), c1, _p(xp2), c2, _p(pack), co, _p(bias), 1, 1.0,
                                              _p(y), None, 0, 0, None, nb, d, h, w, _stream()), "conv")
            yb = torch.zeros(rows, co, dtype=torch.bfloat16, device="cuda")
            check(lib.trtt_b200_conv3_forward(_p(xp1), c1, _p(xp2), c2, _p(pack), co, _p(bias), 0, 0.1,
                                              _p(yb), None, 0, 0, None, nb, d, h, w, _stream()), "conv")
            check(lib.trtt_b200_unet_status(_stream()), "status")
            outs.append((y.cpu(), yb.cpu()))
    finally:
        lib.trtt_b200_conv3_set_tma(-1)
    for o in outs[1:]:
        assert torch.equal(outs[0][0], o[0])
        assert torch.equal(outs[0][1], o[1])
    ref = _conv_ref(torch.cat([x1, x2], 1) if c2 else x1, _bf(wt), bias.double().cpu())
    got = outs[1][0].reshape(nb, d + 2, h + 2, w + 2, co)[:, 1:-1, 1:-1, 1:-1].permute(0, 4, 1, 2, 3).double()
    assert rel_l2(got.numpy(), ref.numpy()) <= 1e-5


@pytest.mark.gpu
def test_unet_training_step_tma_staging():
    """A U-Net forward and backward (input gradients run the same kernel)
    with TMA staging: the same forward output as the cp.async staging, the
    same loss and gradients to summation order."""
    from yoricktrtt_b200 import _lib
    from yoricktrtt_b200.unet import UNet3D
    lib = _lib.load()
    x = torch.rand(1, 32, 32, 32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    t = torch.rand(1, 32, 32, 32, device="cuda", generator=torch.Generator(device="cuda").manual_seed(2))
    res = []
    try:
        for tma in (0, 1, 2):
            _lib.check(lib.trtt_b200_conv3_set_tma(tma), "set_tma")
            net = UNet3D(seed=3)
            y = net.forward(x).clone()
            loss = net.backward(x, t)
            net.status()
            res.append((y.cpu(), float(loss),
                        {(k, n): g.clone().cpu() for k, v in net._grads.items() for n, g in v.items()}))
    finally:
        lib.trtt_b200_conv3_set_tma(-1)
    for r in res[1:]:
        assert torch.equal(res[0][0], r[0])
        # the loss and the bias gradients are sums with float atomics: equal
        # to FP32 summation order
        assert abs(res[0][1] - r[1]) <= 1e-6 * abs(res[0][1])
        for key, g0 in res[0][2].items():
            assert rel_l2(r[2][key].double().numpy(), g0.double().numpy()) <= 1e-5, key
