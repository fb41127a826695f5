"""GPU: the warm-start network's tensor-core convolutions (forward, data gradient, weight
gradient) and the whole network's gradients against torch CPU references of the same ops.

BF16 inputs are rounded identically for the references; the CUDA path accumulates in FP32 and
stores BF16 activations, so forward / data-gradient outputs agree to BF16 rounding (rel. 1e-2),
weight gradients (FP32 results) to 1e-3, and the whole-network gradients to 5e-2 relative L2
(BF16 activations at every layer).
"""

import ctypes

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
F = torch.nn.functional


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _rand(shape, rng, scale=1.0):
    return torch.from_numpy((rng.standard_normal(shape) * scale).astype(np.float32))


def _ref_conv(x_nhwc, w_oc9i, b, relu):
    """torch CPU fp64 reference: NHWC input, [cout][9][cin] weights."""
    x = x_nhwc.double().permute(0, 3, 1, 2)
    co, _, ci = w_oc9i.shape
    w = w_oc9i.double().reshape(co, 3, 3, ci).permute(0, 3, 1, 2)
    y = F.conv2d(x, w, None if b is None else b.double(), padding=1)
    if relu:
        y = F.relu(y)
    return y.permute(0, 2, 3, 1)


@pytest.mark.parametrize("b,h,w,cin,cout", [(2, 16, 16, 32, 64), (1, 24, 40, 16, 16), (3, 8, 8, 256, 128), (1, 32, 32, 64, 256)])
def test_conv_fwd_matches_torch(b, h, w, cin, cout, cuda):
    from pycorrectedemissionct_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(cin * cout + h)
    x = _rand((b, h, w, cin), rng).bfloat16()
    wt = _rand((cout, 9, cin), rng, 1 / np.sqrt(9 * cin)).bfloat16()
    bias = _rand((cout,), rng, 0.1)
    y = torch.empty((b, h, w, cout), dtype=torch.bfloat16, device=cuda)
    xd, wd, bd = x.to(cuda), wt.to(cuda), bias.to(cuda)
    d = _lib.ConvDesc(b, h, w, cin, cout)
    _lib.check(lib.cct_conv3x3_fwd(ctypes.byref(d), xd.data_ptr(), wd.data_ptr(), bd.data_ptr(), 1, y.data_ptr(), None))
    torch.cuda.synchronize()
    ref = _ref_conv(x.float(), wt.float(), bias, True)
    assert rel_l2(y.float().cpu().numpy(), ref.numpy()) < 1e-2
    v = ctypes.c_int32(0)
    _lib.check(lib.cct_net_timeout(1, ctypes.byref(v)))
    assert v.value == 0


@pytest.mark.parametrize("b,h,w,cin,cout", [(2, 16, 16, 32, 64), (1, 24, 40, 16, 16), (2, 8, 8, 128, 256)])
def test_conv_gradients_match_torch(b, h, w, cin, cout, cuda):
    from pycorrectedemissionct_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(7 * cin + cout)
    x = _rand((b, h, w, cin), rng).bfloat16()
    wt = _rand((cout, 9, cin), rng, 1 / np.sqrt(9 * cin)).bfloat16()
    dy = _rand((b, h, w, cout), rng).bfloat16()
    # torch fp64 autograd reference
    xr = x.double().permute(0, 3, 1, 2).requires_grad_(True)
    wr = wt.double().reshape(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous().requires_grad_(True)
    yr = F.conv2d(xr, wr, padding=1)
    yr.backward(dy.double().permute(0, 3, 1, 2))
    gx_ref = xr.grad.permute(0, 2, 3, 1).numpy()
    gw_ref = wr.grad.permute(0, 2, 3, 1).reshape(cout, 9, cin).numpy()
    xd, wd, dyd = x.to(cuda), wt.to(cuda), dy.to(cuda)
    gw = torch.zeros((cout, 9, cin), dtype=torch.float32, device=cuda)
    d = _lib.ConvDesc(b, h, w, cin, cout)
    _lib.check(lib.cct_conv3x3_wgrad(ctypes.byref(d), xd.data_ptr(), dyd.data_ptr(), gw.data_ptr(), None))
    wf = torch.empty((cin, 9, cout), dtype=torch.bfloat16, device=cuda)
    _lib.check(lib.cct_net_flip_weights(wd.data_ptr(), wf.data_ptr(), cin, cout, None))
    gx = torch.empty((b, h, w, cin), dtype=torch.bfloat16, device=cuda)
    dd = _lib.ConvDesc(b, h, w, cout, cin)
    _lib.check(lib.cct_conv3x3_fwd(ctypes.byref(dd), dyd.data_ptr(), wf.data_ptr(), None, 0, gx.data_ptr(), None))
    torch.cuda.synchronize()
    assert rel_l2(gw.cpu().numpy(), gw_ref) < 1e-3
    assert rel_l2(gx.float().cpu().numpy(), gx_ref) < 1e-2


def _torch_net(net, x):
    """fp64 CPU re-statement of WarmStartNet.forward with the same (bf16-rounded) weights."""
    L = net.layers

    def conv(name, t):
        l = L[name]
        w = l.w16.float().cpu().double().reshape(l.cout, 3, 3, l.cin).permute(0, 3, 1, 2)
        y = F.conv2d(t, w, l.b.cpu().double(), padding=1)
        return F.relu(y) if l.relu else y

    pool = lambda t: F.avg_pool2d(t, 2)  # noqa: E731
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")  # noqa: E731
    e1 = conv("e1b", conv("e1a", x))
    e2 = conv("e2b", conv("e2a", pool(e1)))
    e3 = conv("e3b", conv("e3a", pool(e2)))
    bt = conv("b2", conv("b1", pool(e3)))
    d3 = conv("d3b", conv("d3a", up(bt)) + e3)
    d2 = conv("d2b", conv("d2a", up(d3)) + e2)
    d1 = conv("d1b", conv("d1a", up(d2)) + e1)
    return conv("head", d1)


def test_network_gradients_against_cpu_autograd(cuda):
    from pycorrectedemissionct_b200.warmstart import WarmStartNet

    net = WarmStartNet(seed=3, device=cuda)
    net.layers["head"].w.normal_(0, 0.05)
    net.layers["head"].w16 = net.layers["head"].w.to(torch.bfloat16)
    rng = np.random.default_rng(11)
    x = _rand((2, 16, 16, 16), rng).bfloat16()
    target = _rand((2, 16, 16), rng)
    out = net.forward(x.to(cuda))
    net.zero_grad()
    loss, grad = net.mse(out, target.to(cuda))
    net.backward(grad)
    torch.cuda.synchronize()
    # reference
    layers = net.layers
    params = {}
    for k, l in layers.items():
        params[k] = l.w16.float().cpu().double().requires_grad_(True)
    xr = x.double().permute(0, 3, 1, 2)

    def bf(t):
        # round activations to bfloat16 where the CUDA path stores them (value only, identity gradient)
        return t + (t.detach().bfloat16().double() - t.detach())

    def conv(name, t):
        l = layers[name]
        w = params[name].reshape(l.cout, 3, 3, l.cin).permute(0, 3, 1, 2)
        y = F.conv2d(t, w, l.b.cpu().double(), padding=1)
        return bf(F.relu(y) if l.relu else y)

    pool = lambda t: bf(F.avg_pool2d(t, 2))  # noqa: E731
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")  # noqa: E731
    e1 = conv("e1b", conv("e1a", xr))
    e2 = conv("e2b", conv("e2a", pool(e1)))
    e3 = conv("e3b", conv("e3a", pool(e2)))
    bt = conv("b2", conv("b1", pool(e3)))
    d3 = conv("d3b", bf(conv("d3a", up(bt)) + e3))
    d2 = conv("d2b", bf(conv("d2a", up(d3)) + e2))
    d1 = conv("d1b", bf(conv("d1a", up(d2)) + e1))
    head = conv("head", d1)
    ref_loss = ((head[:, 0] - target.double()) ** 2).mean()
    ref_loss.backward()
    assert abs(float(loss.item()) - float(ref_loss.detach())) / float(ref_loss.detach()) < 2e-2
    assert rel_l2(out[..., 0].float().cpu().numpy(), head[:, 0].detach().numpy()) < 2e-2
    # gradients pass through up to 15 bf16-rounded data-gradient layers: the bound grows with depth
    for k in ("head", "d1b", "d2a", "e2a", "b1", "e1a"):
        g, r = layers[k].gw.cpu().numpy().ravel(), params[k].grad.numpy().ravel()
        cos = float(np.dot(g, r) / (np.linalg.norm(g) * np.linalg.norm(r)))
        assert rel_l2(g, r) < 0.1 and cos > 0.995, (k, rel_l2(g, r), cos)


def test_adam_and_elementwise(cuda):
    from pycorrectedemissionct_b200 import _lib

    lib = _lib.load()
    n = 1000
    rng = np.random.default_rng(5)
    p = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(cuda)
    g = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(cuda)
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    p16 = torch.empty(n, dtype=torch.bfloat16, device=cuda)
    ref = p.clone().cpu()
    _lib.check(lib.cct_net_adam(p.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), p16.data_ptr(), n, 1e-2, 0.9, 0.999, 1e-8, 1, None))
    gc = g.cpu()
    mh = 0.1 * gc / (1 - 0.9)
    vh = 0.001 * gc * gc / (1 - 0.999)
    ref = ref - 1e-2 * mh / (vh.sqrt() + 1e-8)
    torch.cuda.synchronize()
    assert rel_l2(p.cpu().numpy(), ref.numpy()) < 1e-6
    # pooling / upsampling adjoint pairs: <pool x, y> == <x, pool^T y>
    x = torch.from_numpy(rng.standard_normal((2, 8, 8, 16)).astype(np.float32)).bfloat16().to(cuda)
    y = torch.from_numpy(rng.standard_normal((2, 4, 4, 16)).astype(np.float32)).bfloat16().to(cuda)
    px = torch.empty_like(y)
    pty = torch.empty_like(x)
    _lib.check(lib.cct_net_avgpool2(x.data_ptr(), px.data_ptr(), 2, 8, 8, 16, 0, None))
    _lib.check(lib.cct_net_avgpool2(y.data_ptr(), pty.data_ptr(), 2, 8, 8, 16, 1, None))
    ux = torch.empty_like(x)
    uty = torch.empty_like(y)
    _lib.check(lib.cct_net_upsample2(y.data_ptr(), ux.data_ptr(), 2, 4, 4, 16, 0, None))
    _lib.check(lib.cct_net_upsample2(x.data_ptr(), uty.data_ptr(), 2, 4, 4, 16, 1, None))
    torch.cuda.synchronize()
    a1 = float((px.double() * y.double()).sum()); a2 = float((x.double() * pty.double()).sum())
    assert abs(a1 - a2) < 2e-2 * (abs(a1) + 1)
    b1 = float((ux.double() * x.double()).sum()); b2 = float((y.double() * uty.double()).sum())
    assert abs(b1 - b2) < 2e-2 * (abs(b1) + 1)
