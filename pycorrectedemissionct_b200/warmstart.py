"""Learned warm start for MLEM: a small convolutional encoder-decoder on the tensor cores.

No reference counterpart.  The reference's MLEM accepts an initial solution ``x0``
(``corrct``: ``src/corrct/solvers.py:747-752``); this module predicts one from the first
MLEM iterates, and the plain MLEM then finishes to the same data-residual tolerance, so the
plain solver stays both the fallback and the judge of the network's error.

Network (about 1.76 M parameters, BF16 weights and activations, FP32 accumulation):

    in (16 ch: 10 MLEM iterates + normalised back-projection, zero padded)
    enc1 2 x conv3x3 -> 32   @ H      enc2 2 x conv -> 64  @ H/2
    enc3 2 x conv -> 128 @ H/4        bottleneck 2 x conv -> 256 @ H/8
    dec3 up, conv -> 128, + enc3, conv   dec2 up, conv -> 64, + enc2, conv
    dec1 up, conv -> 32, + enc1, conv    head conv -> 16 (channel 0 = correction)

All ReLU except the head; 2x2 average pooling down, nearest upsampling up, additive skips.
The prediction is ``x0 = max(x10 + scale * head[0], eps)`` with ``scale`` the slice's mean of
the 10th iterate.  Every convolution, its data and weight gradients, and the elementwise
pieces (ReLU backward, pooling, upsampling, skips, MSE, Adam) are this project's kernels
(``cct_conv3x3_*``, ``cct_net_*``); torch only provides device memory.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .core import require_cuda, stream_handle

IN_CHANNELS = 16
N_ITERATES = 10
EPS = float(np.finfo(np.float32).eps)
BF16 = torch.bfloat16


def _p(t: torch.Tensor | None):
    return None if t is None else t.data_ptr()


class Conv:
    """One 3x3 convolution layer: FP32 master weights [cout][3][3][cin], bias, Adam moments."""

    def __init__(self, cin: int, cout: int, relu: bool, rng: np.random.Generator, device):
        self.cin, self.cout, self.relu = cin, cout, relu
        std = math.sqrt(2.0 / (9 * cin))
        w = rng.normal(0.0, std, size=(cout, 9, cin)).astype(np.float32)
        self.w = torch.from_numpy(w).to(device)
        self.b = torch.zeros(cout, dtype=torch.float32, device=device)
        self.w16 = self.w.to(BF16)
        self.wflip = torch.empty((cin, 9, cout), dtype=BF16, device=device)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.x = self.y = None

    def params(self):
        return [self.w, self.b]


class WarmStartNet:
    def __init__(self, seed: int = 0, device=None, channels=(32, 64, 128, 256)):
        self.device = require_cuda(device)
        rng = np.random.default_rng(seed)
        c1, c2, c3, c4 = channels
        d = self.device
        self.layers = {
            "e1a": Conv(IN_CHANNELS, c1, True, rng, d), "e1b": Conv(c1, c1, True, rng, d),
            "e2a": Conv(c1, c2, True, rng, d), "e2b": Conv(c2, c2, True, rng, d),
            "e3a": Conv(c2, c3, True, rng, d), "e3b": Conv(c3, c3, True, rng, d),
            "b1": Conv(c3, c4, True, rng, d), "b2": Conv(c4, c4, True, rng, d),
            "d3a": Conv(c4, c3, True, rng, d), "d3b": Conv(c3, c3, True, rng, d),
            "d2a": Conv(c3, c2, True, rng, d), "d2b": Conv(c2, c2, True, rng, d),
            "d1a": Conv(c2, c1, True, rng, d), "d1b": Conv(c1, c1, True, rng, d),
            "head": Conv(c1, IN_CHANNELS, False, rng, d),
        }
        # the head starts near zero so the first prediction is the 10th iterate itself
        self.layers["head"].w.mul_(0.01)
        self.layers["head"].w16 = self.layers["head"].w.to(BF16)
        self.step_count = 0
        self.lib = _lib.load()
        # target parameterisation: additive correction (x_target - x10) / scale, or multiplicative
        # log((x_target + floor * scale) / (x10 + floor * scale))
        self.multiplicative = False
        self.log_floor = 1e-2
        # inputs: 0 = the first 10 MLEM iterates; k > 0 = 10 snapshots of the iterate taken during
        # one ordered-subsets pass over subsets of k angles each (A // k subsets)
        self.pass_angles = 0
        # ordered-subsets levels around the network: the snapshot pass's level and a finishing
        # level with about finish_factor times fewer subsets (os_levels)
        self.finish_factor = 5

    # ------------------------------------------------------------------ helpers
    def pass_subsets(self, n_angles: int) -> int:
        """Subsets of the one ordered-subsets pass that makes the inputs (0: MLEM inputs)."""
        return 0 if self.pass_angles <= 0 else min(n_angles, max(N_ITERATES, n_angles // self.pass_angles))

    def os_levels(self, n_angles: int) -> list[int]:
        """Subset counts [k1, k2] of the ordered-subsets passes around the network: k1 is the snapshot
        pass's, k2 the largest divisor of k1 that is at most k1 / finish_factor.  Data, maps and
        geometry go in ``engine.subset_permutation(A, os_levels(A))`` order."""
        k1 = self.pass_subsets(n_angles)
        if k1 <= 0:
            return []
        cap = max(1, k1 // max(1, self.finish_factor))
        k2 = max(d for d in range(1, cap + 1) if k1 % d == 0)
        return [k1, k2]

    def n_params(self) -> int:
        return sum(l.w.numel() + l.b.numel() for l in self.layers.values())

    def _desc(self, b, h, w, cin, cout):
        d = _lib.ConvDesc()
        d.batch, d.height, d.width, d.cin, d.cout = b, h, w, cin, cout
        return d

    def _conv(self, layer: Conv, x: torch.Tensor) -> torch.Tensor:
        b, h, w, _ = x.shape
        y = torch.empty((b, h, w, layer.cout), dtype=BF16, device=self.device)
        desc = self._desc(b, h, w, layer.cin, layer.cout)
        _lib.check(self.lib.cct_conv3x3_fwd(ctypes.byref(desc), x.data_ptr(), layer.w16.data_ptr(), layer.b.data_ptr(),
                                            int(layer.relu), y.data_ptr(), stream_handle(self.device)))
        layer.x, layer.y = x, y
        return y

    def _pool(self, x, backward=False, full_shape=None):
        h = self.device
        if not backward:
            b, hh, ww, c = x.shape
            y = torch.empty((b, hh // 2, ww // 2, c), dtype=BF16, device=h)
            _lib.check(self.lib.cct_net_avgpool2(x.data_ptr(), y.data_ptr(), b, hh, ww, c, 0, stream_handle(h)))
            return y
        b, hh, ww, c = full_shape
        y = torch.empty(full_shape, dtype=BF16, device=h)
        _lib.check(self.lib.cct_net_avgpool2(x.data_ptr(), y.data_ptr(), b, hh, ww, c, 1, stream_handle(h)))
        return y

    def _up(self, x, backward=False):
        dev = self.device
        if not backward:
            b, hh, ww, c = x.shape
            y = torch.empty((b, 2 * hh, 2 * ww, c), dtype=BF16, device=dev)
            _lib.check(self.lib.cct_net_upsample2(x.data_ptr(), y.data_ptr(), b, hh, ww, c, 0, stream_handle(dev)))
            return y
        b, hh, ww, c = x.shape
        y = torch.empty((b, hh // 2, ww // 2, c), dtype=BF16, device=dev)
        _lib.check(self.lib.cct_net_upsample2(x.data_ptr(), y.data_ptr(), b, hh // 2, ww // 2, c, 1, stream_handle(dev)))
        return y

    def _add(self, a, b):
        out = torch.empty_like(a)
        _lib.check(self.lib.cct_net_add(a.data_ptr(), b.data_ptr(), out.data_ptr(), a.numel(), stream_handle(self.device)))
        return out

    # ------------------------------------------------------------------ forward / backward
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: NHWC bf16 (B, H, W, 16), H and W divisible by 8.  Returns the head output (B, H, W, 16)."""
        L = self.layers
        e1 = self._conv(L["e1b"], self._conv(L["e1a"], x))
        e2 = self._conv(L["e2b"], self._conv(L["e2a"], self._pool(e1)))
        e3 = self._conv(L["e3b"], self._conv(L["e3a"], self._pool(e2)))
        bt = self._conv(L["b2"], self._conv(L["b1"], self._pool(e3)))
        self._s3 = self._add(self._conv(L["d3a"], self._up(bt)), e3)
        d3 = self._conv(L["d3b"], self._s3)
        self._s2 = self._add(self._conv(L["d2a"], self._up(d3)), e2)
        d2 = self._conv(L["d2b"], self._s2)
        self._s1 = self._add(self._conv(L["d1a"], self._up(d2)), e1)
        d1 = self._conv(L["d1b"], self._s1)
        self._shapes = dict(e1=e1.shape, e2=e2.shape, e3=e3.shape)
        return self._conv(L["head"], d1)

    def _conv_bwd(self, layer: Conv, dy: torch.Tensor) -> torch.Tensor:
        dev = self.device
        h = stream_handle(dev)
        if layer.relu:
            dpre = torch.empty_like(dy)
            _lib.check(self.lib.cct_net_relu_bwd(layer.y.data_ptr(), dy.data_ptr(), dpre.data_ptr(), dy.numel(), h))
        else:
            dpre = dy
        b, hh, ww, _ = dpre.shape
        desc = self._desc(b, hh, ww, layer.cin, layer.cout)
        _lib.check(self.lib.cct_conv3x3_wgrad(ctypes.byref(desc), layer.x.data_ptr(), dpre.data_ptr(), layer.gw.data_ptr(), h))
        _lib.check(self.lib.cct_net_bias_grad(dpre.data_ptr(), layer.gb.data_ptr(), b * hh * ww, layer.cout, h))
        _lib.check(self.lib.cct_net_flip_weights(layer.w16.data_ptr(), layer.wflip.data_ptr(), layer.cin, layer.cout, h))
        dx = torch.empty((b, hh, ww, layer.cin), dtype=BF16, device=dev)
        ddesc = self._desc(b, hh, ww, layer.cout, layer.cin)
        _lib.check(self.lib.cct_conv3x3_fwd(ctypes.byref(ddesc), dpre.data_ptr(), layer.wflip.data_ptr(), None, 0,
                                            dx.data_ptr(), h))
        return dx

    def backward(self, dout: torch.Tensor) -> None:
        """Accumulate parameter gradients for d loss / d head output."""
        L = self.layers
        dd1 = self._conv_bwd(L["head"], dout)
        ds1 = self._conv_bwd(L["d1b"], dd1)
        du1 = self._conv_bwd(L["d1a"], ds1)             # d1a input = up(d2)
        dd2 = self._up(du1, backward=True)
        ds2 = self._conv_bwd(L["d2b"], dd2)
        du2 = self._conv_bwd(L["d2a"], ds2)
        dd3 = self._up(du2, backward=True)
        ds3 = self._conv_bwd(L["d3b"], dd3)
        du3 = self._conv_bwd(L["d3a"], ds3)
        dbt = self._up(du3, backward=True)
        dp3 = self._conv_bwd(L["b1"], self._conv_bwd(L["b2"], dbt))
        de3 = self._add(ds3, self._pool(dp3, backward=True, full_shape=self._shapes["e3"]))
        dp2 = self._conv_bwd(L["e3a"], self._conv_bwd(L["e3b"], de3))
        de2 = self._add(ds2, self._pool(dp2, backward=True, full_shape=self._shapes["e2"]))
        dp1 = self._conv_bwd(L["e2a"], self._conv_bwd(L["e2b"], de2))
        de1 = self._add(ds1, self._pool(dp1, backward=True, full_shape=self._shapes["e1"]))
        self._conv_bwd(L["e1a"], self._conv_bwd(L["e1b"], de1))

    def zero_grad(self) -> None:
        for l in self.layers.values():
            l.gw.zero_()
            l.gb.zero_()

    def adam_step(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step_count += 1
        h = stream_handle(self.device)
        for l in self.layers.values():
            _lib.check(self.lib.cct_net_adam(l.w.data_ptr(), l.gw.data_ptr(), l.mw.data_ptr(), l.vw.data_ptr(),
                                             l.w16.data_ptr(), l.w.numel(), lr, beta1, beta2, eps, self.step_count, h))
            _lib.check(self.lib.cct_net_adam(l.b.data_ptr(), l.gb.data_ptr(), l.mb.data_ptr(), l.vb.data_ptr(), None,
                                             l.b.numel(), lr, beta1, beta2, eps, self.step_count, h))

    def mse(self, out: torch.Tensor, target: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(loss (1,) FP64 tensor, d loss / d out) for channel 0 of out vs target (B, H, W) FP32."""
        grad = torch.empty_like(out)
        loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        pixels = target.numel()
        _lib.check(self.lib.cct_net_mse(out.data_ptr(), target.data_ptr(), grad.data_ptr(), loss.data_ptr(), pixels,
                                        out.shape[-1], stream_handle(self.device)))
        return loss, grad

    # ------------------------------------------------------------------ inputs / outputs
    def pack(self, planes: list[torch.Tensor], slice_scale: torch.Tensor | None = None) -> torch.Tensor:
        """NHWC bf16 input (B, H, W, 16) from FP32 planar images (B, H, W), one per channel, each
        slice divided by its ``slice_scale``."""
        b, hh, ww = planes[0].shape
        # the planes stacked and their pointer table built on the device: no host copy or wait, so
        # the call can be captured in a CUDA graph (the stream orders the kernel before any reuse
        # of these buffers)
        stacked = torch.stack([p.float() for p in planes])
        step = stacked[0].numel() * stacked.element_size()
        ptrs = torch.arange(len(planes), dtype=torch.int64, device=self.device) * step + stacked.data_ptr()
        out = torch.empty((b, hh, ww, IN_CHANNELS), dtype=BF16, device=self.device)
        _lib.check(self.lib.cct_net_pack_nhwc(ptrs.data_ptr(), len(planes), out.data_ptr(), b * hh * ww, IN_CHANNELS,
                                              _p(slice_scale), hh * ww, stream_handle(self.device)))
        return out

    def predict(self, planes: list[torch.Tensor], base: torch.Tensor, slice_scale: torch.Tensor,
                out: torch.Tensor | None = None) -> torch.Tensor:
        """Warm start from the 10th iterate ``base`` (FP32 (B, H, W)).

        additive:       x0 = max(base + scale * v, eps)
        multiplicative: x0 = max((base + scale * floor) * exp(v) - scale * floor, eps)
        with v = net(planes / scale)[0] and floor = ``self.log_floor``."""
        head = self.forward(self.pack(planes, slice_scale))
        b, hh, ww = base.shape
        if out is None:
            out = torch.empty_like(base)
        mode = 1 if self.multiplicative else 0
        floor = self.log_floor if self.multiplicative else EPS
        _lib.check(self.lib.cct_net_unpack_c0(head.data_ptr(), IN_CHANNELS, base.data_ptr(), slice_scale.data_ptr(),
                                              hh * ww, mode, floor, out.data_ptr(), b * hh * ww, stream_handle(self.device)))
        if self.multiplicative:
            out.clamp_(min=EPS)
        return out

    def save(self, path: str) -> None:
        """BF16 weights, FP32 biases and the target parameterisation."""
        st = {k: (l.w.to(BF16).cpu(), l.b.cpu()) for k, l in self.layers.items()}
        st.update(step=self.step_count, multiplicative=self.multiplicative, log_floor=self.log_floor,
                  pass_angles=self.pass_angles, finish_factor=self.finish_factor)
        torch.save(st, path)

    def load(self, path: str) -> None:
        st = torch.load(path, map_location="cpu")
        for k, l in self.layers.items():
            l.w.copy_(st[k][0].to(self.device, torch.float32))
            l.b.copy_(st[k][1].to(self.device))
            l.w16 = l.w.to(BF16)
        self.step_count = int(st.get("step", 0))
        self.multiplicative = bool(st.get("multiplicative", False))
        self.log_floor = float(st.get("log_floor", 1e-2))
        self.pass_angles = int(st.get("pass_angles", 0))
        self.finish_factor = int(st.get("finish_factor", 5))
