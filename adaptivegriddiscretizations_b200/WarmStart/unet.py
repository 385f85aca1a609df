"""The warm start's U-Net: four levels (32, 64, 128, 256 channels at 1, 1/2,
1/4, 1/8 of the input resolution), two 3x3 convolutions with ReLU per level,
2x2 average pooling down, nearest 2x upsampling and concatenation with the
skip connection up, and a 1x1 head.  bf16 weights and activations, fp32
accumulation, fp32 master weights and Adam moments.

Every layer runs in libagd_b200 through include/agd_warmstart.h: the 3x3
convolutions (forward, input gradient, weight gradient) as implicit GEMMs on
the tcgen05 tensor cores, the rest as memory-bound kernels.  torch only holds
the device buffers.  The reference has no learned component.
"""
import ctypes
import math

import torch

from .. import _lib

LEVELS = (32, 64, 128, 256)
IN_CHANNELS = 8


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class ConvLayer:
    """One 3x3 convolution: fp32 master weights (cout, kpad), their bf16 copy,
    the flipped bf16 weights of the input gradient, bias, gradients, Adam moments."""

    def __init__(self, cin, cout, gen):
        L = _lib.lib()
        self.cin, self.cout = cin, cout
        self.kpad = L.agd_conv_kpad(cin)
        self.kpad_t = L.agd_conv_kpad(cout)
        w = torch.zeros((cout, self.kpad), dtype=torch.float32)
        w[:, :9 * cin] = torch.randn((cout, 9 * cin), generator=gen) * math.sqrt(2.0 / (9 * cin))
        self.w = w.cuda()
        self.b = torch.zeros(cout, dtype=torch.float32, device="cuda")
        self.wb = torch.empty((cout, self.kpad), dtype=torch.bfloat16, device="cuda")
        self.wt = torch.empty((cin, self.kpad_t), dtype=torch.bfloat16, device="cuda")
        self.dw = torch.zeros_like(self.w)
        self.db = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)
        self.refresh()

    def refresh(self):
        """bf16 copy and flipped weights from the master weights."""
        self.wb.copy_(self.w)
        self.flip()

    def flip(self):
        _lib.check(_lib.lib().agd_conv_weight_flip(self.cin, self.cout, _p(self.wb), _p(self.wt), _lib.stream_ptr()),
                   "weight flip")

    def state(self):
        return {"w": self.w, "b": self.b}


def _conv_desc(n, H, W, srcs, cout):
    c = _lib.AgdConv()
    c.n, c.H, c.W, c.cout = n, H, W, cout
    for k, (t, ch, up) in enumerate(srcs):
        c.src[k].data = t.data_ptr()
        c.src[k].channels = ch
        c.src[k].up = up
    return c


class UNet:
    """Forward, backward and Adam step of the network on batches of n images of
    H x W input pixels (H, W multiples of 16), with buffers kept per shape."""

    def __init__(self, seed=0):
        gen = torch.Generator().manual_seed(seed)
        c0, c1, c2, c3 = LEVELS
        self.enc = [ConvLayer(IN_CHANNELS, c0, gen), ConvLayer(c0, c0, gen), ConvLayer(c0, c1, gen),
                    ConvLayer(c1, c1, gen), ConvLayer(c1, c2, gen), ConvLayer(c2, c2, gen),
                    ConvLayer(c2, c3, gen), ConvLayer(c3, c3, gen)]
        self.dec = [ConvLayer(c3 + c2, c2, gen), ConvLayer(c2, c2, gen), ConvLayer(c2 + c1, c1, gen),
                    ConvLayer(c1, c1, gen), ConvLayer(c1 + c0, c0, gen), ConvLayer(c0, c0, gen)]
        self.hw = (torch.randn(c0, generator=gen) * math.sqrt(1.0 / c0)).cuda()
        self.hb = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.dhw, self.dhb = torch.zeros_like(self.hw), torch.zeros_like(self.hb)
        self.mhw, self.vhw = torch.zeros_like(self.hw), torch.zeros_like(self.hw)
        self.mhb, self.vhb = torch.zeros_like(self.hb), torch.zeros_like(self.hb)
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.t = 0
        self._buf = {}

    # ------------------------------------------------------------ buffers ---
    def buffers(self, n, H, W):
        key = (n, H, W)
        if key in self._buf:
            return self._buf[key]
        c0, c1, c2, c3 = LEVELS
        R = [(H >> k, W >> k) for k in range(4)]

        def bf(level, ch):
            h, w = R[level]
            return torch.empty((n, h, w, ch), dtype=torch.bfloat16, device="cuda")

        def f32(level, ch):
            h, w = R[level]
            return torch.empty((n, h, w, ch), dtype=torch.float32, device="cuda")

        B = dict(u2=bf(2, c3), u1=bf(1, c2), u0=bf(0, c1),  # upsampled decoder inputs
                 a0=bf(0, c0), y0=bf(0, c0), p0=bf(1, c0), a1=bf(1, c1), y1=bf(1, c1), p1=bf(2, c1),
                 a2=bf(2, c2), y2=bf(2, c2), p2=bf(3, c2), a3=bf(3, c3), y3=bf(3, c3),
                 d2a=bf(2, c2), d2=bf(2, c2), d1a=bf(1, c1), d1=bf(1, c1), d0a=bf(0, c0), d0=bf(0, c0),
                 r=torch.empty((n, H, W), dtype=torch.float32, device="cuda"),
                 # backward: output gradients (bf16, ReLU mask applied), input gradients (fp32)
                 gz=bf(0, c0), dx=f32(0, c0),
                 dcat0=f32(0, c1 + c0), dcat1=f32(1, c2 + c1), dcat2=f32(2, c3 + c2))
        B["gz_views"] = {}
        self._buf[key] = B
        return B

    def _gz(self, B, shape, ch):
        """A bf16 output-gradient buffer of the given shape (views of one allocation)."""
        n, h, w = shape
        need = n * h * w * ch
        if B["gz"].numel() < need:
            B["gz"] = torch.empty(need, dtype=torch.bfloat16, device="cuda")
        return B["gz"].view(-1)[:need].view(n, h, w, ch)

    # -------------------------------------------------------------- layers ---
    def _conv(self, layer, n, H, W, srcs, out_bf=None, out_f=None, relu=True, bias=True, weights=None):
        c = _conv_desc(n, H, W, srcs, out_bf.shape[-1] if out_bf is not None else out_f.shape[-1])
        _lib.check(_lib.lib().agd_conv3x3_forward(ctypes.byref(c), _p(weights if weights is not None else layer.wb),
                                                  _p(layer.b) if bias else None, int(relu), _p(out_bf), _p(out_f),
                                                  _p(self.err), _lib.stream_ptr()), "conv3x3")

    def _wgrad(self, layer, n, H, W, srcs, dz):
        c = _conv_desc(n, H, W, srcs, layer.cout)
        L = _lib.lib()
        _lib.check(L.agd_conv3x3_weight_grad(ctypes.byref(c), _p(dz), _p(layer.dw), _p(self.err),
                                             _lib.stream_ptr()), "conv3x3 weight grad")
        _lib.check(L.agd_ws_bias_grad(_p(dz), n * H * W, layer.cout, _p(layer.db), _lib.stream_ptr()), "bias grad")

    def _dgrad(self, layer, n, H, W, dz, out):
        """Input gradient (fp32 NHWC, layer.cin channels) of the output gradient dz."""
        self._conv(layer, n, H, W, [(dz, layer.cout, 0)], out_f=out, relu=False, bias=False, weights=layer.wt)

    def _pool(self, x, y):
        n, H, W, C = x.shape
        _lib.check(_lib.lib().agd_ws_avgpool(_p(x), n, H, W, C, _p(y), _lib.stream_ptr()), "avgpool")

    def _upsample(self, x, y):
        n, H, W, C = x.shape
        _lib.check(_lib.lib().agd_ws_upsample(_p(x), n, H, W, C, _p(y), _lib.stream_ptr()), "upsample")

    def _route(self, y, terms, dz):
        n, H, W, C = y.shape
        ts = [_lib.AgdWsTerm() for _ in range(2)]
        for t, (buf, mode, off) in zip(ts, terms):
            t.data, t.mode, t.channels, t.offset = buf.data_ptr(), mode, buf.shape[-1], off
        _lib.check(_lib.lib().agd_ws_route(n, H, W, C, _p(y), ts[0], ts[1], _p(dz), _lib.stream_ptr()), "route")

    # ------------------------------------------------------------- forward ---
    def forward(self, x0):
        """r (n, H, W) fp32 from the input features x0 (n, H, W, 8) bf16."""
        n, H, W, _ = x0.shape
        B = self.buffers(n, H, W)
        c0, c1, c2, c3 = LEVELS
        e, d = self.enc, self.dec
        R = [(H >> k, W >> k) for k in range(4)]
        self._x0 = x0
        self._conv(e[0], n, *R[0], [(x0, IN_CHANNELS, 0)], B["a0"])
        self._conv(e[1], n, *R[0], [(B["a0"], c0, 0)], B["y0"])
        self._pool(B["y0"], B["p0"])
        self._conv(e[2], n, *R[1], [(B["p0"], c0, 0)], B["a1"])
        self._conv(e[3], n, *R[1], [(B["a1"], c1, 0)], B["y1"])
        self._pool(B["y1"], B["p1"])
        self._conv(e[4], n, *R[2], [(B["p1"], c1, 0)], B["a2"])
        self._conv(e[5], n, *R[2], [(B["a2"], c2, 0)], B["y2"])
        self._pool(B["y2"], B["p2"])
        self._conv(e[6], n, *R[3], [(B["p2"], c2, 0)], B["a3"])
        self._conv(e[7], n, *R[3], [(B["a3"], c3, 0)], B["y3"])
        self._upsample(B["y3"], B["u2"])
        self._conv(d[0], n, *R[2], [(B["u2"], c3, 0), (B["y2"], c2, 0)], B["d2a"])
        self._conv(d[1], n, *R[2], [(B["d2a"], c2, 0)], B["d2"])
        self._upsample(B["d2"], B["u1"])
        self._conv(d[2], n, *R[1], [(B["u1"], c2, 0), (B["y1"], c1, 0)], B["d1a"])
        self._conv(d[3], n, *R[1], [(B["d1a"], c1, 0)], B["d1"])
        self._upsample(B["d1"], B["u0"])
        self._conv(d[4], n, *R[0], [(B["u0"], c1, 0), (B["y0"], c0, 0)], B["d0a"])
        self._conv(d[5], n, *R[0], [(B["d0a"], c0, 0)], B["d0"])
        _lib.check(_lib.lib().agd_ws_head_forward(_p(B["d0"]), n * H * W, _p(self.hw), _p(self.hb), _p(B["r"]),
                                                  _lib.stream_ptr()), "head")
        return B["r"]

    # ------------------------------------------------------------ backward ---
    def backward(self, target, ncount):
        """Mean squared error of the last forward's r against target (NaN:
        ignored; ncount finite entries), added to self.loss; gradients
        accumulated into the layers."""
        x0 = self._x0
        n, H, W, _ = x0.shape
        B = self.buffers(n, H, W)
        c0, c1, c2, c3 = LEVELS
        e, d = self.enc, self.dec
        R = [(H >> k, W >> k) for k in range(4)]
        L = _lib.lib()
        SAME, POOL, UPSUM = 1, 2, 3
        dz = self._gz(B, (n,) + R[0], c0)
        _lib.check(L.agd_ws_head_loss_backward(_p(B["d0"]), n * H * W, _p(self.hw), _p(B["r"]), _p(target),
                                               int(ncount), _p(dz), _p(self.dhw), _p(self.dhb), _p(self.loss),
                                               _lib.stream_ptr()), "head loss")

        def conv_back(layer, level, srcs, dz, dx_out):
            self._wgrad(layer, n, *R[level], srcs, dz)
            if dx_out is not None:
                self._dgrad(layer, n, *R[level], dz, dx_out)

        def scratch(level, ch):
            h, w = R[level]
            need = n * h * w * ch
            if B["dx"].numel() < need:
                B["dx"] = torch.empty(need, dtype=torch.float32, device="cuda")
            return B["dx"].view(-1)[:need].view(n, h, w, ch)

        # level 0 decoder
        dx = scratch(0, c0)
        conv_back(d[5], 0, [(B["d0a"], c0, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[0], c0)
        self._route(B["d0a"], [(dx, SAME, 0)], dz)
        conv_back(d[4], 0, [(B["d1"], c1, 1), (B["y0"], c0, 0)], dz, B["dcat0"])
        # level 1 decoder
        dz = self._gz(B, (n,) + R[1], c1)
        self._route(B["d1"], [(B["dcat0"], UPSUM, 0)], dz)
        dx = scratch(1, c1)
        conv_back(d[3], 1, [(B["d1a"], c1, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[1], c1)
        self._route(B["d1a"], [(dx, SAME, 0)], dz)
        conv_back(d[2], 1, [(B["d2"], c2, 1), (B["y1"], c1, 0)], dz, B["dcat1"])
        # level 2 decoder
        dz = self._gz(B, (n,) + R[2], c2)
        self._route(B["d2"], [(B["dcat1"], UPSUM, 0)], dz)
        dx = scratch(2, c2)
        conv_back(d[1], 2, [(B["d2a"], c2, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[2], c2)
        self._route(B["d2a"], [(dx, SAME, 0)], dz)
        conv_back(d[0], 2, [(B["y3"], c3, 1), (B["y2"], c2, 0)], dz, B["dcat2"])
        # bottleneck
        dz = self._gz(B, (n,) + R[3], c3)
        self._route(B["y3"], [(B["dcat2"], UPSUM, 0)], dz)
        dx = scratch(3, c3)
        conv_back(e[7], 3, [(B["a3"], c3, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[3], c3)
        self._route(B["a3"], [(dx, SAME, 0)], dz)
        dx = scratch(3, c2)
        conv_back(e[6], 3, [(B["p2"], c2, 0)], dz, dx)
        # level 2 encoder: pooled path and skip connection
        dz = self._gz(B, (n,) + R[2], c2)
        self._route(B["y2"], [(dx, POOL, 0), (B["dcat2"], SAME, c3)], dz)
        dx = scratch(2, c2)
        conv_back(e[5], 2, [(B["a2"], c2, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[2], c2)
        self._route(B["a2"], [(dx, SAME, 0)], dz)
        dx = scratch(2, c1)
        conv_back(e[4], 2, [(B["p1"], c1, 0)], dz, dx)
        # level 1 encoder
        dz = self._gz(B, (n,) + R[1], c1)
        self._route(B["y1"], [(dx, POOL, 0), (B["dcat1"], SAME, c2)], dz)
        dx = scratch(1, c1)
        conv_back(e[3], 1, [(B["a1"], c1, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[1], c1)
        self._route(B["a1"], [(dx, SAME, 0)], dz)
        dx = scratch(1, c0)
        conv_back(e[2], 1, [(B["p0"], c0, 0)], dz, dx)
        # level 0 encoder
        dz = self._gz(B, (n,) + R[0], c0)
        self._route(B["y0"], [(dx, POOL, 0), (B["dcat0"], SAME, c1)], dz)
        dx = scratch(0, c0)
        conv_back(e[1], 0, [(B["a0"], c0, 0)], dz, dx)
        dz = self._gz(B, (n,) + R[0], c0)
        self._route(B["a0"], [(dx, SAME, 0)], dz)
        conv_back(e[0], 0, [(x0, IN_CHANNELS, 0)], dz, None)

    # ----------------------------------------------------------- optimiser ---
    def layers(self):
        return self.enc + self.dec

    def step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        """One Adam step on every weight; clears the gradients."""
        self.t += 1
        L = _lib.lib()
        s = _lib.stream_ptr()
        for layer in self.layers():
            _lib.check(L.agd_ws_adam(_p(layer.w), _p(layer.dw), _p(layer.mw), _p(layer.vw), layer.w.numel(),
                                     lr, beta1, beta2, eps, self.t, _p(layer.wb), s), "adam")
            _lib.check(L.agd_ws_adam(_p(layer.b), _p(layer.db), _p(layer.mb), _p(layer.vb), layer.b.numel(),
                                     lr, beta1, beta2, eps, self.t, None, s), "adam")
            layer.flip()
        _lib.check(L.agd_ws_adam(_p(self.hw), _p(self.dhw), _p(self.mhw), _p(self.vhw), self.hw.numel(), lr,
                                 beta1, beta2, eps, self.t, None, s), "adam")
        _lib.check(L.agd_ws_adam(_p(self.hb), _p(self.dhb), _p(self.mhb), _p(self.vhb), 1, lr, beta1, beta2, eps,
                                 self.t, None, s), "adam")

    def zero_grad(self):
        for layer in self.layers():
            layer.dw.zero_()
            layer.db.zero_()
        self.dhw.zero_()
        self.dhb.zero_()

    def check_err(self):
        if int(self.err.item()):
            raise _lib.AgdError(_lib.AGD_STATUS_WATCHDOG, "a convolution kernel's bounded wait gave up")

    def state_dict(self):
        out = {}
        for k, layer in enumerate(self.layers()):
            out[f"conv{k}.w"] = layer.w.cpu()
            out[f"conv{k}.b"] = layer.b.cpu()
        out["head.w"], out["head.b"] = self.hw.cpu(), self.hb.cpu()
        return out

    def load_state_dict(self, sd):
        for k, layer in enumerate(self.layers()):
            layer.w.copy_(sd[f"conv{k}.w"])
            layer.b.copy_(sd[f"conv{k}.b"])
            layer.refresh()
        self.hw.copy_(sd["head.w"])
        self.hb.copy_(sd["head.b"])
