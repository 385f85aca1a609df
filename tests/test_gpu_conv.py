"""The tensor-core 3x3 convolutions of the learned warm start
(agd_conv3x3_forward / agd_conv3x3_weight_grad, include/agd_warmstart.h)
against a plain PyTorch fp32 reference of the same operation on the same
bf16-rounded operands: forward with bias and ReLU, the input gradient (the
forward call on flipped weights), and the weight gradient, for single inputs
and for the decoder's concatenation of an upsampled tensor and a skip tensor.
Tolerance: fp32 accumulation against fp32 (the reference in float64 here):
relative Frobenius error 2e-3 (bf16 outputs) or 1e-4 (fp32 outputs)."""
import ctypes

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def _lib():
    from adaptivegriddiscretizations_b200 import _lib as L
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _conv(n, H, W, srcs, cout):
    L = _lib()
    c = L.AgdConv()
    c.n, c.H, c.W, c.cout = n, H, W, cout
    for k, (t, ch, up) in enumerate(srcs):
        c.src[k].data, c.src[k].channels, c.src[k].up = t.data_ptr(), ch, up
    return c


def _input(srcs):
    """The convolution input in NCHW float64: concatenation of the (upsampled) sources."""
    parts = []
    for t, ch, up in srcs:
        x = t.double().permute(0, 3, 1, 2)
        if up:
            x = x.repeat_interleave(2, 2).repeat_interleave(2, 3)
        parts.append(x)
    return torch.cat(parts, 1)


def _weights(cout, cin, gen):
    L = _lib()
    kpad = L.lib().agd_conv_kpad(cin)
    w = torch.zeros((cout, kpad), dtype=torch.float32)
    w[:, :9 * cin] = torch.randn((cout, 9 * cin), generator=gen) * (2.0 / (9 * cin)) ** 0.5
    wb = w.to(torch.bfloat16).cuda()
    # (cout, kpad) with column tap * cin + ci -> OIHW
    w4 = wb[:, :9 * cin].double().view(cout, 3, 3, cin).permute(0, 3, 1, 2).contiguous()
    return wb, w4


def _rel(a, b):
    return float((a - b).norm() / b.norm().clamp_min(1e-30))


CASES = [  # (n, H, W, [(cin, up)], cout)
    (2, 32, 48, [(8, 0)], 32),
    (3, 16, 16, [(32, 0)], 64),
    (1, 24, 40, [(64, 0)], 256),
    (2, 32, 32, [(64, 1), (32, 0)], 32),
    (2, 16, 16, [(256, 1), (128, 0)], 128),
    (1, 8, 8, [(128, 0)], 384),
    # bulk-copy (TMA) operand path: inputs at the output resolution, channels
    # multiples of 32, W | 128, 128 | H W; mixed 64- and 32-channel blocks
    (2, 32, 32, [(64, 0), (32, 0)], 32),
    (4, 64, 64, [(32, 0)], 64),
    (2, 16, 16, [(256, 0), (128, 0)], 128),
    (1, 128, 128, [(32, 0)], 32),
    (2, 32, 32, [(128, 0)], 256),
]


@pytest.mark.parametrize("case", CASES)
def test_conv_forward_and_gradients(case):
    L = _lib()
    lib = L.lib()
    n, H, W, spec, cout = case
    gen = torch.Generator().manual_seed(sum(ch for ch, _ in spec) + cout)
    srcs = []
    for ch, up in spec:
        t = torch.randn((n, H >> up, W >> up, ch), generator=gen).to(torch.bfloat16).cuda()
        srcs.append((t, ch, up))
    cin = sum(ch for ch, _ in spec)
    wb, w4 = _weights(cout, cin, gen)
    bias = (0.1 * torch.randn(cout, generator=gen)).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = L.stream_ptr()
    c = _conv(n, H, W, srcs, cout)
    x = _input(srcs)
    ref = F.relu(F.conv2d(x, w4, bias.double(), padding=1)).permute(0, 2, 3, 1)
    out = torch.empty((n, H, W, cout), dtype=torch.bfloat16, device="cuda")
    L.check(lib.agd_conv3x3_forward(ctypes.byref(c), _p(wb), _p(bias), 1, _p(out), None, _p(err), s))
    outf = torch.empty((n, H, W, cout), dtype=torch.float32, device="cuda")
    L.check(lib.agd_conv3x3_forward(ctypes.byref(c), _p(wb), None, 0, None, _p(outf), _p(err), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert _rel(out.double(), ref) < 4e-3
    assert _rel(outf.double(), F.conv2d(x, w4, padding=1).permute(0, 2, 3, 1)) < 1e-4
    # input gradient (the network needs none for its 8-channel input layer):
    # forward call with the flipped weights on dz
    dz = torch.randn((n, H, W, cout), generator=gen).to(torch.bfloat16).cuda()
    xr = x.clone().requires_grad_(True)
    wr = w4.clone().requires_grad_(True)
    y = F.conv2d(xr, wr, padding=1)
    y.backward(dz.double().permute(0, 3, 1, 2))
    if cin % 16 == 0:
        wt = torch.empty((cin, lib.agd_conv_kpad(cout)), dtype=torch.bfloat16, device="cuda")
        L.check(lib.agd_conv_weight_flip(cin, cout, _p(wb), _p(wt), s))
        dx = torch.empty((n, H, W, cin), dtype=torch.float32, device="cuda")
        cd = _conv(n, H, W, [(dz, cout, 0)], cin)
        L.check(lib.agd_conv3x3_forward(ctypes.byref(cd), _p(wt), None, 0, None, _p(dx), _p(err), s))
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert _rel(dx.double().permute(0, 3, 1, 2), xr.grad) < 1e-4
    # weight gradient, accumulated onto a non-zero buffer
    dw = torch.full((cout, lib.agd_conv_kpad(cin)), 0.5, dtype=torch.float32, device="cuda")
    L.check(lib.agd_conv3x3_weight_grad(ctypes.byref(c), _p(dz), _p(dw), _p(err), s))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    gw = (dw[:, :9 * cin].double() - 0.5).view(cout, 3, 3, cin).permute(0, 3, 1, 2)
    assert _rel(gw, wr.grad) < 1e-4
    if dw.shape[1] > 9 * cin:  # padding columns untouched
        assert float(dw[:, 9 * cin:].sub(0.5).abs().max()) == 0.0
