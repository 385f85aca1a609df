"""The U-Net of the learned warm start on the GPU against its CPU oracle
(oracle/unet_oracle.py, float64 with the GPU's bf16 rounding points): the
prediction, the loss and the gradient of every weight after one forward and
backward pass of a small batch.  Tolerances: prediction and loss 5e-3
relative (14 layers of bf16 activations, whose rounding flips by one unit
where the float32 and float64 sums straddle a rounding boundary); gradients
2e-2 in relative Frobenius norm."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_unet_gradients_vs_cpu_oracle():
    from adaptivegriddiscretizations_b200.WarmStart import UNet
    from oracle import unet_oracle as U
    torch.manual_seed(0)
    n, H, W = 2, 32, 48
    net = UNet(seed=3)
    for layer in net.layers():  # non-zero biases, so that they matter
        layer.b.copy_(0.05 * torch.randn(layer.cout))
    net.hb.fill_(0.3)
    g = torch.Generator().manual_seed(5)
    x0 = torch.randn((n, H, W, 8), generator=g).to(torch.bfloat16).cuda()
    target = torch.randn((n, H, W), generator=g).cuda()
    target[0, :3, :5] = float("nan")
    count = int(torch.isfinite(target).sum())
    r = net.forward(x0)
    net.zero_grad()
    net.loss.zero_()
    net.backward(target, count)
    torch.cuda.synchronize()
    net.check_err()
    convs = []
    for layer in net.layers():
        convs.append((layer.wb[:, :9 * layer.cin].double().cpu().numpy(), layer.b.double().cpu().numpy()))
    ref = U.Net(convs, (net.hw.double().cpu().numpy(), net.hb.double().cpu().numpy()))
    rr = ref.forward(x0.double().cpu().numpy())
    assert _rel(r.cpu().numpy(), rr) < 5e-3
    loss, grads, (dhw, dhb) = ref.backward(target.double().cpu().numpy())
    assert abs(float(net.loss.item()) - loss) <= 5e-3 * loss
    for k, (layer, (dw, db)) in enumerate(zip(net.layers(), grads)):
        assert _rel(layer.dw[:, :9 * layer.cin].cpu().numpy(), dw) < 2e-2, k
        assert _rel(layer.db.cpu().numpy(), db) < 2e-2, k
        if layer.kpad > 9 * layer.cin:
            assert float(layer.dw[:, 9 * layer.cin:].abs().max()) == 0.0
    assert _rel(net.dhw.cpu().numpy(), dhw) < 5e-3
    assert _rel(net.dhb.cpu().numpy(), dhb) < 5e-3
