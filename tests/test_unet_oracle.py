"""The CPU oracle of the warm start's U-Net (oracle/unet_oracle.py) checked
on its own: with the bf16 rounding switched off, its hand-written backward
pass matches central finite differences of its forward pass (float64)."""
import numpy as np

from oracle import unet_oracle as U

CINS = [8, 32, 32, 64, 64, 128, 128, 256, 384, 128, 192, 64, 96, 32]
COUTS = [32, 32, 64, 64, 128, 128, 256, 256, 128, 128, 64, 64, 32, 32]


def test_oracle_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(U, "bf16", lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    convs = [(rng.standard_normal((co, 9 * ci)) * np.sqrt(2.0 / (9 * ci)), rng.standard_normal(co) * 0.05)
             for ci, co in zip(CINS, COUTS)]
    head = (rng.standard_normal(32) * 0.2, np.array([0.3]))
    net = U.Net(convs, head)
    x0 = rng.standard_normal((1, 16, 16, 8))
    t = rng.standard_normal((1, 16, 16))
    t[0, 0, :4] = np.nan
    net.forward(x0)
    loss, grads, (dhw, dhb) = net.backward(t)

    def L():
        net.forward(x0)
        return net.backward(t)[0]

    eps = 1e-6
    for k in (0, 5, 8, 13):
        w, b = convs[k]
        for _ in range(3):
            i, j = rng.integers(w.shape[0]), rng.integers(w.shape[1])
            w0 = w[i, j]
            w[i, j] = w0 + eps
            lp = L()
            w[i, j] = w0 - eps
            lm = L()
            w[i, j] = w0
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grads[k][0][i, j]) <= 1e-5 * max(1.0, abs(fd)), (k, i, j, fd, grads[k][0][i, j])
        i = rng.integers(b.shape[0])
        b0 = b[i]
        b[i] = b0 + eps
        lp = L()
        b[i] = b0 - eps
        lm = L()
        b[i] = b0
        assert abs((lp - lm) / (2 * eps) - grads[k][1][i]) <= 1e-5 * max(1.0, abs(grads[k][1][i]))
    hw = head[0]
    h0 = hw[3]
    hw[3] = h0 + eps
    lp = L()
    hw[3] = h0 - eps
    lm = L()
    hw[3] = h0
    assert abs((lp - lm) / (2 * eps) - dhw[3]) <= 1e-6
