"""CPU oracle of the learned warm start's U-Net (float64 numpy).

TEST INFRASTRUCTURE: imported only by tests/, as the checker of the GPU
kernels' forward pass, loss and gradients; the product never imports it.

It restates the network of adaptivegriddiscretizations_b200/WarmStart/unet.py
(there is no reference counterpart: the reference has no learned component)
with the same data layout (NHWC; 3x3 weights as (cout, 9 cin) matrices,
column tap * cin + ci, tap = 3 (dy + 1) + (dx + 1)) and the same rounding
points: everything the GPU stores in bf16 (features, activations, pooled
activations, output gradients) is rounded to bf16 here too; sums are float64
here and float32 on the GPU.
"""
import numpy as np

LEVELS = (32, 64, 128, 256)


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def im2col(x):
    """(n, H, W, C) -> (n H W, 9 C), column tap * C + c, zero padding."""
    n, H, W, C = x.shape
    xp = np.zeros((n, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, dy:dy + H, dx:dx + W] for dy in range(3) for dx in range(3)]
    return np.stack(cols, 3).reshape(n * H * W, 9 * C)


def col2im(g, shape):
    """Adjoint of im2col: (n H W, 9 C) -> (n, H, W, C)."""
    n, H, W, C = shape
    g = g.reshape(n, H, W, 9, C)
    xp = np.zeros((n, H + 2, W + 2, C))
    for t in range(9):
        dy, dx = divmod(t, 3)
        xp[:, dy:dy + H, dx:dx + W] += g[:, :, :, t]
    return xp[:, 1:-1, 1:-1]


def up(x):
    return x.repeat(2, 1).repeat(2, 2)


def upsum(g):
    n, H, W, C = g.shape
    return g.reshape(n, H // 2, 2, W // 2, 2, C).sum((2, 4))


def pool(x):
    n, H, W, C = x.shape
    return x.reshape(n, H // 2, 2, W // 2, 2, C).mean((2, 4))


class Net:
    """Weights: convs[k] = (w (cout, 9 cin) float64 of the bf16 weights, b),
    head (w (32,), b); order enc0a..enc3b, dec2a..dec0b."""

    def __init__(self, convs, head):
        self.convs, self.head = convs, head

    def conv(self, k, x):
        w, b = self.convs[k]
        n, H, W, _ = x.shape
        y = im2col(x) @ w.T + b
        return bf16(np.maximum(y, 0.0)).reshape(n, H, W, -1)

    def forward(self, x0):
        c = self.conv
        a = {"x0": x0}
        a["a0"] = c(0, x0)
        a["y0"] = c(1, a["a0"])
        a["p0"] = bf16(pool(a["y0"]))
        a["a1"] = c(2, a["p0"])
        a["y1"] = c(3, a["a1"])
        a["p1"] = bf16(pool(a["y1"]))
        a["a2"] = c(4, a["p1"])
        a["y2"] = c(5, a["a2"])
        a["p2"] = bf16(pool(a["y2"]))
        a["a3"] = c(6, a["p2"])
        a["y3"] = c(7, a["a3"])
        a["c2"] = np.concatenate([up(a["y3"]), a["y2"]], -1)
        a["d2a"] = c(8, a["c2"])
        a["d2"] = c(9, a["d2a"])
        a["c1"] = np.concatenate([up(a["d2"]), a["y1"]], -1)
        a["d1a"] = c(10, a["c1"])
        a["d1"] = c(11, a["d1a"])
        a["c0"] = np.concatenate([up(a["d1"]), a["y0"]], -1)
        a["d0a"] = c(12, a["c0"])
        a["d0"] = c(13, a["d0a"])
        hw, hb = self.head
        a["r"] = a["d0"] @ hw + hb[0]
        self.a = a
        return a["r"]

    def backward(self, target):
        """Loss (mean squared error over the finite targets) and gradients:
        list of (dw (cout, 9 cin), db) per conv, (dhw, dhb)."""
        a = self.a
        fin = np.isfinite(target)
        cnt = fin.sum()
        d = np.where(fin, a["r"] - np.where(fin, target, 0.0), 0.0)
        loss = float((d * d).sum() / cnt)
        dr = 2.0 * d / cnt
        hw, hb = self.head
        dhw = np.einsum("nhw,nhwc->c", dr, a["d0"])
        dhb = np.array([dr.sum()])
        grads = [None] * 14

        def mask(y, g):
            return bf16(np.where(y > 0, g, 0.0))

        def back(k, x, dz, want_dx=True):
            w, b = self.convs[k]
            n, H, W, _ = x.shape
            dzf = dz.reshape(n * H * W, -1)
            grads[k] = (dzf.T @ im2col(x), dzf.sum(0))
            return col2im(dzf @ w, x.shape) if want_dx else None

        dz = mask(a["d0"], dr[..., None] * hw)
        dz = mask(a["d0a"], back(13, a["d0a"], dz))
        dc0 = back(12, a["c0"], dz)
        c0, c1, c2, c3 = LEVELS
        dz = mask(a["d1"], upsum(dc0[..., :c1]))
        dz = mask(a["d1a"], back(11, a["d1a"], dz))
        dc1 = back(10, a["c1"], dz)
        dz = mask(a["d2"], upsum(dc1[..., :c2]))
        dz = mask(a["d2a"], back(9, a["d2a"], dz))
        dc2 = back(8, a["c2"], dz)
        dz = mask(a["y3"], upsum(dc2[..., :c3]))
        dz = mask(a["a3"], back(7, a["a3"], dz))
        dp2 = back(6, a["p2"], dz)
        dz = mask(a["y2"], up(dp2) / 4 + dc2[..., c3:])
        dz = mask(a["a2"], back(5, a["a2"], dz))
        dp1 = back(4, a["p1"], dz)
        dz = mask(a["y1"], up(dp1) / 4 + dc1[..., c2:])
        dz = mask(a["a1"], back(3, a["a1"], dz))
        dp0 = back(2, a["p0"], dz)
        dz = mask(a["y0"], up(dp0) / 4 + dc0[..., c1:])
        dz = mask(a["a0"], back(1, a["a0"], dz))
        back(0, a["x0"], dz, want_dx=False)
        return loss, grads, (dhw, dhb)
