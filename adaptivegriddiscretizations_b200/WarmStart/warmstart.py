"""Training and use of the learned warm start on Riemann2 problems.

Data: random Riemann2 fields drawn on the GPU (metric R(theta) diag(1, lambda)
R(theta)^T, theta the angle of a periodic Gaussian-smoothed random vector
field, lambda uniform in [1, 100] per point, random seeds), solved cold by
the batched solver itself (Eikonal.BatchSolver); the training pairs are the
block features of agd_ws_features and the log-ratio targets of agd_ws_target.

Use: the prediction (block arrival times T = dref exp(r)) gives every tile a
release epoch (agd_ws_release: tiles are visited no earlier than the epoch at
which the predicted front reaches them) and, optionally, warm-start values
(agd_ws_warm_values: (1 + margin) T, an upper bound where the prediction is
good, since the scheme's values only decrease).  The solver still runs to the
reference's stopping test, so the fixed point is the one of the cold start up
to the stopping tolerance.  The cold solve is the check: evaluate() compares
every warm result with the cold one and counts the instances that would fall
back to it.
"""
import ctypes
import math
import time

import numpy as np
import torch

from .. import _lib
from .unet import UNet


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def riemann2_fields(n, batch, gen, sigma=8.0, nseeds=4):
    """Metric fields (batch, n, n, 3) [m00, m10, m11] and seeds (batch, nseeds, 2)
    in domain coordinates [0.05, 0.95]^2, on the device: theta = atan2 of two
    independent periodic Gaussian-smoothed white noises (sigma pixels), lambda
    uniform in [1, 100]."""
    g = torch.randn((batch, 2, n, n), generator=gen, device="cuda")
    k = torch.fft.fftfreq(n, device="cuda")
    G = torch.exp(-2.0 * math.pi ** 2 * sigma ** 2 * (k[:, None] ** 2 + k[None, :] ** 2))
    g = torch.fft.ifft2(torch.fft.fft2(g) * G).real
    th = torch.atan2(g[:, 0], g[:, 1])
    lam = 1.0 + 99.0 * torch.rand((batch, n, n), generator=gen, device="cuda")
    c, s = torch.cos(th), torch.sin(th)
    metric = torch.stack([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], -1).float().contiguous()
    seeds = (0.05 + 0.9 * torch.rand((batch, nseeds, 2), generator=gen, device="cuda")).contiguous()
    return metric, seeds


class WarmStart:
    """A U-Net and the Riemann2 n x n configuration it serves (gridScale 1/n,
    default tolerances), with a BatchSolver of `batch` instances."""

    def __init__(self, n=512, batch=128, seed=0, template=None):
        from .. import Eikonal
        self.n, self.batch = n, batch
        self.nb = n // 4  # prediction resolution (4x4 blocks)
        self.net = UNet(seed=seed)
        if template is None:
            template = Eikonal.dictIn({"model": "Riemann2", "mode": "gpu", "verbosity": 0, "dims": [n, n],
                                       "gridScale": 1.0 / n, "origin": [0.0, 0.0]})
        self.solver = Eikonal.BatchSolver(template, batch, nbuffers=1)
        self.h = 1.0 / n
        self.epochs, self.lag, self.margin = 160.0, 0, None
        self.history = []

    # ---------------------------------------------------------------- data ---
    def features(self, metric, seeds):
        """Input features (batch, nb, nb, 8) bf16 and dref (batch, nb, nb)."""
        b = metric.shape[0]
        x0 = torch.empty((b, self.nb, self.nb, 8), dtype=torch.bfloat16, device="cuda")
        dref = torch.empty((b, self.nb, self.nb), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().agd_ws_features(_p(metric), _p(seeds), seeds.shape[1], b, self.n, self.n, self.h,
                                              _p(x0), _p(dref), _lib.stream_ptr()), "features")
        return x0, dref

    def target(self, values, dref):
        t = torch.empty_like(dref)
        _lib.check(_lib.lib().agd_ws_target(_p(values), values.shape[0], self.n, self.n, _p(dref), _p(t),
                                            _lib.stream_ptr()), "target")
        return t

    def solve(self, metric, seeds, release=None, values=None):
        """Values (batch, n, n) of a batched solve (device tensor, valid until the
        next solve), solver time (s) by CUDA events, tile visits per instance."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        st = self.solver._bufs[0].stream
        e0.record(st)
        job = self.solver.submit(metric=metric, seeds=seeds, release=release, values=values)
        e1.record(st)
        out = job.result()
        return out, e0.elapsed_time(e1) / 1e3, job.tile_visits

    def generate(self, count, gen):
        """count solver-generated training pairs: x0 (count, nb, nb, 8) bf16,
        target (count, nb, nb) fp32."""
        B = self.batch
        nbatch = (count + B - 1) // B
        X = torch.empty((nbatch * B, self.nb, self.nb, 8), dtype=torch.bfloat16, device="cuda")
        T = torch.empty((nbatch * B, self.nb, self.nb), dtype=torch.float32, device="cuda")
        for k in range(nbatch):
            metric, seeds = riemann2_fields(self.n, B, gen)
            values, _, _ = self.solve(metric, seeds)
            x0, dref = self.features(metric, seeds)
            X[k * B:(k + 1) * B] = x0
            T[k * B:(k + 1) * B] = self.target(values, dref)
        return X[:count], T[:count]

    # ------------------------------------------------------------ training ---
    def train(self, X, T, steps, batch=32, lr=1e-3, gen=None, log_every=50):
        """Adam on the mean squared error of r, random mini-batches of the pairs,
        cosine learning-rate decay; returns the loss history (mean per log period)."""
        net = self.net
        N = X.shape[0]
        count = batch * self.nb * self.nb
        net.zero_grad()
        hist = []
        t0 = time.perf_counter()
        for s in range(steps):
            idx = torch.randint(0, N, (batch,), generator=gen, device="cuda")
            x, t = X.index_select(0, idx), T.index_select(0, idx)
            t = torch.nan_to_num(t, nan=0.0)
            net.forward(x)
            net.backward(t, count)
            net.step(lr * 0.5 * (1.0 + math.cos(math.pi * s / steps)) + 1e-5)
            if (s + 1) % log_every == 0 or s + 1 == steps:
                loss = float(net.loss.item()) / (log_every if (s + 1) % log_every == 0 else (s + 1) % log_every)
                net.loss.zero_()
                hist.append((s + 1, loss))
        torch.cuda.synchronize()
        net.check_err()
        self.train_seconds = time.perf_counter() - t0
        self.history += hist
        return hist

    def eval_loss(self, X, T, batch=64):
        """Mean squared error of r on the pairs (no gradient step)."""
        net = self.net
        tot, cnt = 0.0, 0
        for k in range(0, X.shape[0], batch):
            x, t = X[k:k + batch], T[k:k + batch]
            r = net.forward(x)
            fin = torch.isfinite(t)
            tot += float(((r - torch.nan_to_num(t)) ** 2)[fin].sum())
            cnt += int(fin.sum())
        return tot / max(cnt, 1)

    # ----------------------------------------------------------------- use ---
    def predict(self, metric, seeds):
        """Block arrival times (batch, nb, nb) = dref exp(r)."""
        x0, dref = self.features(metric, seeds)
        r = self.net.forward(x0)
        return dref * torch.exp(r)

    def release(self, pred, epochs=None, lag=None):
        rel = torch.empty((pred.shape[0], (self.nb // 2) ** 2), dtype=torch.int16, device="cuda")
        _lib.check(_lib.lib().agd_ws_release(_p(pred), pred.shape[0], self.nb, self.nb,
                                             float(self.epochs if epochs is None else epochs),
                                             int(self.lag if lag is None else lag), _p(rel), _lib.stream_ptr()),
                   "release")
        return rel

    def warm_values(self, pred, margin):
        v = torch.empty((pred.shape[0], self.n * self.n), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().agd_ws_warm_values(_p(pred), pred.shape[0], self.n, self.n, float(margin), _p(v),
                                                 _lib.stream_ptr()), "warm values")
        return v

    def warm_solve(self, metric, seeds, margin=None):
        """Prediction, release epochs (and warm values) and the gated solve:
        (values, total device seconds including the prediction, tile visits)."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pred = self.predict(metric, seeds)
        rel = self.release(pred)
        vals = self.warm_values(pred, margin) if margin is not None else None
        e1.record()
        out, t_solve, visits = self.solve(metric, seeds, release=rel, values=vals)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3 + t_solve, visits

    def fallback_mask(self, warm, cold, tol_factor=8.0):
        """Instances (batch,) whose warm values differ from the cold ones by more
        than tol_factor stopping tolerances somewhere: they fall back to the
        cold result.  Two solves that each meet the parity criteria (within 4
        stopping tolerances of the discrete solution) are within 8 of each other."""
        B = warm.shape[0]
        fin = torch.isfinite(cold)
        diff = (warm - cold).abs()
        atol = float(np.float32(1.0 * np.finfo(np.float32).resolution * 5.0))
        bad = (diff > tol_factor * (atol + float(self.solver.rtol) * cold.abs())) & fin
        bad |= torch.isfinite(warm) != fin
        return bad.reshape(B, -1).any(1)

    def checked_solve(self, metric, seeds, margin=None, tol_factor=8.0):
        """The warm solve with the cold solve as check and fallback: values
        (batch, n, n) (device tensor) and the fallback mask (batch,)."""
        cold, _, _ = self.solve(metric, seeds)
        cold = cold.clone()
        warm, _, _ = self.warm_solve(metric, seeds, margin=margin)
        bad = self.fallback_mask(warm, cold, tol_factor)
        return torch.where(bad.reshape(-1, *([1] * (cold.dim() - 1))), cold, warm), bad

    def tune(self, metric, seeds, candidates=(100.0, 130.0, 160.0, 200.0, 260.0)):
        """Chooses the release epoch scale on one batch: the fastest gated solve."""
        pred = self.predict(metric, seeds)
        best = None
        for E in candidates:
            rel = self.release(pred, epochs=E)
            _, t, _ = self.solve(metric, seeds, release=rel)
            _, t2, _ = self.solve(metric, seeds, release=rel)
            t = min(t, t2)
            if best is None or t < best[1]:
                best = (E, t)
        self.epochs = best[0]
        return best

    def evaluate(self, nheld, gen, margin=None, tol_factor=8.0):
        """Cold and warm solves of nheld held-out instances: solves/s of each
        (device time; the warm one includes the prediction), tile visits, the
        largest relative difference of the warm result from the cold one, and
        the instances whose warm result differs from the cold one by more than
        tol_factor stopping tolerances somewhere (they fall back to the cold
        result).  Two solves that each meet the parity criteria (within 4
        stopping tolerances of the discrete solution) are within 8 of each
        other, hence the default."""
        B = self.batch
        t_cold = t_warm = 0.0
        v_cold = v_warm = 0
        worst, fallbacks, done = 0.0, 0, 0
        while done < nheld:
            metric, seeds = riemann2_fields(self.n, B, gen)
            cold, tc, vc = self.solve(metric, seeds)
            cold = cold.clone()
            warm, tw, vw = self.warm_solve(metric, seeds, margin=margin)
            t_cold += tc
            t_warm += tw
            v_cold += int(vc.sum())
            v_warm += int(vw.sum())
            fin = torch.isfinite(cold)
            diff = (warm - cold).abs()
            rel = torch.where(fin, diff / cold.abs().clamp_min(1e-30), torch.zeros_like(diff))
            worst = max(worst, float(rel.max()))
            fallbacks += int(self.fallback_mask(warm, cold, tol_factor).sum())
            done += B
        return {"instances": done, "cold_solves_per_s": done / t_cold, "warm_solves_per_s": done / t_warm,
                "gain": t_cold / t_warm, "cold_tile_visits": v_cold, "warm_tile_visits": v_warm,
                "max_rel_diff_vs_cold": worst, "fallbacks": fallbacks, "release_epochs": self.epochs,
                "warm_values_margin": margin}
