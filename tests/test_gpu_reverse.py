"""GPU parity of the reverse-mode sensitivity (agd_reverse).

Against the reference's golden costSensitivity / seedValueSensitivity, the
known answer of EikonalAD_GPU.ipynb, and central finite differences of the
float64 oracle.
"""
import numpy as np
import pytest
import torch

from conftest import load_case, make_dictin
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["iso2", "riem2", "iso3", "riem3", "ad_notebook", "riem3_32"])
def test_reverse_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k != "tips"}
    out = make_dictin(case).Run()
    cs = out["costSensitivity"].cpu().numpy()
    want = ref["costSensitivity"]
    assert cs.shape == want.shape
    assert np.abs(cs - want).max() <= 1e-4 * np.abs(want).max()
    sv = out["seedValueSensitivity"].cpu().numpy()
    np.testing.assert_allclose(sv, ref["seedValueSensitivity"], rtol=1e-4, atol=1e-5)


def test_reverse_known_answer():
    """EikonalAD_GPU.ipynb cell 42: seedValueSensitivity == [[0],[1]] within 1e-6."""
    case, _ = load_case("ad_notebook")
    out = make_dictin(case).Run()
    sv = out["seedValueSensitivity"].cpu().numpy()
    assert np.abs(sv - np.array([[0.0], [1.0]])).max() < 1e-6


def _small_riemann(n=36, seed=3):
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, np.pi)
    c, s = np.cos(th), np.sin(th)
    lam = 4.0
    m = np.array([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], np.float32)
    metric = np.broadcast_to(m, (n, n, 3)).astype(np.float32).copy()
    cost = np.exp(0.3 * rng.standard_normal((n, n))).astype(np.float32)
    return dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), metric=metric, cost=cost, seeds=np.array([[0.2, 0.25]], np.float32))


def test_reverse_vs_finite_differences():
    """dJ/dcost = lam * cost against central differences (h = 1e-3 relative) of
    the float64 oracle, J = sum of the values at receivers."""
    case = _small_riemann()
    n = int(case["dims"][0])
    rng = np.random.default_rng(11)
    recv = rng.choice(n * n, 6, replace=False)
    sens = np.zeros((n, n, 1), np.float32)
    sens.reshape(-1)[recv] = 1.0
    out = make_dictin(dict(case, sensitivity=sens)).Run()
    lam = out["costSensitivity"].cpu().numpy()[..., 0]
    grad = lam * case["cost"]
    tight = dict(atol=1e-13, rtol=1e-13)
    base = O.run(dict(case, **tight), np.float64)["values"].reshape(-1)[recv].sum()
    for idx in rng.choice(n * n, 12, replace=False):
        if grad.reshape(-1)[idx] == 0:
            continue
        hstep = 1e-3 * case["cost"].reshape(-1)[idx]
        vals = []
        for sgn in (1, -1):
            c2 = case["cost"].astype(np.float64).copy()
            c2.reshape(-1)[idx] += sgn * hstep
            vals.append(O.run(dict(case, cost=c2.astype(np.float32), **tight), np.float64)["values"]
                        .reshape(-1)[recv].sum())
        fd = (vals[0] - vals[1]) / (2 * hstep)
        assert abs(fd - grad.reshape(-1)[idx]) <= 2e-3 * abs(fd) + 1e-6 * abs(base), (idx, fd, grad.reshape(-1)[idx])


def test_autograd_function(monkeypatch):
    """The backward pass reverse-sweeps the flow recorded by the forward pass: one
    eikonal solve in all, and the gradient is the reference's costSensitivity
    times the cost."""
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    from adaptivegriddiscretizations_b200.autograd import eikonal_values
    case = _small_riemann(n=32)
    h = Eikonal.dictIn({k: case[k] for k in ("model", "dims", "gridScales", "origin", "metric", "seeds")}
                       | {"verbosity": 0})
    cost = torch.as_tensor(case["cost"], device="cuda").requires_grad_(True)
    solves = []
    solve = Interface.Solve
    monkeypatch.setattr(Interface, "Solve", lambda self: (solves.append(1), solve(self))[1])
    u = eikonal_values(h, cost)
    w = torch.zeros_like(u)
    w[-1, -1] = 1.0
    w[5, 20] = 2.0
    (u * w).sum().backward()
    assert len(solves) == 1, "the backward pass solved the eikonal equation again"
    monkeypatch.setattr(Interface, "Solve", solve)
    g = cost.grad.cpu().numpy()
    out = make_dictin(dict(case, sensitivity=w.cpu().numpy()[..., None])).Run()
    lam = out["costSensitivity"].cpu().numpy()[..., 0]
    np.testing.assert_allclose(g, lam * case["cost"], rtol=1e-5, atol=1e-7)
