"""GPU parity of the forward-mode variation (agd_forward, hfmOut['valueVariation']).

Against the reference's forward AD (its own linear kernel, golden fixtures),
the scaling identity (a cost varied by itself and seed values varied by
themselves vary the solution by itself), linearity in the variations, and the
adjoint identity <s, du> = <lam, rhs> with the reverse mode.
"""
import numpy as np
import pytest
import torch

from conftest import load_case, make_dictin

pytestmark = pytest.mark.gpu


def _forward_case(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    extra = {"costVariation": case.pop("costVariation"), "seedValueVariation": case.pop("seedValueVariation")}
    return case, extra, ref


@pytest.mark.parametrize("name", ["iso2", "riem2", "riem3"])
def test_forward_vs_reference(name):
    case, extra, ref = _forward_case(name)
    out = make_dictin(case, extra=extra).Run()
    vv = out["valueVariation"].cpu().numpy()
    want = ref["valueVariation"]
    assert vv.shape == want.shape
    assert np.abs(vv - want).max() <= 2e-4 * np.abs(want).max()
    assert out["stats"]["forwardAD"]["niter_o"] > 0


@pytest.mark.parametrize("name", ["iso2", "riem2"])
def test_forward_scaling_identity(name):
    """costVariation = cost and seedValueVariation = seedValues give
    valueVariation = values (tight tolerances: the identity holds at the fixed point)."""
    case, _, _ = _forward_case(name)
    shape = tuple(int(s) for s in case["dims"])
    cost = np.broadcast_to(np.asarray(case.get("cost", 1.0), np.float32), shape)
    extra = {"costVariation": cost[..., None].copy(),
             "seedValueVariation": np.asarray(case.get("seedValues", np.zeros(len(case["seeds"]))),
                                              np.float32)[None, :],
             "atol": 1e-8, "rtol": 1e-8, "exportValues": True}
    out = make_dictin(case, extra=extra).Run()
    u = out["values"].cpu().numpy()
    vv = out["valueVariation"].cpu().numpy()[..., 0]
    fin = np.isfinite(u)
    assert np.abs(vv[fin] - u[fin]).max() <= 2e-5 * np.abs(u[fin]).max()


def test_forward_linearity_and_adjoint_identity():
    """Variations a, b and a + 2b give du_a + 2 du_b; and <s, du> = <lam, rhs>
    for the reverse sensitivity lam of the receivers' indicator s."""
    case, extra, _ = _forward_case("riem2")
    cv = extra["costVariation"]
    sv = extra["seedValueVariation"]
    cv3 = np.concatenate([cv, cv[..., :1] + 2 * cv[..., 1:2]], -1)
    sv3 = np.concatenate([sv, sv[:1] + 2 * sv[1:2]], 0)
    shape = tuple(int(s) for s in case["dims"])
    rng = np.random.default_rng(5)
    sens = np.zeros(shape + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(shape)), 7, replace=False)] = 1.0
    out = make_dictin(case, extra={"costVariation": cv3, "seedValueVariation": sv3, "sensitivity": sens}).Run()
    vv = out["valueVariation"].cpu().numpy()
    comb = vv[..., 0] + 2 * vv[..., 1]
    assert np.abs(vv[..., 2] - comb).max() <= 1e-4 * np.abs(comb).max()
    # adjoint identity: sum_x s(x) du(x) = sum_x c(x) dc(x) lam(x) + sum_seeds dseed * seedSensitivity
    cost = np.broadcast_to(np.asarray(case.get("cost", 1.0), np.float32), shape)
    lam = out["costSensitivity"].cpu().numpy()[..., 0]
    seed_s = out["seedValueSensitivity"].cpu().numpy()[:, 0]
    for j in range(2):
        lhs = float((sens[..., 0] * vv[..., j]).sum())
        rhs = float((lam * cost * cv[..., j]).sum() + (seed_s * sv[j]).sum())
        assert abs(lhs - rhs) <= 1e-3 * max(abs(lhs), 1e-3)


def test_forward_only_seed_variation():
    """Only seedValueVariation given: the cost variation is zero."""
    case, extra, ref = _forward_case("iso2")
    out = make_dictin(case, extra={"seedValueVariation": extra["seedValueVariation"]}).Run()
    vv = out["valueVariation"].cpu().numpy()
    out2 = make_dictin(case, extra={"seedValueVariation": extra["seedValueVariation"],
                                    "costVariation": np.zeros_like(extra["costVariation"])}).Run()
    np.testing.assert_allclose(vv, out2["valueVariation"].cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_autograd_forward_mode():
    """torch.autograd.forward_ad through EikonalValues: the tangent of the values
    equals valueVariation, and <w, J t> = <J^T w, t> with the backward pass."""
    import torch.autograd.forward_ad as fwAD
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.autograd import eikonal_values
    case, _, _ = _forward_case("riem2")
    keys = ("model", "dims", "gridScales", "origin", "metric", "seeds", "seedValues")
    h = Eikonal.dictIn({k: case[k] for k in keys} | {"verbosity": 0})
    shape = tuple(int(s) for s in case["dims"])
    rng = np.random.default_rng(8)
    cost = torch.as_tensor(np.exp(0.2 * rng.standard_normal(shape)).astype(np.float32), device="cuda")
    t = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device="cuda")
    with fwAD.dual_level():
        u = eikonal_values(h, fwAD.make_dual(cost, t))
        jt = fwAD.unpack_dual(u).tangent
    ref = make_dictin(dict(case, cost=cost.cpu().numpy()),
                      extra={"costVariation": t.cpu().numpy()[..., None]}).Run()["valueVariation"][..., 0]
    # two solves, two schedules: agreement to the linear solver's tolerance
    torch.testing.assert_close(jt, ref, rtol=1e-4, atol=1e-4 * float(ref.abs().max()))
    w = torch.as_tensor(rng.standard_normal(shape).astype(np.float32), device="cuda")
    c = cost.clone().requires_grad_(True)
    (eikonal_values(h, c) * w).sum().backward()
    lhs, rhs = float((w * jt).sum()), float((c.grad * t).sum())
    assert abs(lhs - rhs) <= 1e-3 * max(abs(lhs), abs(rhs))


@pytest.mark.parametrize("name", ["riem2_radius", "iso2_radius"])
def test_spread_seed_variations(name):
    """Seeds spread over a radius: a unit variation of the seed value shifts every
    reachable value by 1 (forward), and the seed-value sensitivity of a sum of
    receivers is their number (reverse, aggregated over the spread points)."""
    case, _ = load_case(name)
    shape = tuple(int(s) for s in case["dims"])
    sens = np.zeros(shape + (1,), np.float32)
    rng = np.random.default_rng(4)
    sens.reshape(-1)[rng.choice(int(np.prod(shape)), 9, replace=False)] = 1.0
    out = make_dictin(case, extra={"seedValueVariation": np.ones((1, 1), np.float32), "sensitivity": sens,
                                   "exportValues": True}).Run()
    vv = out["valueVariation"].cpu().numpy()[..., 0]
    fin = np.isfinite(out["values"].cpu().numpy())
    assert np.abs(vv[fin] - 1.0).max() < 1e-4
    ss = out["seedValueSensitivity"].cpu().numpy()
    assert ss.shape == (1, 1)
    assert abs(ss[0, 0] - 9.0) < 1e-3
