"""GPU parity of the Rander2/3 models (a Riemannian metric plus a drift:
F(x) = |x|_M + <w, x>; the Riemann scheme on M^-1 with the neighbour values
shifted by -/+<w, e>, cuda/Riemann_.h:23-29, FiniteDifferences.h:41-45).

Against the golden outputs of the reference's own kernels built with the drift
(values, exported flow, geodesics, forward and reverse AD with the flow
normalisation of drift models, factorisation, second order, walls,
multiprecision), the float64 oracle's discrete solution on a larger seeded
case, and identities: a zero drift gives the Riemann solution, the dual metric
gives the same solution as the metric.
"""
import numpy as np
import pytest
import torch

from conftest import RANDER_CASES, load_case, make_dictin
from parity import REL, TIGHT, TIGHT_REL, assert_near_discrete, discrete_solution, rel_err

pytestmark = pytest.mark.gpu
_AD_KEYS = ("tips", "sensitivity", "costVariation", "seedValueVariation")


def _split(ref):
    L, G = ref["geodesic_lengths"], ref["geodesics_concat"]
    o, out = 0, []
    for l in L:
        out.append(G[:, o:o + l])
        o += l
    return out


@pytest.mark.parametrize("name", RANDER_CASES)
def test_values_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in _AD_KEYS}
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    if name.endswith("order2"):  # update-order dependence of the second order scheme
        fin = np.isfinite(ref["values"]) & (ref["values"] > 0)
        assert np.array_equal(np.isfinite(v), np.isfinite(ref["values"]))
        rel = np.abs(v - ref["values"])[fin] / ref["values"][fin]
        assert rel.max() < 6e-2 and rel.mean() < 4e-3
        return
    assert rel_err(v, ref["values"]) < (3e-5 if "factor" in name else REL)


def test_multiprecision_vs_reference():
    case, ref = load_case("rand2_mp")
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    assert rel_err(v, ref["values"]) < REL


@pytest.mark.parametrize("name", ["rand2", "rand3", "rand2_walls"])
def test_flow_geodesics_vs_reference(name):
    """The exported flow of a drift model is normalised by the metric norm of
    the flow (_PostProcess.py:80-92)."""
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("sensitivity", "costVariation", "seedValueVariation")}
    out = make_dictin(case, extra={"exportGeodesicFlow": True}).Run()
    flow = out["flow"].cpu().numpy()
    want = ref["flow_export"]
    fin = np.isfinite(want).all(0)
    assert np.abs(flow[:, fin] - want[:, fin]).max() <= 1e-3 * np.abs(want[:, fin]).max()
    assert list(out["geodesic_stopping_criteria"]) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    for g, w in zip(out["geodesics"], _split(ref)):
        g = g.cpu().numpy()
        assert abs(g.shape[1] - w.shape[1]) <= max(2, 0.02 * w.shape[1])
        m = min(g.shape[1], w.shape[1])
        assert np.abs(g[:, :m] - w[:, :m]).max() < 2e-3 * np.abs(w).max()


@pytest.mark.parametrize("name", ["rand2", "rand3"])
def test_reverse_ad_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "costVariation", "seedValueVariation")}
    out = make_dictin(case).Run()
    cs = out["costSensitivity"].cpu().numpy()
    want = ref["costSensitivity"]
    assert np.abs(cs - want).max() <= 1e-4 * np.abs(want).max()
    np.testing.assert_allclose(out["seedValueSensitivity"].cpu().numpy(), ref["seedValueSensitivity"],
                               rtol=1e-4, atol=1e-5)


def test_forward_ad_vs_reference():
    case, ref = load_case("rand2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    extra = {"costVariation": case.pop("costVariation"), "seedValueVariation": case.pop("seedValueVariation")}
    vv = make_dictin(case, extra=extra).Run()["valueVariation"].cpu().numpy()
    want = ref["valueVariation"]
    assert np.abs(vv - want).max() <= 2e-4 * np.abs(want).max()


def _rander_case(n, seed, wmax=0.6):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g1 = gaussian_filter(rng.standard_normal((n, n)), n / 24, mode="wrap")
    g2 = gaussian_filter(rng.standard_normal((n, n)), n / 24, mode="wrap")
    th = np.arctan2(g1, g2)
    lam = rng.uniform(1, 10.0, (n, n))
    c, s = np.cos(th), np.sin(th)
    M = np.stack([np.stack([c * c + lam * s * s, c * s * (1 - lam)], -1),
                  np.stack([c * s * (1 - lam), s * s + lam * c * c], -1)], -2)
    w = np.stack([gaussian_filter(rng.standard_normal((n, n)), n / 24, mode="wrap") for _ in range(2)], -1)
    wn = np.sqrt(np.einsum("...i,...ij,...j->...", w, np.linalg.inv(M), w))
    w = w / wn.max() * wmax
    flat = np.stack([M[..., 0, 0], M[..., 1, 0], M[..., 1, 1], w[..., 0], w[..., 1]], -1).astype(np.float32)
    return dict(model="Rander2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), metric=flat,
                seeds=rng.uniform(0.1, 0.9, (3, 2)).astype(np.float32))


def test_vs_discrete_solution():
    case = _rander_case(160, 5)
    exact = discrete_solution(case)
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    assert_near_discrete(v, case, exact)
    tight = make_dictin(case, extra=dict(TIGHT, exportValues=True)).Run()["values"].cpu().numpy()
    assert rel_err(tight, exact) < TIGHT_REL


def test_zero_drift_and_dual_metric():
    """A zero drift gives the Riemann2 solution of the same quadratic part; the
    dual metric (Rander.dual) gives the solution of the metric.  Tight
    tolerances: the same discrete scheme up to float32 rounding of the inputs."""
    from adaptivegriddiscretizations_b200 import Metrics
    case = _rander_case(96, 6)
    m = case.pop("metric")
    tight = dict(TIGHT, exportValues=True)
    zero = m.copy()
    zero[..., 3:] = 0
    vr = make_dictin(case, extra=dict(tight, metric=zero)).Run()["values"].cpu().numpy()
    riem = dict(case, model="Riemann2")
    vm = make_dictin(riem, extra=dict(tight, metric=zero[..., :3].copy())).Run()["values"].cpu().numpy()
    assert rel_err(vr, vm) < 2 * TIGHT_REL
    base = make_dictin(case, extra=dict(tight, metric=m)).Run()["values"].cpu().numpy()
    R = Metrics.Rander.from_HFM(m.astype(np.float64))
    D = R.dual()
    dual = np.moveaxis(D.flatten(), 0, -1).astype(np.float32)
    vd = make_dictin(case, extra=dict(tight, dualMetric=dual)).Run()["values"].cpu().numpy()
    assert rel_err(vd, base) < 4 * TIGHT_REL
    vo = make_dictin(case, extra=dict(tight, metric=R)).Run()["values"].cpu().numpy()
    assert rel_err(vo, base) < 2 * TIGHT_REL
