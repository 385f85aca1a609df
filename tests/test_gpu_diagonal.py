"""GPU parity of the Diagonal2/3 models (axis costs per point, the Isotropic
scheme with per-point weights, cuda/Isotropic_.h:32-36).

Against the golden outputs of the reference's own Diagonal kernels (values,
flow, geodesics, forward and reverse AD, with factorisation, second order and
walls), the float64 oracle's discrete solution on larger seeded cases, and the
identities between inputs: the dual metric, a constant metric, a
Metrics.Diagonal object, equal costs against the Isotropic model.
"""
import numpy as np
import pytest
import torch

from conftest import DIAG_CASES, load_case, make_dictin
from parity import REL, TIGHT, TIGHT_REL, assert_near_discrete, discrete_solution, rel_err

pytestmark = pytest.mark.gpu


def _split(ref):
    L, G = ref["geodesic_lengths"], ref["geodesics_concat"]
    o, out = 0, []
    for l in L:
        out.append(G[:, o:o + l])
        o += l
    return out


@pytest.mark.parametrize("name", DIAG_CASES)
def test_values_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity", "costVariation",
                                                       "seedValueVariation")}
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    if name.endswith("order2"):  # update-order dependence of the second order scheme
        fin = np.isfinite(ref["values"]) & (ref["values"] > 0)
        assert np.array_equal(np.isfinite(v), np.isfinite(ref["values"]))
        rel = np.abs(v - ref["values"])[fin] / ref["values"][fin]
        assert rel.max() < 6e-2 and rel.mean() < 4e-3
        return
    assert rel_err(v, ref["values"]) < (3e-5 if "factor" in name else REL)


@pytest.mark.parametrize("name", ["diag2", "diag3", "diag2_walls"])
def test_flow_geodesics_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("sensitivity", "costVariation", "seedValueVariation")}
    out = make_dictin(case, extra={"exportGeodesicFlow": True}).Run()
    flow = out["flow"].cpu().numpy()
    h = np.asarray(case["gridScales"], np.float32).reshape((-1,) + (1,) * len(case["dims"]))
    want = -h * ref["flow_vector"]
    assert np.abs(flow - want).max() <= 1e-3 * np.abs(want).max()
    assert list(out["geodesic_stopping_criteria"]) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    for g, w in zip(out["geodesics"], _split(ref)):
        g = g.cpu().numpy()
        assert abs(g.shape[1] - w.shape[1]) <= max(2, 0.02 * w.shape[1])
        m = min(g.shape[1], w.shape[1])
        assert np.abs(g[:, :m] - w[:, :m]).max() < 2e-3 * np.abs(w).max()


@pytest.mark.parametrize("name", ["diag2", "diag3"])
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
    case, ref = load_case("diag2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    extra = {"costVariation": case.pop("costVariation"), "seedValueVariation": case.pop("seedValueVariation")}
    vv = make_dictin(case, extra=extra).Run()["valueVariation"].cpu().numpy()
    want = ref["valueVariation"]
    assert np.abs(vv - want).max() <= 2e-4 * np.abs(want).max()


def _diag_case(shape, seed, nseeds=2):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    nd = len(shape)
    costs = []
    for k in range(nd):
        g = gaussian_filter(rng.standard_normal(shape), 4.0, mode="wrap")
        costs.append(np.exp(0.5 * (g - g.mean()) / g.std()) * (1.0 + k))
    return dict(model=f"Diagonal{nd}", dims=np.array(shape, np.float32),
                gridScales=np.full(nd, 1.0 / shape[0], np.float32), origin=np.zeros(nd, np.float32),
                metric=np.stack(costs, -1).astype(np.float32),
                seeds=rng.uniform(0.1, 0.9, (nseeds, nd)).astype(np.float32) * np.array(shape) / shape[0])


@pytest.mark.parametrize("make", [lambda: _diag_case((200, 150), 3), lambda: _diag_case((40, 36, 44), 4)],
                         ids=["diag2_200x150", "diag3_40"])
def test_vs_discrete_solution(make):
    case = make()
    exact = discrete_solution(case)
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    assert_near_discrete(v, case, exact)
    tight = make_dictin(case, extra=dict(TIGHT, exportValues=True)).Run()["values"].cpu().numpy()
    assert rel_err(tight, exact) < TIGHT_REL
    mp = make_dictin(case, extra=dict(TIGHT, exportValues=True, multiprecision=True)).Run()["values"].cpu().numpy()
    assert rel_err(mp, exact) < TIGHT_REL


def test_metric_forms():
    """One problem, four inputs: the costs, the dual metric (1/costs), a
    Metrics.Diagonal object, and (for equal costs c on both axes) the Isotropic
    model with cost c; a constant metric against the same metric as a field.
    Each is a float32 rounding of the same discrete scheme, solved to tight
    tolerances: within two float32 parity bars of one another."""
    from adaptivegriddiscretizations_b200 import Metrics
    case = _diag_case((96, 80), 7)
    m = case.pop("metric")
    tight = dict(TIGHT, exportValues=True)
    base = make_dictin(case, extra=dict(tight, metric=m)).Run()["values"].cpu().numpy()
    v = make_dictin(case, extra=dict(tight, dualMetric=(1.0 / m).astype(np.float32))).Run()["values"]
    assert rel_err(v.cpu().numpy(), base) < 2 * TIGHT_REL
    v = make_dictin(case, extra=dict(tight, metric=Metrics.Diagonal(np.moveaxis(m, -1, 0)))).Run()["values"]
    assert rel_err(v.cpu().numpy(), base) < 2 * TIGHT_REL
    c = np.exp(np.random.default_rng(1).uniform(-0.3, 0.3, (96, 80))).astype(np.float32)
    iso = dict(model="Isotropic2", dims=case["dims"], gridScales=case["gridScales"], origin=case["origin"],
               seeds=case["seeds"], cost=c, traits={"shape_i": (16, 16), "niter_i": 16})
    vi = make_dictin(iso, extra=tight).Run()["values"].cpu().numpy()
    vd = make_dictin(case, extra=dict(tight, metric=np.stack([c, c], -1))).Run()["values"].cpu().numpy()
    assert rel_err(vd, vi) < 2 * TIGHT_REL
    vc = make_dictin(case, extra=dict(tight, metric=np.array([1.0, 2.5], np.float32))).Run()["values"]
    full = np.broadcast_to(np.array([1.0, 2.5], np.float32), (96, 80, 2)).copy()
    vf = make_dictin(case, extra=dict(tight, metric=full)).Run()["values"].cpu().numpy()
    assert rel_err(vc.cpu().numpy(), vf) < 2 * TIGHT_REL


def test_active_neighs_vs_reference():
    case, ref = load_case("diag2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity", "costVariation",
                                                       "seedValueVariation")}
    bits = make_dictin(case, extra={"exportActiveNeighs": True}).Run()["activeNeighs"].cpu().numpy()
    assert (bits != ref["activeNeighs"]).mean() <= 5e-3
