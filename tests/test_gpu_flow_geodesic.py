"""GPU parity of the upwind flow and of geodesic backtracking.

Flow vectors and weight sums against the reference's golden flow pass; geodesic
stop codes, lengths and paths against the reference's golden geodesics.
"""
import numpy as np
import pytest
import torch

from conftest import CASES, ORDER2_CASES, load_case, make_dictin

pytestmark = pytest.mark.gpu
GEO_CASES = [c for c in CASES if c != "ad_notebook"] + ["riem2_factor", "riem2_pastseed"]


def _split(ref):
    L, G = ref["geodesic_lengths"], ref["geodesics_concat"]
    o, out = 0, []
    for l in L:
        out.append(G[:, o:o + l])
        o += l
    return out


@pytest.mark.parametrize("name", GEO_CASES)
def test_flow_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportGeodesicFlow": True, "exportValues": True}).Run()
    flow = out["flow"].cpu().numpy()  # physical units: -h * flow_vector
    h = np.asarray(case["gridScales"], np.float32).reshape((-1,) + (1,) * len(case["dims"]))
    want = -h * ref["flow_vector"]
    scale = np.abs(want).max()
    assert flow.shape == want.shape
    # the flow weights are products of (u - v) differences: float32 cancellation
    assert np.abs(flow - want).max() <= 1e-3 * scale


@pytest.mark.parametrize("name", GEO_CASES)
def test_geodesics_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k != "sensitivity"}
    out = make_dictin(case).Run()
    stops = out["geodesic_stopping_criteria"]
    assert list(stops) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    for g, want in zip(out["geodesics"], _split(ref)):
        g = g.cpu().numpy()
        assert g.shape[0] == want.shape[0]
        # paths follow the same cells; lengths may differ by a few steps at the seed
        assert abs(g.shape[1] - want.shape[1]) <= max(2, 0.02 * want.shape[1])
        m = min(g.shape[1], want.shape[1])
        assert np.abs(g[:, :m] - want[:, :m]).max() < 2e-3 * np.abs(want).max()
        assert np.linalg.norm(g[:, -1] - want[:, -1]) < 3 * float(np.max(case["gridScales"]))


@pytest.mark.parametrize("name", ORDER2_CASES)
def test_geodesics_order2(name):
    """Second order: the values depend on the order of the in-tile updates (see
    test_values_vs_reference), so the paths are compared by their stop codes and
    their ends, which must reach the seed."""
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k != "sensitivity"}
    out = make_dictin(case).Run()
    assert list(out["geodesic_stopping_criteria"]) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    for g, want in zip(out["geodesics"], _split(ref)):
        g = g.cpu().numpy()
        assert np.linalg.norm(g[:, -1] - want[:, -1]) < 3 * float(np.max(case["gridScales"]))
        assert np.linalg.norm(g[:, 0] - want[:, 0]) < 1e-5


@pytest.mark.parametrize("name", ["iso2", "iso3", "riem2", "riem3", "riem2_walls"])
def test_active_neighs_vs_reference(name):
    """exportActiveNeighs: bit k set where the k-th finite difference has a
    positive flow weight.  A weight is a difference of two nearly equal values
    where the upwind direction is ambiguous, so the masks may differ at such
    points: at most 0.5 % of them, and the bits are those of the exported
    flow weights' signs."""
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportActiveNeighs": True}).Run()
    bits = out["activeNeighs"].cpu().numpy()
    assert bits.dtype == np.int32 and bits.shape == ref["activeNeighs"].shape
    assert (bits != ref["activeNeighs"]).mean() <= 5e-3
    assert "exportActiveNeighs" in out["keys"]["used"]
