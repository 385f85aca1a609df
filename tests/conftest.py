import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built CUDA library")


def load_case(name):
    """Golden fixture -> (dictIn-like case dict, reference outputs dict)."""
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = {k[3:]: d[k] for k in d.files if k.startswith("in_")}
    case["model"] = str(case["model"])
    if "traits_shape_i" in case:
        case["traits"] = dict(shape_i=tuple(int(s) for s in case.pop("traits_shape_i")),
                              niter_i=int(case.pop("traits_niter_i")))
    if "multiprecision" in case:
        case["multiprecision"] = bool(case["multiprecision"])
    for k in ("seedRadius", "factoringRadius"):
        if k in case:
            case[k] = float(case[k])
    if "order" in case:
        case["order"] = int(case["order"])
    out = {k[4:]: d[k] for k in d.files if k.startswith("out_")}
    return case, out


CASES = ["iso2", "riem2", "riem2_aniso", "iso3", "riem3", "ad_notebook"]
RADIUS_CASES = ["riem2_radius", "iso2_radius"]  # seeds spread over a radius (values only)
FACTOR_CASES = ["riem2_factor", "iso2_factor"]  # source factorisation (factoringRadius)
ORDER2_CASES = ["riem2_order2", "iso2_order2", "riem3_order2"]  # second order scheme (order: 2)
# the second order scheme with source factorisation, with multiprecision, and with both
ORDER2_FACTOR_CASES = ["riem2_order2_factor", "iso2_order2_factor", "riem3_order2_factor"]
ORDER2_MP_CASES = ["riem2_order2_mp", "iso2_order2_mp", "riem3_order2_mp",
                   "riem2_order2_factor_mp", "iso2_order2_factor_mp", "riem3_order2_factor_mp"]
WALL_CASES = ["riem2_walls", "iso2_walls", "riem3_walls"]  # obstacles (walls, wallDistBound)
DIAG_CASES = ["diag2", "diag2_factor", "diag2_order2", "diag2_walls", "diag3"]  # Diagonal2/3 models
RANDER_CASES = ["rand2", "rand2_factor", "rand2_order2", "rand2_walls", "rand3"]  # Rander2/3 (drift)


@pytest.fixture(params=CASES)
def golden_case(request):
    return (request.param,) + load_case(request.param)


def make_dictin(case, mode="gpu", extra=None):
    """dictIn for the package under test from a golden-case dict."""
    from adaptivegriddiscretizations_b200 import Eikonal
    d = {"model": case["model"], "mode": mode, "arrayOrdering": "RowMajor", "verbosity": 0}
    for k in ("dims", "gridScales", "origin", "seeds", "seedValues", "cost", "tips", "traits", "sensitivity",
              "seedRadius", "factoringRadius", "order", "walls", "wallDistBound", "pastseed_delay", "tol"):
        if k in case:
            d[k] = case[k]
    if "metric" in case:
        d["metric"] = np.asarray(case["metric"], np.float32)
    if extra:
        d.update(extra)
    return Eikonal.dictIn(d)


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False
