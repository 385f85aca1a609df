"""The batched serving path (BatchSolver, and SubmitBatch's uniform batches)
for the Diagonal and Rander models and for obstacles, shared by the batch or
per instance.  Each instance must give the values of the reference's own
kernels for it (golden fixtures, 2e-5 relative), and a metric scaled by 4
(costs by 2, Rander drift by 2) with seed values doubled must double them."""
import numpy as np
import pytest
import torch

from conftest import load_case

pytestmark = pytest.mark.gpu
# Two instances solved together stop at other points of the stopping tolerance
# than the reference's run of one (the order of the visits differs), so the
# bound is twice that of the single-instance golden tests.
REL = 2e-5
DATA = ("metric", "cost", "seeds", "seedValues", "walls", "tips", "sensitivity", "costVariation",
        "seedValueVariation")


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), "finite masks differ"
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


def _template(case, walls=True):
    from adaptivegriddiscretizations_b200 import Eikonal
    d = {"mode": "gpu", "verbosity": 0}
    for k, v in case.items():
        if k not in DATA or (walls and k == "walls"):
            d[k] = v
    return Eikonal.dictIn(d)


def _scaled(case):
    """Metric of the case scaled so that its distances double, seed values doubled."""
    model = case["model"]
    m = np.array(case["metric"], np.float32)
    nd = int(model[-1])
    sd = nd * (nd + 1) // 2
    if model.startswith("Riemann"):
        m = 4 * m
    elif model.startswith("Diagonal"):
        m = 2 * m
    else:  # Rander: F(v) = sqrt(<v, m v>) + <w, v>
        m[..., :sd] *= 4
        m[..., sd:] *= 2
    sv = 2 * np.asarray(case.get("seedValues", np.zeros(len(case["seeds"]))), np.float32)
    return m, sv


def _stack(case, key):
    a = np.asarray(case[key], np.float32)
    return np.stack([a, a])


@pytest.mark.parametrize("name", ["diag2", "diag3", "rand2", "rand3"])
def test_batch_solver_diagonal_rander(name):
    from adaptivegriddiscretizations_b200 import Eikonal
    case, ref = load_case(name)
    m2, sv2 = _scaled(case)
    solver = Eikonal.BatchSolver(_template(case), 2)
    sv = np.asarray(case.get("seedValues", np.zeros(len(case["seeds"]))), np.float32)
    for rep in range(2):  # the second submission reuses the buffers and plan
        kw = dict(metric=np.stack([np.asarray(case["metric"], np.float32), m2]),
                  seeds=_stack(case, "seeds"), seedValues=np.stack([sv, sv2]))
        if "cost" in case:
            kw["cost"] = _stack(case, "cost")
        out = solver.solve(**kw).cpu().numpy()
        assert _rel(out[0], ref["values"]) < REL
        assert _rel(out[1], 2 * np.asarray(ref["values"], np.float64)) < REL


@pytest.mark.parametrize("name", ["riem2_walls", "iso2_walls", "diag2_walls", "rand2_walls", "riem3_walls"])
@pytest.mark.parametrize("where", ["template", "instances"])
def test_batch_solver_walls(name, where):
    """Obstacles in the template (one wall distance map for the batch) or given
    per instance at submission (batched distance maps)."""
    from adaptivegriddiscretizations_b200 import Eikonal
    case, ref = load_case(name)
    solver = Eikonal.BatchSolver(_template(case, walls=where == "template"), 2)
    kw = dict(seeds=_stack(case, "seeds"))
    if "seedValues" in case:
        kw["seedValues"] = _stack(case, "seedValues")
    for k in ("metric", "cost"):
        if k in case:
            kw[k] = _stack(case, k)
    if where == "instances":
        kw["walls"] = np.stack([case["walls"], case["walls"]])
    job = solver.submit(**kw)
    out = job.result().cpu().numpy()
    for i in range(2):
        assert _rel(out[i], ref["values"]) < REL
    # the first epoch holds the tiles of the seeds alone (not those of the wall
    # points, which are seeds of value +inf): the trigger of each instance
    trig = solver._bufs[0].trigger.cpu().numpy()
    idx = np.round((np.asarray(case["seeds"], np.float32) - solver.start) / solver.h).astype(int)  # as submit()
    shape_o = [(s + t - 1) // t for s, t in zip(solver.shape, solver.shape_i)]
    want = np.zeros(int(np.prod(shape_o)), np.uint8)
    want[np.ravel_multi_index((idx // np.array(solver.shape_i)).T, shape_o)] = 1
    for i in range(2):
        np.testing.assert_array_equal(trig[i], want)


@pytest.mark.parametrize("name", ["diag2", "rand2", "riem2_walls"])
def test_submit_batch_uniform_models(name):
    """SubmitBatch of dictIn that differ only in their data: the batched
    preparation path for these models (and shared walls)."""
    from adaptivegriddiscretizations_b200 import Eikonal
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import UniformBatchJob
    case, ref = load_case(name)
    hs = []
    for _ in range(3):
        d = {"mode": "gpu", "verbosity": 0, "exportValues": True}
        d.update({k: v for k, v in case.items() if k not in ("tips", "sensitivity", "costVariation",
                                                                "seedValueVariation")})
        hs.append(Eikonal.dictIn(d))
    job = Eikonal.SubmitBatch(hs)
    assert isinstance(job, UniformBatchJob)
    for o in job.result():
        assert _rel(o["values"].cpu().numpy(), ref["values"]) < REL
    torch.cuda.synchronize()
