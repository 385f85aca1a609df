"""BatchSolver (repeated batched solves of one configuration): every instance
of a batch must give the values of the reference's own kernels (golden case,
1e-5 relative) or the scheme's discrete solution (seeded cases, the criteria
of parity.py) for that instance, on two submissions in a row, from host
(page-locked or not) and from device inputs."""
import numpy as np
import pytest
import torch

from conftest import load_case
from parity import TIGHT, TIGHT_REL, assert_near_discrete, discrete_solution

pytestmark = pytest.mark.gpu
REL = 1e-5


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), "finite masks differ"
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


def _template(case):
    from adaptivegriddiscretizations_b200 import Eikonal
    keys = ("model", "dims", "gridScales", "origin", "atol", "rtol")
    return Eikonal.dictIn({"mode": "gpu", "verbosity": 0, **{k: case[k] for k in keys if k in case}})


def _riemann_fields(n, batch, seed, nseeds=3, nd=2):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    ms, ss = [], []
    for _ in range(batch):
        if nd == 2:
            g1 = gaussian_filter(rng.standard_normal((n, n)), n / 32, mode="wrap")
            g2 = gaussian_filter(rng.standard_normal((n, n)), n / 32, mode="wrap")
            th = np.arctan2(g1, g2)
            lam = rng.uniform(1, 30, (n, n))
            c, s = np.cos(th), np.sin(th)
            ms.append(np.stack([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], -1))
        else:
            a = rng.standard_normal((n, n, n, 3, 3)) * 0.3
            m = np.eye(3) + np.einsum("...ij,...kj->...ik", a, a)
            ms.append(np.stack([m[..., 0, 0], m[..., 1, 0], m[..., 1, 1], m[..., 2, 0], m[..., 2, 1], m[..., 2, 2]],
                               -1))
        ss.append(rng.uniform(0.1, 0.9, (nseeds, nd)))
    return np.stack(ms).astype(np.float32), np.stack(ss).astype(np.float32)


def _case(model, n, m, seeds, cost=None):
    nd = int(model[-1])
    c = dict(model=model, dims=np.full(nd, n, np.float32), gridScales=np.full(nd, 1.0 / n, np.float32),
             origin=np.zeros(nd, np.float32), seeds=seeds)
    if m is not None:
        c["metric"] = m
    if cost is not None:
        c["cost"] = cost
    return c


def test_golden_case_twice_in_a_row():
    from adaptivegriddiscretizations_b200 import Eikonal
    case, ref = load_case("riem2")
    B = 3
    solver = Eikonal.BatchSolver(_template(case), B)
    metric = torch.from_numpy(np.stack([case["metric"]] * B)).pin_memory()
    seeds = torch.from_numpy(np.stack([case["seeds"]] * B)).pin_memory()
    vals = torch.from_numpy(np.stack([case["seedValues"]] * B)).pin_memory()
    outs = [torch.empty((B,) + ref["values"].shape).pin_memory() for _ in range(2)]
    jobs = [solver.submit(metric=metric, seeds=seeds, seedValues=vals, out=o) for o in outs]
    for job in jobs:
        v = job.result().numpy()
        for i in range(B):
            assert _rel(v[i], ref["values"]) < REL
        assert (job.niter_o > 0).all() and (job.tile_visits > 0).all()


def test_riemann2_batch_vs_oracle_host_and_device_inputs():
    from adaptivegriddiscretizations_b200 import Eikonal
    n, B = 96, 4
    ms, ss = _riemann_fields(n, B, 11)
    solver = Eikonal.BatchSolver(_template(_case("Riemann2", n, None, ss[0])), B)
    v_host = solver.solve(metric=ms, seeds=ss).cpu().numpy()  # pageable numpy inputs
    v_dev = solver.solve(metric=torch.from_numpy(ms).cuda(), seeds=torch.from_numpy(ss).cuda()).cpu().numpy()
    tight = Eikonal.BatchSolver(_template(dict(_case("Riemann2", n, None, ss[0]), **TIGHT)), B)
    v_tight = tight.solve(metric=ms, seeds=ss).cpu().numpy()
    for i in range(B):
        case = _case("Riemann2", n, ms[i], ss[i])
        exact = discrete_solution(case)
        assert_near_discrete(v_host[i], case, exact)
        assert_near_discrete(v_dev[i], case, exact)
        assert _rel(v_tight[i], exact) < TIGHT_REL


def test_isotropic2_per_instance_cost_tolerance():
    from adaptivegriddiscretizations_b200 import Eikonal
    from scipy.ndimage import gaussian_filter
    n, B = 80, 3
    rng = np.random.default_rng(12)
    costs = np.stack([np.exp(gaussian_filter(rng.standard_normal((n, n)), 3.0)) * (i + 1) for i in range(B)])
    costs = costs.astype(np.float32)
    seeds = rng.uniform(0.1, 0.9, (B, 2, 2)).astype(np.float32)
    solver = Eikonal.BatchSolver(_template(_case("Isotropic2", n, None, seeds[0])), B)
    v = solver.solve(cost=costs, seeds=seeds).cpu().numpy()
    for i in range(B):
        assert_near_discrete(v[i], _case("Isotropic2", n, None, seeds[i], cost=costs[i]))


def test_riemann3_batch_vs_oracle():
    from adaptivegriddiscretizations_b200 import Eikonal
    n, B = 24, 2
    ms, ss = _riemann_fields(n, B, 13, nseeds=2, nd=3)
    solver = Eikonal.BatchSolver(_template(_case("Riemann3", n, None, ss[0])), B)
    v = solver.solve(metric=ms, seeds=ss).cpu().numpy()
    for i in range(B):
        assert_near_discrete(v[i], _case("Riemann3", n, ms[i], ss[i]))


def test_seeds_outside_the_domain():
    from adaptivegriddiscretizations_b200 import Eikonal
    n, B = 32, 2
    ms, ss = _riemann_fields(n, B, 14, nseeds=1)
    solver = Eikonal.BatchSolver(_template(_case("Riemann2", n, None, ss[0])), B)
    bad = ss.copy()
    bad[1, 0, 0] = 1.5
    with pytest.raises(ValueError, match="outside"):
        solver.submit(metric=ms, seeds=bad)
    job = solver.submit(metric=torch.from_numpy(ms).cuda(), seeds=torch.from_numpy(bad).cuda())
    with pytest.raises(ValueError, match="outside"):
        job.result()
    v = solver.solve(metric=ms, seeds=ss)  # the solver stays usable
    assert torch.isfinite(v).all()
