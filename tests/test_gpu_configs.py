"""The benchmark configurations at their full sizes, checked through properties
that hold at any size (seeded synthetic fields with the configurations'
shapes and distributions):

  * Isotropic2 256^2 (cost exp(0.5 g), g smoothed white noise of unit
    variance, sigma 8 px, one seed at the centre, tolerance 1e-6; the
    Isotropic scheme of cuda/Isotropic_.h:20-41): the parity criteria against
    the float64 oracle's discrete solution, through dictIn.Run;
  * Riemann2 1024^2 (angle field smoothed over 16 px, lambda in [1, 100], 4
    seeds) with geodesics from 64 tips: the parity criteria against the float64
    oracle's discrete solution, the stop codes of the oracle's geodesics, paths
    that start at their tip and end at a seed;
  * Riemann3 200^3 (eigenvalues log-uniform in [1, 25], orientations smoothed
    over 6 voxels, 1 source) with the reverse sensitivity of the sum of the
    arrival times at 128 receivers: against central differences (h = 1e-3 of
    the cost) of multiprecision solves at tight tolerances with float64 values,
    on 32 voxels drawn uniformly over the grid and on 8 voxels where the
    sensitivity is not negligible (4 drawn among them, the 4 largest);
  * 512 Isotropic2 / Riemann2 instances of sides 64 to 512 with 1 to 8 seeds,
    solved in one persistent launch replayed from a CUDA graph: every instance
    converges; after the replays, one instance of every side and model meets
    the parity criteria against the discrete solution.
"""
import os
import sys

import numpy as np
import pytest
import torch

from conftest import make_dictin
from parity import assert_near_discrete, discrete_solution

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def _riemann2(n, seed, nseeds=4, sigma=16.0):
    """The angle field smoothed over sigma pixels at 1024^2 (in proportion on
    smaller grids), lambda uniform in [1, 100], nseeds seeds."""
    import bench
    metrics, _ = bench.make_fields(n, 1, seed, sigma=sigma * n / 1024.0)
    seeds = np.random.default_rng(seed + 7).uniform(0.05, 0.95, (nseeds, 2)).astype(np.float32)
    return dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), metric=metrics[0], seeds=seeds)


def test_isotropic2_256_config():
    import bench
    case = bench.make_iso256(11)
    out = make_dictin(case, extra={"exportValues": True}).Run()
    assert out["keys"]["used"].count("tol") == 1
    v = out["values"].cpu().numpy()
    assert_near_discrete(v, case, discrete_solution(case, nthreads=os.cpu_count()))


def test_riemann2_1024_with_64_tips():
    from oracle import oracle as O
    n = 1024
    case = _riemann2(n, 21)
    tips = np.random.default_rng(22).uniform(0.02, 0.98, (64, 2)).astype(np.float32)
    out = make_dictin(case, extra={"tips": tips, "exportValues": True}).Run()
    v = out["values"].cpu().numpy()
    assert_near_discrete(v, case, discrete_solution(case, nthreads=os.cpu_count()))
    ref = O.run(dict(case, tips=tips), np.float32, nthreads=os.cpu_count())
    # lambda is drawn per pixel, so the flow is rough and many geodesics stop as
    # Stationnary (about half here, in the oracle's restatement of the
    # reference's ODE too); which test fires first depends on the last bits of
    # the flow: 60 of 64 stop codes agree.
    stops = list(out["geodesic_stopping_criteria"])
    assert sum(a == b for a, b in zip(stops, ref["geodesic_stopping_criteria"])) >= 60
    seeds = np.asarray(case["seeds"], np.float64)
    for g, tip, stop in zip(out["geodesics"], tips, stops):
        g = g.cpu().numpy()
        assert np.linalg.norm(g[:, 0] - tip) < 1e-5
        if stop == "AtSeed":  # the test fires within the target tolerance (6 pixels) of a seed
            assert np.min(np.linalg.norm(seeds - g[:, -1], axis=1)) < 8.0 / n


def test_riemann2_1024_geodesics_from_oracle_values():
    """The flow and geodesic kernels on the oracle's own float32 values of the
    Riemann2 1024^2 configuration (the solve replaced by them): all 64 stop
    codes are the oracle's, the paths within 1.5 grid steps of its paths and
    their lengths within 2 % (the oracle's threads update in an order that
    moves its values by a few 1e-6, and a path's last steps with them).  The
    stop codes that differ in the end-to-end test above come from the last
    bits of the solved values, not from the flow or the ODE."""
    import ctypes
    from oracle import oracle as O
    from adaptivegriddiscretizations_b200 import Eikonal, _lib
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    n = 1024
    case = _riemann2(n, 21)
    tips = np.random.default_rng(22).uniform(0.02, 0.98, (64, 2)).astype(np.float32)
    ref = O.run(dict(case, tips=tips), np.float32, nthreads=os.cpu_count())
    itf = Interface(Eikonal.dictIn(dict(case, mode="gpu", verbosity=0, tips=tips)))
    itf.SetKernelTraits()
    itf.SetGeometry()
    itf.SetArgs()
    v = torch.as_tensor(np.ascontiguousarray(ref["values"], np.float32), device="cuda").reshape(-1)
    _lib.check(_lib.lib().agd_block_expand(itf.ndim, itf.c_shape, itf.c_shape_i, 1, _lib.ptr(v), 0,
                                           ctypes.c_float(float("inf")), _lib.ptr(itf.values_t), itf.stream))
    itf.PostProcess()
    itf.GetGeodesics()
    assert list(itf.hfmOut["geodesic_stopping_criteria"]) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    dev, dlen = [], []
    for g, w in zip(itf.hfmOut["geodesics"], ref["geodesics"]):
        g = g.cpu().numpy()
        m = min(g.shape[1], w.shape[1])
        dev.append(np.abs(g[:, :m] - w[:, :m]).max())
        dlen.append(abs(g.shape[1] - w.shape[1]) / w.shape[1])
    print("path deviation", max(dev) * n, "grid steps; length difference", max(dlen))
    assert max(dev) < 1.5 / n and max(dlen) < 0.02


def _riemann3_200(seed):
    from scipy.ndimage import gaussian_filter
    n = 200
    rng = np.random.default_rng(seed)
    # orientations: unit quaternions, uniformly random, smoothed over 6 voxels
    q = gaussian_filter(rng.standard_normal((4, n, n, n)).astype(np.float32), (0, 6, 6, 6), mode="wrap")
    q /= np.linalg.norm(q, axis=0, keepdims=True)
    w, x, y, z = q
    rot = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
                    np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
                    np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], -2)
    del q, w, x, y, z
    ev = np.exp(rng.uniform(0, np.log(25.0), (n, n, n, 3))).astype(np.float32)
    M = rot @ (ev[..., :, None] * np.swapaxes(rot, -1, -2))
    metric = np.stack([M[..., i, j] for i in range(3) for j in range(i + 1)], -1).astype(np.float32)
    cost = np.ones((n, n, n), np.float32)
    return dict(model="Riemann3", dims=np.array([n] * 3, np.float32), gridScales=np.full(3, 1.0 / n, np.float32),
                origin=np.zeros(3, np.float32), metric=metric, cost=cost,
                seeds=np.array([[0.5, 0.5, 0.5]], np.float32))


def test_riemann3_200_reverse_vs_finite_differences():
    case = _riemann3_200(31)
    n = 200
    rng = np.random.default_rng(32)
    recv = rng.choice(n ** 3, 128, replace=False)
    sens = np.zeros((n, n, n, 1), np.float32)
    sens.reshape(-1)[recv] = 1.0
    out = make_dictin(dict(case, sensitivity=sens)).Run()
    lam = out["costSensitivity"].cpu().numpy()[..., 0].reshape(-1)
    grad = lam * case["cost"].reshape(-1)  # dJ/dcost = lam * cost
    # multiprecision at tight tolerances, values exported in float64, resolves the
    # 1e-3 perturbations (the float32 values would round them away)
    tight = {"values_float64": True, "atol": 1e-12, "rtol": 0.0}
    flat_recv = torch.as_tensor(recv, device="cuda")

    def J(cost):
        u = make_dictin(dict(case, cost=cost), extra=dict(tight, exportValues=True)).Run()["values"]
        return float(u.double().reshape(-1)[flat_recv].sum())

    # 32 voxels drawn uniformly over the grid (most have no receiver downstream,
    # so the difference quotient must vanish there too), and voxels where the
    # sensitivity is not negligible: 4 drawn among them, the 4 largest
    gmax = np.abs(grad).max()
    voxels = list(rng.choice(n ** 3, 32, replace=False)) + \
        list(rng.choice(np.flatnonzero(np.abs(grad) > 1e-2 * gmax), 4, replace=False)) + \
        list(np.argsort(-np.abs(grad))[:4])
    for idx in voxels:
        h = 1e-3 * case["cost"].reshape(-1)[idx]
        vals = []
        for sgn in (1, -1):
            c2 = case["cost"].copy()
            c2.reshape(-1)[idx] += sgn * h
            vals.append(J(c2))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - grad[idx]) <= 2e-2 * abs(grad[idx]) + 1e-4 * gmax, (idx, fd, grad[idx])


def test_batched_512_mixed_cuda_graph():
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import BatchPlan, Interface
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(41)
    cases = []
    for i in range(512):
        n = int(rng.choice([64, 128, 256, 384, 512]))
        nseeds = int(rng.integers(1, 9))
        if rng.uniform() < 0.5:
            c = _riemann2(n, 1000 + i, nseeds=nseeds)
        else:
            g = gaussian_filter(rng.standard_normal((n, n)), 8.0 * n / 256, mode="wrap")
            c = dict(model="Isotropic2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                     origin=np.zeros(2, np.float32), cost=np.exp(0.5 * g / g.std()).astype(np.float32),
                     seeds=rng.uniform(0.05, 0.95, (nseeds, 2)).astype(np.float32))
        cases.append(c)
    itfs = []
    for c in cases:
        it = Interface(make_dictin(c, extra={"exportValues": True}))
        it.SetKernelTraits()
        it.SetGeometry()
        it.SetArgs()
        itfs.append(it)
    plan = BatchPlan(itfs)
    inf = float("inf")

    def step():
        for it in itfs:
            it.values_t.fill_(inf)
        plan.run()

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        step()  # warm up outside the capture
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    for _ in range(2):
        graph.replay()
    torch.cuda.synchronize()
    niter, status, visits = plan.read_stats()
    assert not status.any() and (niter > 0).all()
    # one instance of every side and model, after the graph replays
    sample = {}
    for i, c in enumerate(cases):
        sample.setdefault((int(c["dims"][0]), c["model"]), i)
    assert len(sample) == 10
    for i in sample.values():
        it = itfs[i]
        v = it.squeeze(it.values_t).cpu().numpy()
        assert_near_discrete(v, cases[i])
