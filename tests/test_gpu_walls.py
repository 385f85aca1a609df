"""GPU parity of obstacles (walls, wallDistBound).

Against: the golden outputs of the reference's own kernels built with walls
(values, flow, geodesics, the wall distance map bit for bit), and the float64
oracle's discrete solution on larger seeded cases, including walls combined
with source factorisation and multiprecision.  Walls are +inf seeds, and a
neighbour whose segment meets a wall reads +inf (cuda/Walls.h:18-50).
"""
import ctypes

import numpy as np
import pytest
import torch

from conftest import WALL_CASES, load_case, make_dictin
from parity import REL, TIGHT, TIGHT_REL, assert_near_discrete, discrete_solution, rel_err

pytestmark = pytest.mark.gpu


def _split(ref):
    L, G = ref["geodesic_lengths"], ref["geodesics_concat"]
    o, out = 0, []
    for l in L:
        out.append(G[:, o:o + l])
        o += l
    return out


@pytest.mark.parametrize("name", WALL_CASES)
def test_wall_distance_bitexact(name):
    """agd_prep_walls: the wall distance map equals the reference's, and the
    wall points become seeds of value +inf."""
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k != "tips"}
    it = Interface(make_dictin(case))
    it.SetKernelTraits()
    it.SetGeometry()
    it.SetArgs()
    # the map is in tile layout: back to the grid through a float copy
    wd = it.squeeze(it.wall_dist.float().contiguous()).cpu().numpy()
    assert np.array_equal(wd.astype(np.uint8), ref["wall_dist"])
    rhs = it.squeeze(it.rhs_t).cpu().numpy()
    walls = np.asarray(case["walls"], bool)
    assert np.isinf(rhs[walls]).all() and np.isfinite(rhs[~walls]).all()
    bits = np.unpackbits(it.seedbits.cpu().numpy(), bitorder="little").astype(np.float32)
    bits_t = torch.as_tensor(bits, device="cuda")
    seeds = it.squeeze(bits_t).cpu().numpy().astype(bool)
    assert seeds[walls].all()


@pytest.mark.parametrize("name", WALL_CASES)
def test_values_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k != "tips"}
    out = make_dictin(case, extra={"exportValues": True}).Run()
    v = out["values"].cpu().numpy()
    assert rel_err(v, ref["values"]) < REL
    walls = np.asarray(case["walls"], bool)
    assert np.isinf(v[walls]).all()


@pytest.mark.parametrize("name", WALL_CASES)
def test_flow_and_geodesics_vs_reference(name):
    case, ref = load_case(name)
    out = make_dictin(case, extra={"exportGeodesicFlow": True}).Run()
    flow = out["flow"].cpu().numpy()
    h = np.asarray(case["gridScales"], np.float32).reshape((-1,) + (1,) * len(case["dims"]))
    want = -h * ref["flow_vector"]
    assert np.abs(flow - want).max() <= 1e-3 * np.abs(want).max()
    if "tips" not in case:
        return
    assert list(out["geodesic_stopping_criteria"]) == [str(s) for s in ref["geodesic_stopping_criteria"]]
    for g, w in zip(out["geodesics"], _split(ref)):
        g = g.cpu().numpy()
        assert abs(g.shape[1] - w.shape[1]) <= max(2, 0.02 * w.shape[1])
        m = min(g.shape[1], w.shape[1])
        assert np.abs(g[:, :m] - w[:, :m]).max() < 2e-3 * np.abs(w).max()


def _walled_riemann2(n, seed, nseeds=1, lam_max=30.0, sigma=1 / 32):
    """Seeded Riemann2 case with a long wall with two gaps and a ring-shaped wall."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g1 = gaussian_filter(rng.standard_normal((n, n)), n * sigma, mode="wrap")
    g2 = gaussian_filter(rng.standard_normal((n, n)), n * sigma, mode="wrap")
    th = np.arctan2(g1, g2)
    lam = rng.uniform(1, lam_max, (n, n))
    c, s = np.cos(th), np.sin(th)
    m = np.stack([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], -1).astype(np.float32)
    w = np.zeros((n, n), bool)
    w[n // 2, n // 8:] = True
    w[n // 2, n // 4:n // 4 + 3] = False
    w[n // 2, 3 * n // 4:3 * n // 4 + 2] = False
    X, Y = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    r = np.hypot(X - 0.25 * n, Y - 0.7 * n)
    w |= (r > 0.12 * n) & (r < 0.12 * n + 1.5) & (Y < 0.7 * n + 0.08 * n)
    seeds = np.array([[0.2, 0.3], [0.8, 0.4], [0.7, 0.85]], np.float32)[:nseeds]
    return dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), metric=m, seeds=seeds, walls=w)


def _walled_riemann3(n, seed):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    a = gaussian_filter(rng.standard_normal((3, 3, n, n, n)), (0, 0, 2, 2, 2), mode="wrap")
    am = np.moveaxis(a, (0, 1), (-2, -1))
    u, _, vt = np.linalg.svd(am)
    rot = u @ vt
    ev = np.exp(rng.uniform(0, np.log(8.0), (n, n, n, 3)))
    M = rot @ (ev[..., :, None] * np.swapaxes(rot, -1, -2))
    m = np.stack([M[..., i, j] for i in range(3) for j in range(i + 1)], -1).astype(np.float32)
    w = np.zeros((n, n, n), bool)
    w[:, n // 2, :] = True
    w[n // 3:n // 3 + 3, n // 2, n // 3:n // 3 + 3] = False
    return dict(model="Riemann3", dims=np.array([n] * 3, np.float32), gridScales=np.full(3, 1.0 / n, np.float32),
                origin=np.zeros(3, np.float32), metric=m, seeds=np.array([[0.3, 0.2, 0.6]], np.float32), walls=w,
                wallDistBound=6)


@pytest.mark.parametrize("make", [lambda: _walled_riemann2(160, 3, nseeds=3), lambda: _walled_riemann3(36, 4)],
                         ids=["riem2_160", "riem3_36"])
def test_walls_vs_discrete_solution(make):
    case = make()
    out = make_dictin(case, extra={"exportValues": True}).Run()
    exact = discrete_solution(case)
    assert_near_discrete(out["values"].cpu().numpy(), case, exact)
    tight = make_dictin(case, extra=dict(TIGHT, exportValues=True)).Run()["values"].cpu().numpy()
    assert rel_err(tight, exact) < TIGHT_REL


@pytest.mark.parametrize("extra", [{"factoringRadius": 12.0}, {"multiprecision": True}],
                         ids=["factor", "multiprecision"])
def test_walls_with_options_vs_discrete_solution(extra):
    """Walls with source factorisation (a wall crossing the factored disk) and
    with multiprecision: float32 rounding of the discrete solution at tight
    tolerances.  The metric varies slowly: the factored scheme has no lower
    bound where the metric changes much inside the factoring radius."""
    case = _walled_riemann2(128, 8, lam_max=4.0, sigma=1 / 4)
    case["seeds"] = np.array([[0.45, 0.3]], np.float32)  # 7 pixels from the long wall
    case = dict(case, **extra)
    exact = discrete_solution(case)
    tight = make_dictin(case, extra=dict(TIGHT, exportValues=True, **extra)).Run()["values"].cpu().numpy()
    assert rel_err(tight, exact) < TIGHT_REL


def test_walls_order2_accuracy():
    """Second order with walls: the values depend on the order of the in-tile
    updates (non-monotone correction), so the GPU solve is compared with the
    oracle's float64 run of the same scheme at the level of that dependence."""
    case = dict(_walled_riemann2(128, 9, nseeds=2), order=2)
    v = make_dictin(case, extra={"exportValues": True}).Run()["values"].cpu().numpy()
    exact = discrete_solution(case)
    fin = np.isfinite(exact) & (exact > 0)
    assert np.array_equal(np.isfinite(v), np.isfinite(exact))
    rel = np.abs(v[fin] - exact[fin]) / exact[fin]
    assert rel.max() < 6e-2 and rel.mean() < 4e-3


def test_walls_forward_and_reverse_ad():
    """AD with walls: a cost varied by itself varies the solution by itself away
    from the walls, the variation vanishes on the walls (their right-hand side
    +inf is a constant), and <s, du> = <lam, c dc> with the reverse mode."""
    case = _walled_riemann2(96, 11, nseeds=2)
    shape = (96, 96)
    rng = np.random.default_rng(2)
    dc = rng.standard_normal(shape).astype(np.float32)
    sens = np.zeros(shape + (1,), np.float32)
    sens.reshape(-1)[rng.choice(96 * 96, 11, replace=False)] = 1.0
    out = make_dictin(case, extra=dict(TIGHT, exportValues=True, sensitivity=sens,
                                       costVariation=np.stack([np.ones(shape, np.float32), dc], -1))).Run()
    u = out["values"].cpu().numpy()
    vv = out["valueVariation"].cpu().numpy()
    walls = case["walls"]
    fin = np.isfinite(u)
    assert np.abs(vv[..., 0][fin] - u[fin]).max() <= 2e-5 * np.abs(u[fin]).max()
    assert (vv[walls] == 0).all()
    lam = out["costSensitivity"].cpu().numpy()[..., 0]
    lhs = float((sens[..., 0] * np.where(fin, vv[..., 1], 0)).sum())
    rhs = float((np.where(fin & ~walls, lam, 0) * dc).sum())
    assert abs(lhs - rhs) <= 1e-3 * max(abs(lhs), 1e-3)


def test_fixed_scratch_refuses_riemann_walls():
    """The fixed-scratch entry point has no stencil cache, where the wall bits of
    the Riemann stencils live: it refuses such instances with a status."""
    from adaptivegriddiscretizations_b200 import _lib
    from adaptivegriddiscretizations_b200.Eikonal.HFM_CUDA import Interface
    case, _ = load_case("riem2_walls")
    case = {k: v for k, v in case.items() if k != "tips"}
    it = Interface(make_dictin(case))
    it.SetKernelTraits()
    it.SetGeometry()
    it.SetArgs()
    inst = it.instance()
    stats = torch.zeros(2, dtype=torch.int64, device="cuda")
    rc = _lib.lib().agd_eikonal_solve_fixed_scratch(ctypes.byref(inst), 1, _lib.ptr(stats), None, _lib.stream_ptr())
    assert rc == _lib.AGD_STATUS_UNSUPPORTED
