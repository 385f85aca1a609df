"""GPU parity of the eikonal solve through the public dictIn(...).Run() surface.

Against: the golden outputs of the reference's own kernels (small cases, 1e-5
relative), and the scheme's discrete solution from the float64 oracle on
larger seeded cases (the criteria of parity.py: stopping-tolerance bound at the
default tolerances, float32 rounding with tight ones).  Offsets of Selling's
decomposition bit-exact.
"""
import numpy as np
import pytest
import torch

from conftest import (CASES, FACTOR_CASES, GOLDEN, ORDER2_CASES, ORDER2_FACTOR_CASES, ORDER2_MP_CASES, RADIUS_CASES,
                      load_case, make_dictin)
from parity import TIGHT, TIGHT_REL, assert_near_discrete, discrete_solution
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REL = 1e-5


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    fin = np.isfinite(b)
    assert np.array_equal(fin, np.isfinite(a)), "finite masks differ"
    return (np.abs(a[fin] - b[fin]) / np.maximum(np.abs(b[fin]), 1e-30)).max()


@pytest.mark.parametrize("name", CASES + RADIUS_CASES + FACTOR_CASES + ORDER2_CASES)
def test_values_vs_reference(name):
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportValues": True}).Run()
    v = out["values"].cpu().numpy()
    assert v.dtype == np.float32 and v.shape == ref["values"].shape
    if name in ORDER2_CASES:
        # The second order correction is not monotone and values only decrease, so
        # the result depends on the order of the updates inside a tile: the golden
        # values come from the reference's kernels executed thread after thread,
        # while a GPU (the reference's or this one) updates 32 points at once.  The
        # reference's scheme itself moves by up to 1.2e-2 / 1.7e-2 / 4.1e-2 (mean
        # 0.8e-3 / 1.6e-3 / 2.2e-3) on these cases between the two orders.
        fin = np.isfinite(ref["values"]) & (ref["values"] > 0)
        rel = np.abs(v - ref["values"])[fin] / ref["values"][fin]
        assert rel.max() < 6e-2 and rel.mean() < 4e-3
        return
    # factored cases: the reference's own float32 run is up to ~1.5e-5 from the
    # discrete solution there (see test_factorisation_vs_discrete_solution)
    assert _rel(v, ref["values"]) < (3e-5 if name in FACTOR_CASES else REL)
    st = out["stats"]["eikonal"]
    assert st["niter_o"] > 0 and st["grid_updates"] > 0


def _riemann2_case(n, seed, lam_max=50.0, nseeds=4):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g1 = gaussian_filter(rng.standard_normal((n, n)), n / 64, mode="wrap")
    g2 = gaussian_filter(rng.standard_normal((n, n)), n / 64, mode="wrap")
    th = np.arctan2(g1, g2)
    lam = rng.uniform(1, lam_max, (n, n))
    c, s = np.cos(th), np.sin(th)
    m = np.stack([c * c + lam * s * s, c * s * (1 - lam), s * s + lam * c * c], -1).astype(np.float32)
    return dict(model="Riemann2", dims=np.array([n, n], np.float32), gridScales=np.full(2, 1.0 / n, np.float32),
                origin=np.zeros(2, np.float32), metric=m,
                seeds=rng.uniform(0.1, 0.9, (nseeds, 2)).astype(np.float32))


def _iso_case(shape, seed, nseeds=2):
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    g = gaussian_filter(rng.standard_normal(shape), 4.0, mode="wrap")
    g = (g - g.mean()) / g.std()
    nd = len(shape)
    return dict(model=f"Isotropic{nd}", dims=np.array(shape, np.float32),
                gridScales=np.full(nd, 1.0 / shape[0], np.float32), origin=np.zeros(nd, np.float32),
                cost=np.exp(0.5 * g).astype(np.float32),
                seeds=rng.uniform(0.1, 0.9, (nseeds, nd)).astype(np.float32) * np.array(shape) / shape[0])


@pytest.mark.parametrize("make", [lambda: _riemann2_case(192, 5), lambda: _iso_case((200, 150), 6),
                                  lambda: _iso_case((40, 36, 44), 7)], ids=["riem2_192", "iso2_200x150", "iso3_40"])
def test_values_vs_oracle(make):
    """Against the scheme's discrete solution (float64 oracle run to 1e-14): at
    the default stopping tolerances within 4 tolerances everywhere and 1e-5 on
    99.9% of the points; with tight tolerances to float32 rounding."""
    case = make()
    exact = discrete_solution(case)
    out = make_dictin(case, extra={"exportValues": True}).Run()
    assert_near_discrete(out["values"].cpu().numpy(), case, exact)
    tight = make_dictin(case, extra={"exportValues": True, **TIGHT}).Run()
    assert _rel(tight["values"].cpu().numpy(), exact) < TIGHT_REL


def test_gpu_transfer_mode():
    case, ref = load_case("riem2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, mode="gpu_transfer", extra={"exportValues": True}).Run()
    assert isinstance(out["values"], np.ndarray)
    assert _rel(out["values"], ref["values"]) < REL


def test_keys_bookkeeping():
    case, _ = load_case("iso2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportValues": True, "someUnknownKey": 3}).Run()
    keys = out["keys"]
    assert "someUnknownKey" in keys["unused"]
    assert "seeds" in keys["used"] and "nitermax_o" in keys["default"]
    assert keys["default"]["nitermax_o"] == 2000


def test_nonconvergence_raises():
    case, _ = load_case("riem2")
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    with pytest.raises(ValueError, match="did not reach convergence"):
        make_dictin(case, extra={"nitermax_o": 2}).Run()
    out = make_dictin(case, extra={"nitermax_o": 2, "raiseOnNonConvergence": False, "exportValues": True}).Run()
    assert out["stats"]["eikonal"]["niter_o"] <= 3


@pytest.mark.parametrize("nd", [2, 3])
def test_selling_gpu_bitexact(nd):
    import os
    from adaptivegriddiscretizations_b200 import _lib
    f = np.load(os.path.join(GOLDEN, f"selling{nd}.npz"))
    m = torch.as_tensor(f["m"], device="cuda").contiguous()
    n, sd = m.shape
    w = torch.empty((n, sd), dtype=torch.float32, device="cuda")
    e = torch.empty((n, sd, nd), dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().agd_selling(nd, _lib.ptr(m), n, _lib.ptr(w), _lib.ptr(e), _lib.stream_ptr()))
    assert np.array_equal(e.cpu().numpy(), f["ref_e"])
    # A weight is -<b_i, m b_j>, a cancelling sum: the GPU contracts its terms into
    # fused multiply-adds, the host build of the reference does not.  The rounding
    # difference is bounded relative to the size of the tensor, not of the weight.
    # Its terms are bounded by |b|^2 |m|, with |b|^2 <= max |offset|^2.
    wg, wr = w.cpu().numpy(), f["ref_w"]
    mnorm = np.abs(f["m"]).sum(axis=1, keepdims=True) * 2
    b2 = np.maximum((f["ref_e"].astype(np.float64) ** 2).sum(axis=2).max(axis=1, keepdims=True), 1)
    assert (np.abs(wg - wr) <= 4 * np.finfo(np.float32).eps * b2 * mnorm).all()


def test_multiprecision_vs_reference():
    """Multiprecision (u + uq * multip_step): against the reference's own
    multiprecision solution.  Its stopping test is absolute (rtol = 0, atol =
    5e-6 * mean cost), so the bound is absolute: two tolerances."""
    case, ref = load_case("riem2_mp")
    out = make_dictin(case, extra={"exportValues": True, "multiprecision": True}).Run()
    v = out["values"].cpu().numpy()
    want = ref["values"]
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(v))
    assert np.abs(v[fin] - want[fin]).max() <= 2 * float(ref["atol"])
    assert out["keys"]["default"]["rtol"] == 0.0


@pytest.mark.parametrize("name", ["iso2", "riem3", "iso3"])
def test_multiprecision_vs_float64_oracle(name):
    case, _ = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportValues": True, "multiprecision": True}).Run()
    v = out["values"].cpu().numpy().astype(np.float64)
    r64 = O.run(case, np.float64)["values"]
    fin = np.isfinite(r64)
    atol = 5e-6 * float(np.mean(case.get("cost", 1.0)))
    assert np.abs(v[fin] - r64[fin]).max() <= 4 * atol


def test_values_float64():
    case, ref = load_case("riem2_mp")
    out = make_dictin(case, extra={"exportValues": True, "values_float64": True}).Run()
    v = out["values"]
    assert v.dtype == torch.float64
    want = ref["values"]
    fin = np.isfinite(want)
    assert np.abs(v.cpu().numpy()[fin] - want[fin]).max() <= 2 * float(ref["atol"])


@pytest.mark.parametrize("model", ["Riemann2", "Isotropic2", "Riemann3"])
def test_factorisation_constant_metric(model):
    """A constant metric, the factoring radius covering the domain: the factored
    scheme is at least 10x closer to the exact distance |x - seed|_M than the
    plain one (exact for the isotropic metric), and it is the reference's scheme:
    equal to the float64 oracle (both at tolerance 1e-8) to float32 rounding."""
    nd = int(model[-1])
    n = 48 if nd == 2 else 20
    h = 1.0 / n
    M = np.array([[2.0, 0.7], [0.7, 1.0]]) if nd == 2 else np.array([[2.0, 0.3, 0.2], [0.3, 1.5, -0.4],
                                                                      [0.2, -0.4, 1.0]])
    if model.startswith("Isotropic"):
        M = np.eye(nd) * 1.7 ** 2
    seed = np.full(nd, 0.5) + 0.013
    case = dict(model=model, dims=np.full(nd, n, np.float32), gridScales=np.full(nd, h, np.float32),
                origin=np.zeros(nd, np.float32), seeds=seed[None].astype(np.float32), atol=1e-8, rtol=1e-8)
    if model.startswith("Riemann"):
        packed = np.array([M[i, j] for i in range(nd) for j in range(i + 1)], np.float32)
        case["metric"] = np.broadcast_to(packed, (n,) * nd + (len(packed),)).copy()
    else:
        case["cost"] = np.full((n,) * nd, 1.7, np.float32)
    grid = np.stack(np.meshgrid(*([(np.arange(n) + 0.5) * h] * nd), indexing="ij"), -1)
    d = grid - seed
    exact = np.sqrt(np.einsum("...i,ij,...j->...", d, M, d))
    far = exact > 4 * h
    tol = {"exportValues": True, "atol": 1e-8, "rtol": 1e-8}
    plain = make_dictin(case, extra=tol).Run()["values"].cpu().numpy()
    fcase = dict(case, factoringRadius=2.0 * n)
    fact = make_dictin(fcase, extra=dict(tol, factoringRadius=2.0 * n)).Run()["values"].cpu().numpy()
    err_plain = np.abs(plain - exact)[far].max() / exact[far].max()
    err_fact = np.abs(fact - exact)[far].max() / exact[far].max()
    assert err_fact < 0.1 * err_plain
    if model.startswith("Isotropic"):
        assert err_fact < 1e-5
    assert _rel(fact, O.run(fcase, np.float64, nthreads=8)["values"]) < 2e-6


@pytest.mark.parametrize("name", FACTOR_CASES)
def test_factorisation_vs_discrete_solution(name):
    """The golden factorisation cases against the scheme's discrete solution
    (float64 oracle, which reproduces the reference's factored kernels): the
    parity criteria at the default tolerances, float32 rounding at 1e-8."""
    case, _ = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    exact = discrete_solution(case)
    v = make_dictin(case, extra={"exportValues": True, "factoringRadius": case["factoringRadius"]}).Run()
    assert_near_discrete(v["values"].cpu().numpy(), case, exact)
    t = make_dictin(case, extra={"exportValues": True, "factoringRadius": case["factoringRadius"], **TIGHT}).Run()
    assert _rel(t["values"].cpu().numpy(), exact) < TIGHT_REL


@pytest.mark.parametrize("model", ["Isotropic2", "Riemann2", "Riemann3"])
def test_order2_accuracy_vs_reference_scheme(model):
    """Second order on a constant metric: against the exact distance, the error
    of the GPU values is that of the reference's scheme (float64 oracle, pinned
    to the reference's second order kernels) within 1.5x, and several times
    smaller than at first order."""
    nd = int(model[-1])
    n = 96 if nd == 2 else 32
    h = 1.0 / n
    seed = np.full(nd, 0.45) + np.arange(nd) * 0.07
    M = np.eye(nd) * 1.3 ** 2 if model.startswith("Iso") else (
        np.array([[2.0, 0.7], [0.7, 1.0]]) if nd == 2 else np.array([[2.0, 0.3, 0.2], [0.3, 1.5, -0.4], [0.2, -0.4, 1.0]]))
    case = dict(model=model, dims=np.full(nd, n, np.float32), gridScales=np.full(nd, h, np.float32),
                origin=np.zeros(nd, np.float32), seeds=seed[None].astype(np.float32), seedRadius=2.0,
                atol=1e-8, rtol=1e-8)
    if model.startswith("Iso"):
        case["cost"] = np.full((n,) * nd, 1.3, np.float32)
    else:
        packed = np.array([M[i, j] for i in range(nd) for j in range(i + 1)], np.float32)
        case["metric"] = np.broadcast_to(packed, (n,) * nd + (len(packed),)).copy()
    grid = np.stack(np.meshgrid(*([(np.arange(n) + 0.5) * h] * nd), indexing="ij"), -1)
    d = grid - seed
    exact = np.sqrt(np.einsum("...i,ij,...j->...", d, M, d))
    far = exact > 0.1
    extra = {"exportValues": True, "seedRadius": 2.0, "atol": 1e-8, "rtol": 1e-8}
    u1 = make_dictin(case, extra=extra).Run()["values"].cpu().numpy()
    u2 = make_dictin(case, extra=dict(extra, order=2)).Run()["values"].cpu().numpy()
    r2 = O.run(dict(case, order=2), np.float64, nthreads=8)["values"]
    e1, e2, eref = (np.abs(x - exact)[far].mean() for x in (u1, u2, r2))
    assert e2 < 0.3 * e1
    assert e2 < 1.5 * eref + 1e-5


def test_order2_more_accurate():
    """Constant cost, one seed spread over radius 2: the second order scheme is
    closer to the exact distance than the first order one, away from the seed."""
    n = 96
    h = 1.0 / n
    seed = np.array([0.4, 0.55])
    case = dict(model="Isotropic2", dims=np.array([n, n], np.float32), gridScales=np.full(2, h, np.float32),
                origin=np.zeros(2, np.float32), seeds=seed[None].astype(np.float32),
                cost=np.full((n, n), 1.3, np.float32))
    grid = np.stack(np.meshgrid(*([(np.arange(n) + 0.5) * h] * 2), indexing="ij"), -1)
    exact = 1.3 * np.linalg.norm(grid - seed, axis=-1)
    far = exact > 0.1
    base = {"exportValues": True, "seedRadius": 2.0, "atol": 1e-8, "rtol": 1e-8}
    u1 = make_dictin(case, extra=base).Run()["values"].cpu().numpy()
    u2 = make_dictin(case, extra=dict(base, order=2)).Run()["values"].cpu().numpy()
    e1 = np.abs(u1 - exact)[far].mean()
    e2 = np.abs(u2 - exact)[far].mean()
    assert e2 < 0.5 * e1


@pytest.mark.parametrize("solver", ["AGSI", "global_iteration"])
@pytest.mark.parametrize("name", ["iso2", "riem2", "riem3"])
def test_other_solvers_reach_the_discrete_solution(solver, name):
    """The reference's other outer iterations (the `solver` key: adaptive
    Gauss-Seidel, global iteration; _solvers.py:77-193) stop at the same
    discrete fixed point (the parity criteria against the discrete solution);
    a global iteration visits every tile at every epoch."""
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"solver": solver, "exportValues": True}).Run()
    v = out["values"].cpu().numpy()
    assert_near_discrete(v, case)
    st = out["stats"]["eikonal"]
    if solver == "global_iteration":
        shape = [int(s) for s in case["dims"]]
        si = {2: 16 if case["model"].startswith("Iso") else 8, 3: 4}[len(shape)]
        ntiles = int(np.prod([-(-s // si) for s in shape]))
        assert st["nupdate_o_total"] == st["niter_o"] * ntiles


@pytest.mark.parametrize("name", ["riem2_factor_mp", "iso2_factor_mp", "riem3_factor_mp"])
def test_factorisation_with_multiprecision_vs_reference(name):
    """Source factorisation together with multiprecision: against the
    reference's own kernels built with both (absolute stopping test: two
    tolerances), also with float64 values."""
    case, ref = load_case(name)
    want = ref["values"]
    fin = np.isfinite(want)
    for extra in ({"exportValues": True}, {"exportValues": True, "values_float64": True}):
        out = make_dictin(case, extra=dict(extra, multiprecision=True)).Run()
        v = out["values"].cpu().numpy()
        assert np.array_equal(fin, np.isfinite(v))
        assert np.abs(v[fin] - want[fin]).max() <= 2 * float(ref["atol"])


@pytest.mark.parametrize("name", ORDER2_FACTOR_CASES + ORDER2_MP_CASES)
def test_order2_combinations_vs_reference(name):
    """The second order scheme with source factorisation, and with
    multiprecision, against the reference's kernels built with both macros.
    The second order correction is not monotone and values only decrease, so
    the result depends on the order of the updates inside a tile (the
    reference's kernels executed thread after thread here, 32 points at once on
    a GPU): the criterion of the plain second order cases, max < 6e-2 and mean
    < 4e-3 relative, with equal finite masks."""
    case, ref = load_case(name)
    case = {k: v for k, v in case.items() if k not in ("tips", "sensitivity")}
    out = make_dictin(case, extra={"exportValues": True}).Run()
    v = out["values"].cpu().numpy()
    want = ref["values"]
    assert np.array_equal(np.isfinite(v), np.isfinite(want))
    pos = np.isfinite(want) & (want > 0)
    rel = np.abs(v - want)[pos] / want[pos]
    assert rel.max() < 6e-2 and rel.mean() < 4e-3, (rel.max(), rel.mean())
    assert out["stats"]["eikonal"]["niter_o"] > 0

