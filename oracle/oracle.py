"""Python face of the CPU oracle (liboracle.so, built from hfm_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker or the timed CPU baseline.  The
product path never imports it.

`run(case, dtype)` restates the reference's GPU pipeline for one dictIn-like
case dictionary (keys as in agd.Eikonal.dictIn): host preparation
(agd/Eikonal/HFM_CUDA/_SetGeometry.py:127-137,238-253; _SetArgs.py:8-133),
solve (FIM over tiles), flow, geodesics (_GetGeodesics.py:9-147) and reverse
sensitivity (_PostProcess.py:155-219), on the CPU, in float32 or float64.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_P = ctypes.c_void_p
_lib = None

DEFAULT_TRAITS = {  # agd/Eikonal/HFM_CUDA/kernel_traits.py:61-88
    "Riemann2": ((8, 8), 8, 4),
    "Riemann3": ((4, 4, 4), 4, 6),
    "Isotropic2": ((16, 16), 16, 4),
    "Isotropic3": ((4, 4, 4), 8, 4),
    "Diagonal2": ((16, 16), 16, 4),
    "Diagonal3": ((4, 4, 4), 8, 4),
    "Rander2": ((8, 8), 12, 8),
    "Rander3": ((4, 4, 4), 8, 8),
}
STOP_CODES = ["Continue", "AtSeed", "InWall", "Stationnary", "PastSeed", "VanishingFlow"]


def build():
    """Compile liboracle.so (g++, OpenMP)."""
    src = os.path.join(HERE, "hfm_oracle.cpp")
    subprocess.check_call(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-fopenmp", "-ffp-contract=off",
                           "-Wno-unknown-pragmas", src, "-o", LIB])


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "hfm_oracle.cpp")
        if not os.path.exists(LIB) or (os.path.exists(src) and os.path.getmtime(src) > os.path.getmtime(LIB)):
            build()
        _lib = ctypes.CDLL(LIB)
        _lib.agdo_eikonal.restype = ctypes.c_int
        _lib.agdo_reverse.restype = ctypes.c_int
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_P)


def selling(m):
    """Selling decomposition of packed symmetric matrices m (n, symdim) float32.
    Returns weights (n, symdim) and integer offsets (n, symdim, ndim)."""
    m = np.ascontiguousarray(m, np.float32)
    n, sd = m.shape
    nd = 2 if sd == 3 else 3
    w = np.zeros((n, sd), np.float32)
    e = np.zeros((n, sd, nd), np.int32)
    lib().agdo_selling_f32(nd, _p(m), n, _p(w), _p(e))
    return w, e


def dual_metric_flat(metric_hfm, h):
    """Dual of metric.with_costs(h), lower-triangular planes (symdim, *shape), float32.
    metric_hfm: (*shape, symdim) HFM layout (Metrics.Riemann.from_HFM)."""
    mh = np.asarray(metric_hfm, np.float32)
    nd = 2 if mh.shape[-1] == 3 else 3
    M = np.zeros(mh.shape[:-1] + (nd, nd), np.float32)
    k = 0
    for i in range(nd):
        for j in range(i + 1):
            M[..., i, j] = mh[..., k]
            M[..., j, i] = mh[..., k]
            k += 1
    h = np.asarray(h, np.float32)
    M = M * h[:, None] * h[None, :]
    Dm = np.linalg.inv(M).astype(np.float32)
    return np.stack([Dm[..., i, j] for i in range(nd) for j in range(i + 1)]).astype(np.float32)


class Prepared:
    pass


def rander_parts(metric_hfm, nd):
    """Quadratic part (..., nd, nd) and drift (..., nd) of a Rander metric in HFM
    layout (*shape, symdim + nd), float64."""
    a = np.asarray(metric_hfm, np.float64)
    sd = nd * (nd + 1) // 2
    M = np.zeros(a.shape[:-1] + (nd, nd))
    k = 0
    for i in range(nd):
        for j in range(i + 1):
            M[..., i, j] = M[..., j, i] = a[..., k]
            k += 1
    return M, a[..., sd:]


def wall_distance(walls, bound):
    """L1 distance to the nearest wall point, saturated at 255 and set to 255
    beyond `bound` (_SetGeometry.py:262-280): `bound` min-plus passes of the
    3^ndim kernel |o|_1 from 0 at the walls, 255 elsewhere, points outside the
    grid ignored."""
    walls = np.asarray(walls, bool)
    nd = walls.ndim
    d = np.where(walls, 0, 255).astype(np.int32)
    offsets = np.stack(np.meshgrid(*([np.arange(-1, 2)] * nd), indexing="ij"), -1).reshape(-1, nd)
    for _ in range(bound):
        pad = np.pad(d, 1, constant_values=255)
        best = d.copy()
        for o in offsets:
            sl = tuple(slice(1 + c, 1 + c + n) for c, n in zip(o, d.shape))
            best = np.minimum(best, np.minimum(pad[sl] + int(np.abs(o).sum()), 255))
        d = best
    d[d > bound] = 255
    return d.astype(np.uint8)


def prepare(case):
    """Host preparation of a case (model, dims, gridScales, origin, cost, metric,
    seeds, seedValues, traits, multiprecision)."""
    pr = Prepared()
    pr.model = str(case["model"])
    pr.ndim = int(pr.model[-1])
    pr.rander = pr.model.startswith("Rander")
    pr.riemann = pr.model.startswith("Riemann") or pr.rander  # Selling stencil
    pr.diagonal = pr.model.startswith("Diagonal")
    pr.shape = tuple(int(s) for s in np.asarray(case["dims"]))
    pr.h = np.broadcast_to(np.asarray(case.get("gridScales", case.get("gridScale")), np.float32), (pr.ndim,)).copy()
    pr.origin = np.asarray(case.get("origin", np.zeros(pr.ndim)), np.float32)
    si, niter, front = DEFAULT_TRAITS[pr.model]
    tr = case.get("traits")
    if tr is not None:
        si = tuple(int(s) for s in tr.get("shape_i", si))
        niter = int(tr.get("niter_i", niter))
    pr.shape_i, pr.niter_i, pr.front = tuple(si), niter, int(case.get("fim_front_width", front))
    cost = np.broadcast_to(np.asarray(case.get("cost", 1.0), np.float32), pr.shape).astype(np.float32)
    pr.geom = dual_metric_flat(case["metric"], pr.h) if pr.riemann and not pr.rander else None
    if pr.rander:  # metric.with_costs(h).flatten(inverse_m=True), float32 (_SetGeometry.py:138-139)
        mh = np.broadcast_to(np.asarray(case["metric"], np.float32), pr.shape + (pr.ndim * (pr.ndim + 3) // 2,))
        M, w = rander_parts(mh, pr.ndim)
        hf = pr.h.astype(np.float32)
        hh = (hf[:, None] * hf[None, :]).astype(np.float32)  # Rander.with_costs: m * outer(h, h)
        Mi = np.linalg.inv((M.astype(np.float32) * hh).astype(np.float32)).astype(np.float32)
        wh = (w.astype(np.float32) * hf).astype(np.float32)
        planes = [Mi[..., i, j] for i in range(pr.ndim) for j in range(i + 1)] + [wh[..., i] for i in range(pr.ndim)]
        pr.geom = np.ascontiguousarray(np.stack(planes), np.float32)
    if pr.diagonal:  # squared dual costs 1 / (c h)^2, float32 (_SetGeometry.py:134-135)
        costs = np.moveaxis(np.broadcast_to(np.asarray(case["metric"], np.float32), pr.shape + (pr.ndim,)), -1, 0)
        pr.geom = np.ascontiguousarray((np.float32(1) / (costs * pr.h.reshape((-1,) + (1,) * pr.ndim))) ** 2,
                                       np.float32)
    res = np.finfo(np.float32).resolution
    # atol: the `atol` key, else `tol`, else 5 float32 resolutions of the mean cost (_SetGeometry.py:238-250)
    pr.atol = float(case["atol"]) if "atol" in case else float(case["tol"]) if "tol" in case else \
        float(np.float32(np.nanmean(cost) * res * 5.0))
    pr.rtol = float(np.float32(res * 5.0)) if "rtol" not in case else float(case["rtol"])
    seeds = np.asarray(case["seeds"], np.float32).reshape(-1, pr.ndim)
    sv = np.asarray(case.get("seedValues", np.zeros(len(seeds))), np.float32)
    start = pr.origin + 0.5 * pr.h
    pr.order2 = float(case.get("order2_threshold", 0.3)) if int(case.get("order", 1)) == 2 else 0.0
    fr = float(case.get("factoringRadius", 0.0))
    pr.factor = None
    if fr:  # source factorisation around the (single) seed (_Kernel.py:47-49, 301-308)
        seed = ((seeds - start) / pr.h)[0].astype(np.float64)
        m0 = _seed_metric(pr, case, cost, seed)
        if pr.riemann:
            fm = np.array([m0[i, j] for i in range(pr.ndim) for j in range(i + 1)])
        else:
            fm = np.diag(m0).copy()
        pr.factor = (fr * fr, seed, fm)
    radius = float(case.get("seedRadius", 2.0 if fr else 0.0))
    if radius:
        pr.seed_idx, sv = _spread_seed(pr, case, cost, ((seeds - start) / pr.h)[0], float(sv[0]), radius)
    else:
        pr.seed_idx = np.round((seeds - start) / pr.h).astype(int)
    rhs = cost.copy()
    mask = np.zeros(pr.shape, np.uint8)
    pos = tuple(pr.seed_idx.T)
    rhs[pos] = sv
    mask[pos] = 1
    pr.trigger = mask.copy()  # the seeds, walls excluded
    pr.walls = pr.wall_dist = None
    if case.get("walls") is not None:  # walls: seeds of value +inf (_SetArgs.py:124-126)
        pr.walls = np.broadcast_to(np.asarray(case["walls"], bool), pr.shape).copy()
        pr.wall_dist = wall_distance(pr.walls, int(case.get("wallDistBound", 10)))
        mask[pr.walls] = 1
        rhs[pr.walls] = np.inf
    pr.rhs, pr.seed_mask = rhs, mask
    pr.iso_w = (pr.h.astype(np.float64) ** -2) if not (pr.riemann or pr.diagonal) else None
    if pr.iso_w is not None:
        pr.iso_w = np.asarray(pr.h.astype(np.float32) ** -2, np.float64)
    return pr


def _cost_metric(pr, case, cost):
    """Grid point -> the metric with the grid scales and the cost applied, index
    units (Interface.CostMetric, _Interface.py:202-211)."""
    nd = pr.ndim
    h = pr.h.astype(np.float64)
    c = np.asarray(cost, np.float64)
    if pr.rander:  # (M, w) -> (c^2 h M h, c h w): the quadratic part; _cost_drift gives the drift
        M, _ = rander_parts(np.broadcast_to(np.asarray(case["metric"], np.float64),
                                            tuple(pr.shape) + (nd * (nd + 3) // 2,)), nd)

        def cm(p):
            return c[tuple(p)] ** 2 * M[tuple(p)] * np.outer(h, h)
    elif pr.riemann:
        mf = np.broadcast_to(np.asarray(case["metric"], np.float64), tuple(pr.shape) + (nd * (nd + 1) // 2,))
        tri = [(i, j) for i in range(nd) for j in range(i + 1)]

        def cm(p):
            M = np.zeros((nd, nd))
            for q, (i, j) in enumerate(tri):
                M[i, j] = M[j, i] = mf[tuple(p)][q]
            return c[tuple(p)] ** 2 * M * np.outer(h, h)
    elif pr.diagonal:
        mc = np.broadcast_to(np.asarray(case["metric"], np.float64), tuple(pr.shape) + (nd,))

        def cm(p):
            return np.diag((mc[tuple(p)] * c[tuple(p)] * h) ** 2)
    else:
        def cm(p):
            return np.diag((c[tuple(p)] * h) ** 2)
    return cm


def _cost_drift(pr, case, cost):
    """Rander: grid point -> the drift of the cost metric, c h w (index units)."""
    nd = pr.ndim
    _, w = rander_parts(np.broadcast_to(np.asarray(case["metric"], np.float64), tuple(pr.shape) + (nd * (nd + 3) // 2,)),
                        nd)
    c = np.asarray(cost, np.float64)
    h = pr.h.astype(np.float64)
    return lambda p: c[tuple(p)] * h * w[tuple(p)]


def _interp(pr, seed, f):
    """Multilinear interpolation of the grid function f at a continuous index seed."""
    nd = pr.ndim
    shape = np.array(pr.shape)
    lo = np.clip(np.floor(seed).astype(int), 0, shape - 1)
    frac = np.clip(seed - lo, 0.0, 1.0)
    out = 0.0
    for bits in np.ndindex(*([2] * nd)):
        w = np.prod([fr if b else 1.0 - fr for b, fr in zip(bits, frac)])
        out = out + w * f(np.minimum(lo + np.array(bits), shape - 1))
    return out


def _seed_metric(pr, case, cost, seed):
    """The cost metric at a seed (continuous index coordinates), multilinearly
    interpolated: its entries (Riemann), or the costs c*h per axis (Isotropic,
    Diagonal)."""
    nd = pr.ndim
    shape = np.array(pr.shape)
    cm = _cost_metric(pr, case, cost)
    c = np.asarray(cost, np.float64)
    lo = np.clip(np.floor(seed).astype(int), 0, shape - 1)
    frac = np.clip(seed - lo, 0.0, 1.0)
    m0 = np.zeros((nd, nd))
    c0 = np.zeros(nd)
    for bits in np.ndindex(*([2] * nd)):
        w = np.prod([f if b else 1.0 - f for b, f in zip(bits, frac)])
        p = np.minimum(lo + np.array(bits), shape - 1)
        m0 += w * cm(p)
        c0 += w * np.sqrt(np.diag(cm(p)))  # the costs c*h per axis
    return m0 if pr.riemann else np.diag(c0 ** 2)


def _spread_seed(pr, case, cost, seed, seed_value, r):
    """Seed spreading (agd/Eikonal/HFM_CUDA/_SetArgs.py:46-75), float64: the grid
    points within r of the seed (index units) take the value seed_value +
    (|d|_{M(seed)} + |d|_{M(x)}) / 2 with M the cost-scaled metric in index units
    (Interface.CostMetric, _Interface.py:202-211), interpolated multilinearly."""
    nd = pr.ndim
    shape = np.array(pr.shape)
    seed = np.asarray(seed, np.float64)
    axes = [np.arange(int(np.floor(c - r)), int(np.ceil(c + r) + 1)) for c in seed]
    pts = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, nd)
    pts = pts[np.linalg.norm(pts - seed, axis=1) < r]
    pts = pts[np.all((pts >= -0.5) & (pts < shape - 0.5), axis=1)]
    cm = _cost_metric(pr, case, cost)
    m0 = _seed_metric(pr, case, cost, seed)
    drift = _cost_drift(pr, case, cost) if pr.rander else (lambda p: np.zeros(nd))
    w0 = _interp(pr, seed, drift) if pr.rander else np.zeros(nd)
    vals = []
    for p in pts:
        d = p - seed  # Rander norms: sqrt(<d, M d>) + <w, d>
        vals.append(seed_value + 0.5 * (np.sqrt(d @ m0 @ d) + w0 @ d + np.sqrt(d @ cm(p) @ d) + drift(p) @ d))
    return pts.astype(int), np.asarray(vals, np.float32)


def eikonal(pr, dtype=np.float32, values=None, nthreads=1, flow=False, nitermax=2000):
    """Solve; returns dict(values, niter_o, tile_visits[, flow_vector, flow_weightsum, flow_weights, flow_indices])."""
    L = lib()
    N = int(np.prod(pr.shape))
    u = np.full(pr.shape, np.inf, np.float64) if values is None else np.array(values, np.float64)
    visits = ctypes.c_longlong(0)
    nact = pr.ndim * (pr.ndim + 1) // 2 if pr.riemann else pr.ndim
    fv = fws = fw = fi = None
    if flow:
        fv = np.zeros((pr.ndim,) + pr.shape)
        fws = np.zeros(pr.shape)
        fw = np.zeros((nact,) + pr.shape)
        fi = np.zeros((nact,) + pr.shape, np.int32)
    geom = None if pr.geom is None else np.ascontiguousarray(pr.geom, np.float32)
    iso = None if pr.iso_w is None else np.ascontiguousarray(pr.iso_w, np.float64)
    L.agdo_set_order2(ctypes.c_double(getattr(pr, "order2", 0.0)))
    wd = getattr(pr, "wall_dist", None)
    wd = None if wd is None else np.ascontiguousarray(wd, np.uint8)
    L.agdo_set_walls(_p(wd))  # kept by pointer: wd stays alive through the solve
    fac = getattr(pr, "factor", None)
    if fac is None:
        L.agdo_set_factor(ctypes.c_double(0.0), None, None)
    else:
        org = np.zeros(3)
        org[: pr.ndim] = fac[1]
        met = np.zeros(6)
        met[: len(fac[2])] = fac[2]
        L.agdo_set_factor(ctypes.c_double(fac[0]), _p(org), _p(met))
    niter = L.agdo_eikonal(int(dtype == np.float64), pr.ndim,
                           3 if pr.rander else (1 if pr.riemann else (2 if pr.diagonal else 0)),
                           (ctypes.c_int * pr.ndim)(*pr.shape), (ctypes.c_int * pr.ndim)(*pr.shape_i),
                           pr.niter_i, pr.front, _p(iso), _p(geom), _p(np.ascontiguousarray(pr.rhs)),
                           _p(np.ascontiguousarray(pr.seed_mask)), _p(u), ctypes.c_double(pr.atol),
                           ctypes.c_double(pr.rtol), nitermax, nthreads, ctypes.byref(visits), _p(fv), _p(fws),
                           _p(fw), _p(fi))
    L.agdo_set_walls(None)
    out = dict(values=u, niter_o=niter, tile_visits=visits.value)
    if flow:
        out.update(flow_vector=fv, flow_weightsum=fws, flow_weights=fw, flow_indices=fi)
    return out


def geodesics(pr, values, flow_vector, flow_weightsum, tips, step=0.25, causality=4.0, pastseed_delay=0):
    """Backtrack from physical tips; returns (list of (ndim, len) physical paths, stop codes).
    The PastSeed test waits pastseed_delay steps in the first chunk only
    (_GetGeodesics.py:107-109,133)."""
    L = lib()
    nd = pr.ndim
    shp = (ctypes.c_int * nd)(*pr.shape)
    eucl = np.zeros(pr.shape, np.uint8)
    L.agdo_eucl_map(nd, shp, _p(np.ascontiguousarray(pr.trigger)), _p(eucl))  # seeds, not walls
    u = np.ascontiguousarray(values, np.float32)
    fv = np.ascontiguousarray(flow_vector, np.float32)
    fws = np.ascontiguousarray(flow_weightsum, np.float32)
    max_len = int(max(40, 20 * max(pr.shape) / step))
    typical = min(max_len, int(max(40, 0.5 * max(pr.shape) / step)))
    eucl_delay = int(np.sqrt(nd) / step)
    nymin_delay = int(8.0 * np.sqrt(nd) / step)
    start = pr.origin + 0.5 * pr.h
    tips_c = ((np.asarray(tips, np.float32) - start) / pr.h).astype(np.float32)
    geos = [[t.reshape(1, -1)] for t in tips_c]
    stops = ["Stopping criterion"] * len(tips_c)
    corresp = list(range(len(tips_c)))
    it, maxit = 0, int(np.ceil(max_len / typical))
    while corresp and it < maxit:
        it += 1
        n = len(corresp)
        x_s = np.full((n, typical, nd), np.nan, np.float32)
        x_s[:, 0] = np.stack([geos[i][-1][-1] for i in corresp])
        len_s = np.zeros(n, np.int32)
        stop_s = np.zeros(n, np.int8)
        L.agdo_geodesic_chunk(nd, shp, n, typical, pastseed_delay if it == 1 else 0, ctypes.c_float(causality), ctypes.c_float(step), eucl_delay,
                              nymin_delay, _p(u), _p(fv), _p(fws), _p(eucl), _p(x_s), _p(len_s), _p(stop_s))
        nxt = []
        for i, x, l, s in zip(corresp, x_s, len_s, stop_s):
            geos[i].append(x[1:int(l)])
            if s != 0:
                stops[i] = STOP_CODES[int(s)]
            else:
                nxt.append(i)
        corresp = nxt
    paths = [(start + pr.h * np.concatenate(g, 0)).T for g in geos]
    return paths, stops


def reverse(pr, values, flow_weights, flow_indices, flow_weightsum, sens):
    """Reverse sensitivity lam (grid) for rhs `sens` (grid, float)."""
    nact = flow_weights.shape[0]
    N = int(np.prod(pr.shape))
    lam = np.zeros(N)
    lib().agdo_reverse(nact, ctypes.c_long(N), _p(np.ascontiguousarray(values, np.float64).reshape(-1)),
                       _p(np.ascontiguousarray(flow_weights, np.float64).reshape(nact, -1)),
                       _p(np.ascontiguousarray(flow_indices, np.int32).reshape(nact, -1)),
                       _p(np.ascontiguousarray(flow_weightsum, np.float64).reshape(-1)),
                       _p(np.ascontiguousarray(sens, np.float64).reshape(-1)), _p(lam))
    return lam.reshape(pr.shape)


def forward(pr, values, flow_weights, flow_indices, flow_weightsum, rhs):
    """Forward variation du (grid) for the right-hand side `rhs` (grid, float)."""
    nact = flow_weights.shape[0]
    N = int(np.prod(pr.shape))
    du = np.zeros(N)
    lib().agdo_forward(nact, ctypes.c_long(N), _p(np.ascontiguousarray(values, np.float64).reshape(-1)),
                       _p(np.ascontiguousarray(flow_weights, np.float64).reshape(nact, -1)),
                       _p(np.ascontiguousarray(flow_indices, np.int32).reshape(nact, -1)),
                       _p(np.ascontiguousarray(flow_weightsum, np.float64).reshape(-1)),
                       _p(np.ascontiguousarray(rhs, np.float64).reshape(-1)), _p(du))
    return du.reshape(pr.shape)


def forward_rhs(pr, cost_variation, seed_value_variation):
    """Right-hand sides of forward AD, (n, *shape): the seed values' variation
    (n, nseeds) at the seeds, the cost's variation times the cost elsewhere
    (_PostProcess.py:182-183)."""
    cv = np.moveaxis(np.asarray(cost_variation, np.float64), -1, 0).copy()
    pos = tuple(pr.seed_idx.T)
    if seed_value_variation is not None:
        sv = np.asarray(seed_value_variation, np.float64)
        for j in range(len(cv)):
            cv[j][pos] = sv[j]
    else:
        for j in range(len(cv)):
            cv[j][pos] = 0.0
    mask = pr.seed_mask.astype(bool)
    if pr.walls is not None:  # the right-hand side +inf of the walls is a constant
        cv[:, pr.walls] = 0.0
    return np.where(mask, cv, cv * pr.rhs.astype(np.float64))


def run(case, dtype=np.float32, nthreads=1):
    """Whole pipeline for a case; returns a dict like the reference's hfmOut."""
    pr = prepare(case)
    need_flow = "tips" in case or "sensitivity" in case or "costVariation" in case
    r = eikonal(pr, dtype, nthreads=nthreads, flow=need_flow)
    out = dict(values=r["values"], niter_o=r["niter_o"], tile_visits=r["tile_visits"], prepared=pr)
    if need_flow:
        out["flow_vector"], out["flow_weightsum"] = r["flow_vector"], r["flow_weightsum"]
    if "tips" in case:
        out["geodesics"], out["geodesic_stopping_criteria"] = geodesics(
            pr, r["values"], r["flow_vector"], r["flow_weightsum"], case["tips"],
            pastseed_delay=int(case.get("pastseed_delay", 0)))
    norm = flow_normalization(pr, case, r["flow_vector"]) if need_flow and pr.rander else None
    if "costVariation" in case:
        rhs = forward_rhs(pr, case["costVariation"], case.get("seedValueVariation"))
        if norm is not None:  # drift models (_PostProcess.py:185)
            rhs = rhs * norm
        out["valueVariation"] = np.stack(
            [forward(pr, r["values"], r["flow_weights"], r["flow_indices"], r["flow_weightsum"], x) for x in rhs], -1)
    if "sensitivity" in case:
        sens = np.asarray(case["sensitivity"])[..., 0]
        lam = reverse(pr, r["values"], r["flow_weights"], r["flow_indices"], r["flow_weightsum"], sens)
        pos = tuple(pr.seed_idx.T)
        out["seedValueSensitivity"] = lam[pos][:, None]
        cs = lam.copy()
        cs[pos] = 0
        if norm is not None:  # drift models (_PostProcess.py:213-214)
            cs = cs / norm
        out["costSensitivity"] = cs[..., None]
    return out


def flow_normalization(pr, case, flow_vector):
    """Drift models: 1 at the seeds, else the norm of -flow_vector for the
    metric with the grid scales applied (_PostProcess.py:80-88)."""
    nd = pr.ndim
    M, w = rander_parts(np.broadcast_to(np.asarray(case["metric"], np.float64),
                                        tuple(pr.shape) + (nd * (nd + 3) // 2,)), nd)
    h = pr.h.astype(np.float64)
    v = -np.moveaxis(np.asarray(flow_vector, np.float64), 0, -1)
    Mh = M * np.outer(h, h)
    n = np.sqrt(np.einsum("...i,...ij,...j->...", v, Mh, v)) + np.einsum("...i,...i->...", w * h, v)
    return np.where(pr.seed_mask.astype(bool), 1.0, n)
