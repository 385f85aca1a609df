"""Generate the golden fixtures of the GPU eikonal path from the reference itself.

Runs only where the reference source tree is available (``--ref``, default
$AGD_REFERENCE, else a checkout named ``reference`` beside the repository): it imports the reference's numpy modules (``agd.Metrics``,
``agd.FiniteDifferences``, ``agd.Selling``) for the host-side preparation, and
drives the reference's own CUDA kernels compiled for the host by
``oracle/ref_emul/Makefile`` (libraries in ``oracle/_ref/``).

The host loops around the kernels restate, in numpy, the reference's driver code:
  SetGeometry / SetRHS / SetArgs      agd/Eikonal/HFM_CUDA/_SetGeometry.py:16-282, _SetArgs.py:8-177
  fast_iterative_method, InitStop     _solvers.py:94-120, _StopCriterion.py:62-84
  PostProcess (flow), values_expand   _PostProcess.py:19-95
  SolveAD (forward, reverse)          _PostProcess.py:155-219, graph_reverse.py:10-77
  GetGeodesics, inf_convolution       _GetGeodesics.py:9-147, inf_convolution.py:24-93

Output: one ``<case>.npz`` per case in this directory, holding the dictIn inputs
and the reference outputs.  Usage::

    make -C oracle/ref_emul REF=<reference checkout>
    python tests/golden/make_golden.py [--ref <reference checkout>]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFLIB = os.path.join(REPO, "oracle", "_ref")
P = ctypes.c_void_p


def ptr(a):
    return a.ctypes.data_as(P) if a is not None else None


def lib(name):
    return ctypes.CDLL(os.path.join(REFLIB, name))


# ----------------------------------------------------------------------------
# Seeded synthetic fields
# ----------------------------------------------------------------------------
def smooth_noise(rng, shape, sigma):
    from scipy.ndimage import gaussian_filter
    g = gaussian_filter(rng.standard_normal(shape), sigma, mode="wrap")
    return (g - g.mean()) / g.std()


def riemann2_metric(rng, shape, sigma, lam_max):
    th = np.arctan2(smooth_noise(rng, shape, sigma), smooth_noise(rng, shape, sigma))
    lam = rng.uniform(1.0, lam_max, shape)
    c, s = np.cos(th), np.sin(th)
    # M = R diag(1, lam) R^T
    m00 = c * c + lam * s * s
    m01 = c * s * (1 - lam)
    m11 = s * s + lam * c * c
    return np.stack([np.stack([m00, m01]), np.stack([m01, m11])]).astype(np.float32)


def riemann3_metric(rng, shape, sigma, ev_max):
    from scipy.ndimage import gaussian_filter
    a = rng.standard_normal((3, 3) + shape)
    a = gaussian_filter(a, (0, 0) + (sigma,) * 3, mode="wrap")
    am = np.moveaxis(a, (0, 1), (-2, -1))
    u, _, vt = np.linalg.svd(am)
    rot = u @ vt  # polar factor
    ev = np.exp(rng.uniform(0, np.log(ev_max), shape + (3,)))
    m = rot @ (ev[..., :, None] * np.swapaxes(rot, -1, -2))
    return np.moveaxis(m, (-2, -1), (0, 1)).astype(np.float32)


# ----------------------------------------------------------------------------
# Reference pipeline (numpy restatement of the host code + emulated kernels)
# ----------------------------------------------------------------------------
MODELS = {
    "Isotropic2": dict(tag="iso2", shape_i=(16, 16), niter_i=16, front=4),
    "Isotropic3": dict(tag="iso3", shape_i=(4, 4, 4), niter_i=8, front=4),
    "Riemann2": dict(tag="riem2", shape_i=(8, 8), niter_i=8, front=4),
    "Riemann3": dict(tag="riem3", shape_i=(4, 4, 4), niter_i=4, front=6),
    # the linear (AD) kernels depend on the tile shape only: the Isotropic builds serve
    "Diagonal2": dict(tag="diag2", lin="iso2", shape_i=(16, 16), niter_i=16, front=4),
    "Diagonal3": dict(tag="diag3", lin="iso3", shape_i=(4, 4, 4), niter_i=8, front=4),
    "Rander2": dict(tag="rand2", lin="riem2", shape_i=(8, 8), niter_i=12, front=8),
    "Rander3": dict(tag="rand3", lin="riem3", shape_i=(4, 4, 4), niter_i=8, front=8),
}


class RefPipeline:
    def __init__(self, case):
        from agd import FiniteDifferences as fd
        from agd import Metrics
        self.fd, self.Metrics = fd, Metrics
        self.c = case
        self.model = case["model"]
        self.md = MODELS[self.model]
        self.ndim = int(self.model[-1])
        self.shape = tuple(int(s) for s in case["dims"])
        self.h = np.asarray(case["gridScales"], np.float32)
        self.origin = np.asarray(case["origin"], np.float32)
        self.shape_i = self.md["shape_i"]
        self.size_i = int(np.prod(self.shape_i))
        self.shape_o = tuple(int(x) for x in fd.round_up_ratio(np.array(self.shape), np.array(self.shape_i)))
        self.size_o = int(np.prod(self.shape_o))
        self.multip = bool(case.get("multiprecision", False))

    def rander(self, dtype):
        """Metrics.Rander(m, w) from the case's HFM array (*shape, symdim + ndim).
        (The reference's Rander.from_HFM infers the dimension from the array
        length alone, which fails for Rander2: its users build the object.)"""
        nd = self.ndim
        arr = np.moveaxis(np.asarray(self.c["metric"], dtype), -1, 0)
        sd = nd * (nd + 1) // 2
        m = np.zeros((nd, nd) + arr.shape[1:], dtype)
        k = 0
        for i in range(nd):
            for j in range(i + 1):
                m[i, j] = m[j, i] = arr[k]
                k += 1
        return self.Metrics.Rander(m, arr[sd:])

    def bexp(self, a, cval):
        return np.ascontiguousarray(self.fd.block_expand(a, self.shape_i, mode="constant", constant_values=cval))

    def bsq(self, a):
        return self.fd.block_squeeze(a, self.shape)

    def point_from_index(self, idx, to=False):
        start = self.origin + 0.5 * self.h
        idx = np.asarray(idx, np.float32)
        return (idx - start) / self.h if to else start + self.h * idx

    def setup(self):
        c, nd = self.c, self.ndim
        cost = np.asarray(c.get("cost", np.ones(self.shape, np.float32)), np.float32)
        cost = np.broadcast_to(cost, self.shape).astype(np.float32)
        if self.model.startswith("Riemann"):
            metric = self.Metrics.Riemann.from_HFM(np.asarray(c["metric"], np.float32))
            dual = metric.with_costs(self.h).dual()
            self.geom = self.bexp(dual.flatten().astype(np.float32), np.inf)
        elif self.model.startswith("Rander"):  # geom = metric.flatten(inverse_m=True) (_SetGeometry.py:138-139)
            self.metric = self.rander(np.float32).with_costs(self.h)
            self.geom = self.bexp(np.asarray(self.metric.flatten(inverse_m=True), np.float32), np.inf)
        elif self.model.startswith("Diagonal"):  # geom = dualMetric.costs**2 (_SetGeometry.py:134-135)
            metric = self.Metrics.Diagonal.from_HFM(np.asarray(c["metric"], np.float32))
            dual = metric.with_costs(self.h).dual()
            self.geom = self.bexp((dual.costs ** 2).astype(np.float32), np.inf)
        else:
            self.geom = np.zeros(1, np.float32)
        float_res = np.finfo(np.float32).resolution
        self.atol = np.float32(np.nanmean(cost) * float_res * 5.0)
        self.rtol = np.float32(0.0 if self.multip else float_res * 5.0)
        seeds = np.asarray(c["seeds"], np.float32)
        seedValues = np.asarray(c.get("seedValues", np.zeros(len(seeds))), np.float32)
        self.factor = None
        fr = float(c.get("factoringRadius", 0.0))
        if fr:  # _Kernel.py:47-49, 301-308; seedRadius defaults to 2 (_SetArgs.py:40-43)
            seed = self.point_from_index(seeds, to=True)[0].astype(np.float64)
            hfm = np.asarray(self.cost_metric(cost).at(seed).to_HFM(), np.float32)
            if self.model.startswith("Rander"):  # the drift is left out (_Kernel.py:305-306)
                hfm = hfm[: -self.ndim]
            elif not self.model.startswith("Riemann"):
                hfm = hfm ** 2
            self.factor = (seed.astype(np.float32), np.float32(fr * fr), hfm.astype(np.float32))
        radius = float(c.get("seedRadius", 2.0 if fr else 0.0))
        if radius:
            seedIdx, seedValues = self.spread_seed(seeds, seedValues, radius, cost)
        else:
            seedIdx = np.round(self.point_from_index(seeds, to=True)).astype(int)
        self.seedIndices = seedIdx
        rhs = cost.copy()
        seedTags = np.zeros(self.shape, bool)
        pos = tuple(seedIdx.T)
        rhs[pos] = seedValues
        seedTags[pos] = True
        self.trigger = seedTags.copy()
        self.wall_b = None
        if c.get("walls") is not None:  # _SetGeometry.py:262-280, _SetArgs.py:124-126
            walls = np.broadcast_to(np.asarray(c["walls"], bool), self.shape)
            wd = self.wall_distance(walls, int(c.get("wallDistBound", 10)))
            self.wall_grid = wd
            self.wall_b = self.bexp(wd, 255).astype(np.uint8)
            seedTags = np.logical_or(seedTags, walls)
            rhs[walls] = np.inf
        self.seedTags = seedTags
        self.rhs_b = self.bexp(rhs, np.inf).astype(np.float32)
        sp = self.bexp(seedTags, True)
        self.seeds_b = np.packbits(sp.reshape(-1), bitorder="little")
        self.values_b = np.full(self.shape_o + self.shape_i, np.inf, np.float32)
        self.valuesq_b = np.zeros(self.values_b.shape, np.int32) if self.multip else None
        if self.multip:
            hmin = float(np.min(self.h))
            self.multip_step = np.float32(2.0 ** np.floor(np.log2(hmin / 10)))
            self.multip_max = np.float32(np.iinfo(np.int32).max * float(self.multip_step) / 2)
        else:
            self.multip_step = self.multip_max = np.float32(0)
        self.iso_w = (self.h.astype(np.float32) ** -2).astype(np.float32)

    def wall_distance(self, walls, bound):
        """wallDist: `bound` passes of the reference's inf-convolution kernel with
        the L1 kernel (distance_kernel(1, ndim, uint8, ord=1)), cut beyond `bound`."""
        nd = self.ndim
        L = lib(f"libagdref_infconv{nd}.so")
        L.agdref_infconv.restype = P
        X = np.meshgrid(*(np.arange(-1, 2),) * nd)
        kern = np.ascontiguousarray(np.round(sum(np.abs(x).astype(float) for x in X)).astype(np.uint8))
        wd = np.full(self.shape, 255, np.uint8)
        wd[walls] = 0
        out = np.empty_like(wd)
        res = L.agdref_infconv((ctypes.c_int * nd)(*self.shape), ptr(kern), bound, ptr(wd), ptr(out))
        arr = (wd if res == wd.ctypes.data else out).copy()
        arr[arr > bound] = 255
        return arr

    def cost_metric(self, cost):
        """Interface.CostMetric (_Interface.py:202-211): the metric with the grid
        scales and the cost applied, interpolated over the grid (index units)."""
        from agd import AutomaticDifferentiation as ad
        nd = self.ndim
        if self.model.startswith("Riemann"):
            metric = self.Metrics.Riemann.from_HFM(np.asarray(self.c["metric"], np.float64))
        elif self.model.startswith("Diagonal"):
            metric = self.Metrics.Diagonal.from_HFM(np.asarray(self.c["metric"], np.float64))
        elif self.model.startswith("Rander"):
            metric = self.rander(np.float64)
        else:
            metric = self.Metrics.Diagonal(np.ones(nd))
        cm = metric.with_costs(self.h.astype(np.float64)).with_cost(np.asarray(cost, np.float64))
        grid = ad.array(np.meshgrid(*(np.arange(s, dtype=np.float64) for s in self.shape), indexing="ij"))
        cm.set_interpolation(grid)
        return cm

    def spread_seed(self, seeds, seedValues, r, cost):
        """SetRHS's seed spreading (_SetArgs.py:46-75) with the reference's own
        metric interpolation."""
        assert len(seeds) == 1
        seed = self.point_from_index(seeds, to=True)[0].astype(np.float64)
        nd = self.ndim
        cm = self.cost_metric(cost)
        aX = [np.arange(int(np.floor(ci - r)), int(np.ceil(ci + r) + 1)) for ci in seed]
        neigh = np.stack(np.meshgrid(*aX, indexing="ij"), axis=-1).reshape(-1, nd)
        close = np.linalg.norm(neigh - seed, axis=-1) < r
        neigh = neigh[close]
        inRange = np.all(np.logical_and(-0.5 <= neigh, neigh < np.array(self.shape) - 0.5), axis=-1)
        neigh = neigh[inRange]
        diff = (neigh - seed).T
        m0, m1 = cm.at(seed), cm.at(neigh.T.astype(np.float64))
        vals = seedValues[0] + 0.5 * (m0.norm(diff) + m1.norm(diff))
        return neigh.astype(int), vals.astype(np.float32)

    def solve(self):
        md = self.md
        name = f"libagdref_eik_{md['tag']}{'mp' if self.multip else ''}{'f' if self.factor else ''}{self.o2tag}.so"
        L = lib(name)
        self.set_factor(L)
        trig_o = self.bexp(self.trigger, False).reshape(self.shape_o + (-1,)).any(-1).astype(np.uint8)
        nup = ctypes.c_longlong(0)
        L.agdref_fim_solve.restype = ctypes.c_int
        shp = (ctypes.c_int * self.ndim)(*self.shape)
        self.niter_o = L.agdref_fim_solve(
            shp, ctypes.c_float(self.atol), ctypes.c_float(self.rtol), md["front"], ptr(self.iso_w),
            ctypes.c_float(self.multip_step), ctypes.c_float(self.multip_max), ptr(self.values_b),
            ptr(self.valuesq_b), ptr(self.geom), ptr(self.seeds_b), ptr(self.rhs_b), ptr(trig_o), 2000,
            ctypes.byref(nup))
        self.tile_visits = nup.value

    @property
    def o2tag(self):
        return ("o" if int(self.c.get("order", 1)) == 2 else "") + ("w" if self.c.get("walls") is not None else "")

    def set_factor(self, L):
        if self.wall_b is not None:
            L.agdref_set_walls(ptr(self.wall_b))
        if "o" in self.o2tag:  # order2_threshold (_Kernel.py:310-314)
            L.agdref_set_order2(ctypes.c_float(float(self.c.get("order2_threshold", 0.3))))
        if self.factor:
            o, r2, m = self.factor
            L.agdref_set_factor(ptr(np.ascontiguousarray(o)), ctypes.c_float(r2), ptr(np.ascontiguousarray(m)))

    def values(self):
        v = self.values_b
        if self.multip:
            v = v + self.valuesq_b.astype(np.float32) * self.multip_step
        return self.bsq(v)

    def flow(self):
        assert not self.multip
        L = lib(f"libagdref_flow_{self.md['tag']}{'f' if self.factor else ''}{self.o2tag}.so")
        self.set_factor(L)
        nd, st = self.ndim, self.size_o * self.size_i
        nact = self.ndim * (self.ndim + 1) // 2 if self.model.startswith(("Riemann", "Rander")) else self.ndim
        self.nact = nact
        oi = self.shape_o + self.shape_i
        self.fw = np.empty((nact,) + oi, np.float32)
        self.fws = np.empty(oi, np.float32)
        self.fi = np.empty((nact,) + oi, np.int32)
        self.fv = np.empty((nd,) + oi, np.float32)
        L.agdref_flow((ctypes.c_int * nd)(*self.shape), ptr(self.iso_w), ctypes.c_float(0), ctypes.c_float(0),
                      ptr(self.values_b), None, ptr(self.geom), ptr(self.seeds_b), ptr(self.rhs_b),
                      ptr(self.fw), ptr(self.fws), ptr(self.fi), ptr(self.fv))
        self.flow_norm = None
        if self.model.startswith("Rander"):  # drift models: flow normalisation (_PostProcess.py:80-88)
            fv = np.stack([self.bsq(v) for v in self.fv])
            self.flow_norm = np.where(self.seedTags, np.float32(1), self.metric.norm(-fv)).astype(np.float32)

    def infconv_eucl(self):
        nd = self.ndim
        L = lib(f"libagdref_infconv{nd}.so")
        L.agdref_infconv.restype = P
        rg = np.arange(-1, 2)
        X = np.meshgrid(*(rg,) * nd)
        kern = np.round(5 * np.sqrt(sum(x.astype(float) ** 2 for x in X))).astype(np.uint8)
        kern = np.ascontiguousarray(kern)
        eucl = np.full(self.shape, 255, np.uint8)
        eucl[self.trigger] = 0
        out = np.empty_like(eucl)
        res = L.agdref_infconv((ctypes.c_int * nd)(*self.shape), ptr(kern), 6, ptr(eucl), ptr(out))
        arr = eucl if res == eucl.ctypes.data else out
        arr = arr.copy()
        arr[arr > 5 * 6] = 255
        return arr

    def geodesics(self, tips, pastseed_delay=0):
        nd = self.ndim
        L = lib(f"libagdref_geo{nd}_{self.shape_i[0]}.so")
        eucl = self.infconv_eucl()
        eucl_b = self.bexp(eucl, 255).astype(np.uint8)
        step = 0.25
        max_len = int(max(40, 20 * np.max(self.shape) / step))
        typical_len = min(max_len, int(max(40, 0.5 * np.max(self.shape) / step)))
        tips_c = self.point_from_index(tips, to=True).astype(np.float32)
        geos = [[t.reshape(1, -1)] for t in tips_c]
        stops = ["Stopping criterion"] * len(tips_c)
        corresp = list(range(len(tips_c)))
        codes = ["Continue", "AtSeed", "InWall", "Stationnary", "PastSeed", "VanishingFlow"]
        geoIt, geoMaxIt = 0, int(np.ceil(max_len / typical_len))
        pastseed = pastseed_delay  # first chunk only (_GetGeodesics.py:107-109,133)
        while corresp:
            if geoIt >= geoMaxIt:
                break
            geoIt += 1
            nG = len(corresp)
            x_s = np.full((nG, typical_len, nd), np.nan, np.float32)
            x_s[:, 0, :] = np.stack([geos[i][-1][-1, :] for i in corresp])
            len_s = np.full(nG, -1, np.int32)
            stop_s = np.full(nG, -1, np.int8)
            L.agdref_geodesic_chunk((ctypes.c_int * nd)(*self.shape), nG, typical_len, pastseed,
                                    ctypes.c_float(4.0), ctypes.c_float(step), ptr(self.values_b),
                                    ptr(self.fv), ptr(self.fws), ptr(eucl_b), ptr(x_s), ptr(len_s),
                                    ptr(stop_s))
            nxt = []
            for i, x, l, s in zip(corresp, x_s, len_s, stop_s):
                geos[i].append(x[1:int(l)])
                if s != 0:
                    stops[i] = codes[int(s)]
                else:
                    nxt.append(i)
            corresp = nxt
            pastseed = 0
        cat = [np.concatenate(g, axis=0) for g in geos]
        phys = [self.point_from_index(g).T for g in cat]
        return phys, stops, eucl

    def reverse_ad(self, sens):
        """sens: (*shape, 1).  Returns (costSensitivity, seedValueSensitivity)."""
        nd = self.ndim
        diag = self.fws.copy()
        boundary = diag == 0.0
        diag[boundary] = 1.0
        invalid = np.iinfo(np.int32).max
        indices = self.fi.copy()
        weights = self.fw
        indices[weights == 0] = invalid
        idxT, wT = self.graph_reverse(indices, weights, invalid)
        rhs = self.bexp(np.moveaxis(sens, -1, 0).astype(np.float32), np.nan)
        rhs = np.ascontiguousarray(rhs.astype(np.float32))
        tag = self.md.get("lin", self.md["tag"])
        L = lib(f"libagdref_lin_{tag}_r.so")
        L.agdref_nindex.restype = ctypes.c_int
        nidx = L.agdref_nindex()
        assert len(idxT) <= nidx, (len(idxT), nidx)
        st = self.size_o * self.size_i
        idx_pad = np.full((nidx, st), invalid, np.int32)
        w_pad = np.zeros((nidx, st), np.float32)
        idx_pad[: len(idxT)] = idxT.reshape(len(idxT), -1)
        w_pad[: len(wT)] = wT.reshape(len(wT), -1)
        float_res = np.finfo(np.float32).resolution
        rtol = np.float32(float_res * 5)
        fin = rhs[np.isfinite(rhs)]
        atol = np.float32(rtol * np.mean(np.abs(fin)))
        sol = np.full(rhs.shape, np.inf, np.float32)
        domain = np.isfinite(self.values_b)
        trigger = np.logical_and(np.all(w_pad.reshape((nidx,) + domain.shape) == 0.0, axis=0), domain)
        trig_o = trigger.reshape(self.shape_o + (-1,)).any(-1).astype(np.uint8)
        self.rev_niter = L.agdref_linear_solve((ctypes.c_int * nd)(*self.shape_o), ctypes.c_float(atol),
                                               ctypes.c_float(rtol), ptr(sol), ptr(rhs), ptr(diag),
                                               ptr(idx_pad), ptr(w_pad), ptr(trig_o), 2000)
        allS = np.moveaxis(self.bsq(sol), 0, -1)
        pos = tuple(self.seedIndices.T)
        seedS = allS[pos].copy()
        allS[pos] = 0
        if self.flow_norm is not None:  # _PostProcess.py:213-214
            allS = allS / self.flow_norm[..., None]
        return allS, seedS

    def forward_ad(self, cost_var, seed_var):
        """Forward AD, _PostProcess.py:181-191: cost_var (*shape, n), seed_var
        (n, nseeds) as the reference's seedValueVariation key (_SetArgs.py:30-33); rhs = seed variation at seeds, cost variation * cost elsewhere,
        solved with the forward flow graph.  Returns valueVariation (*shape, n)."""
        nd = self.ndim
        diag = self.fws.copy()
        diag[diag == 0.0] = 1.0
        indices, weights = self.fi, self.fw
        cost = np.asarray(self.c.get("cost", np.ones(self.shape, np.float32)), np.float32)
        cost = np.broadcast_to(cost, self.shape)
        value = cost.copy()
        pos = tuple(self.seedIndices.T)
        value[pos] = np.asarray(self.c.get("seedValues", np.zeros(len(self.seedIndices))), np.float32)
        n_ad = cost_var.shape[-1]
        grad = np.moveaxis(np.asarray(cost_var, np.float32), -1, 0).copy()
        for j in range(n_ad):
            grad[j][pos] = seed_var[j]
        rhs_grid = np.where(self.seedTags, grad, grad * value).astype(np.float32)
        if self.flow_norm is not None:  # _PostProcess.py:185
            rhs_grid = (rhs_grid * self.flow_norm).astype(np.float32)
        L = lib(f"libagdref_lin_{self.md.get('lin', self.md['tag'])}_f.so")
        L.agdref_nindex.restype = ctypes.c_int
        assert L.agdref_nindex() == len(indices)
        float_res = np.finfo(np.float32).resolution
        rtol = np.float32(float_res * 5)
        domain = np.isfinite(self.values_b)
        trigger = np.logical_and(np.all(weights == 0.0, axis=0), domain)
        trig_o = trigger.reshape(self.shape_o + (-1,)).any(-1).astype(np.uint8)
        out = []
        for j in range(n_ad):
            rhs = np.ascontiguousarray(self.bexp(rhs_grid[j], np.nan).astype(np.float32))
            fin = rhs[np.isfinite(rhs)]
            atol = np.float32(rtol * np.mean(np.abs(fin)))
            sol = np.full(rhs.shape, np.inf, np.float32)
            L.agdref_linear_solve((ctypes.c_int * nd)(*self.shape_o), ctypes.c_float(atol), ctypes.c_float(rtol),
                                  ptr(sol), ptr(rhs), ptr(diag), ptr(np.ascontiguousarray(indices)),
                                  ptr(np.ascontiguousarray(weights)), ptr(trig_o), 2000)
            out.append(self.bsq(sol))
        return np.stack(out, -1)

    def graph_reverse(self, fwd, fwd_weight, invalid, nrev=None):
        L = lib("libagdref_graphrev.so")
        nfwd = len(fwd)
        shape = fwd.shape[1:]
        size = int(np.prod(shape))
        if nrev is None:
            nrev = 2 * nfwd
        assert nrev <= 127
        rev = np.full((nrev,) + shape, invalid, np.int32)
        rev_w = np.zeros((nrev,) + shape, np.float32)
        irev = np.zeros((nfwd,) + shape, np.int8)
        fwd = np.ascontiguousarray(fwd)
        fwd_weight = np.ascontiguousarray(fwd_weight)
        irev_mmax = 0
        for _ in range(nrev):
            irev_max = int(np.max(irev))
            irev_mmax = max(irev_max, irev_mmax)
            if irev_max == -1:
                return rev[: irev_mmax + 1], rev_w[: irev_mmax + 1]
            if irev_max == nrev:
                return self.graph_reverse(fwd, fwd_weight, invalid, 2 * nrev)
            L.agdref_graph_reverse_launch(size, nfwd, nrev, ptr(fwd), ptr(rev), ptr(irev), ptr(fwd_weight),
                                          ptr(rev_w))
        raise RuntimeError("graph_reverse did not terminate")


# ----------------------------------------------------------------------------
# Cases
# ----------------------------------------------------------------------------
def rect(dims, h, origin=None):
    dims = np.asarray(dims, np.float32)
    return dict(dims=dims, gridScales=np.full(len(dims), h, np.float32),
                origin=np.zeros(len(dims), np.float32) if origin is None else np.asarray(origin, np.float32))


def make_cases():
    cases = {}
    rng = np.random.default_rng(1234)
    # Isotropic2, non-multiple-of-tile shape, variable cost, two seeds, tips, receivers
    sh = (70, 53)
    c = dict(model="Isotropic2", **rect(sh, 1.0 / 70))
    c["cost"] = np.exp(0.5 * smooth_noise(rng, sh, 3.0)).astype(np.float32)
    c["seeds"] = np.array([[0.31, 0.22], [0.72, 0.55]], np.float32)
    c["seedValues"] = np.array([0.0, 0.05], np.float32)
    c["tips"] = c["seeds"][:1] * 0 + rng.uniform(0.05, 0.7, (6, 2)).astype(np.float32)
    cases["iso2"] = c
    # Riemann2 anisotropic, three seeds with seed values
    sh = (61, 77)
    c = dict(model="Riemann2", **rect(sh, 1.0 / 61))
    m = riemann2_metric(rng, sh, 6.0, 20.0)
    c["metric"] = np.moveaxis(np.stack([m[0, 0], m[1, 0], m[1, 1]]), 0, -1)
    c["seeds"] = np.array([[0.2, 0.3], [0.7, 0.9], [0.5, 0.6]], np.float32)
    c["seedValues"] = np.array([0.0, 0.1, 0.05], np.float32)
    c["tips"] = rng.uniform(0.05, 0.95, (6, 2)).astype(np.float32) * np.array([1.0, 77 / 61], np.float32)
    cases["riem2"] = c
    # Same Riemann2 problem with the multiprecision option
    c2 = dict(c)
    c2["multiprecision"] = True
    c2.pop("tips")
    cases["riem2_mp"] = c2
    # Riemann2 with the anisotropy range of the 1024^2 workload (lambda in [1,100])
    sh = (64, 64)
    c = dict(model="Riemann2", **rect(sh, 1.0 / 64))
    m = riemann2_metric(rng, sh, 4.0, 100.0)
    c["metric"] = np.moveaxis(np.stack([m[0, 0], m[1, 0], m[1, 1]]), 0, -1)
    c["seeds"] = rng.uniform(0.1, 0.9, (4, 2)).astype(np.float32)
    c["tips"] = rng.uniform(0.05, 0.95, (8, 2)).astype(np.float32)
    cases["riem2_aniso"] = c
    # Isotropic3
    sh = (21, 18, 23)
    c = dict(model="Isotropic3", **rect(sh, 1.0 / 21))
    c["cost"] = np.exp(0.5 * smooth_noise(rng, sh, 2.0)).astype(np.float32)
    c["seeds"] = np.array([[0.5, 0.4, 0.5]], np.float32)
    c["tips"] = rng.uniform(0.05, 0.8, (4, 3)).astype(np.float32)
    cases["iso3"] = c
    # Riemann3
    sh = (20, 22, 19)
    c = dict(model="Riemann3", **rect(sh, 1.0 / 20))
    m = riemann3_metric(rng, sh, 2.0, 9.0)
    c["metric"] = np.moveaxis(np.stack([m[i, j] for i in range(3) for j in range(i + 1)]), 0, -1)
    c["seeds"] = np.array([[0.45, 0.5, 0.48]], np.float32)
    c["tips"] = rng.uniform(0.05, 0.9, (4, 3)).astype(np.float32)
    cases["riem3"] = c
    # EikonalAD_GPU.ipynb cells 35-42: seedValueSensitivity == [[0],[1]]
    n = 50
    c = dict(model="Isotropic2", dims=np.array([n + 1, n + 1], np.float32),
             gridScales=np.full(2, 1.0 / n, np.float32), origin=np.full(2, -0.5 / n, np.float32))
    c["seeds"] = np.array([[0.0, 0.0], [0.0, 0.5]], np.float32)
    c["cost"] = np.ones((n + 1, n + 1), np.float32)
    c["traits"] = dict(shape_i=(8, 8), niter_i=16)
    sens = np.zeros((n + 1, n + 1, 1), np.float32)
    sens[-1, -1] = 1.0
    c["sensitivity"] = sens
    cases["ad_notebook"] = c
    # receivers sensitivity for the other AD cases
    for key in ("iso2", "riem2", "riem3", "iso3"):
        cc = cases[key]
        shp = tuple(int(s) for s in cc["dims"])
        sens = np.zeros(shp + (1,), np.float32)
        flat = rng.choice(int(np.prod(shp)), 5, replace=False)
        sens.reshape(-1)[flat] = 1.0
        cc["sensitivity"] = sens
    # seeds spread over a radius (_SetArgs.py:46-75): Riemann2 anisotropic, Isotropic2
    c = dict(cases["riem2"])
    for k in ("tips", "sensitivity", "seedValues"):
        c.pop(k, None)
    c["seeds"] = np.array([[0.43, 0.61]], np.float32)
    c["seedValues"] = np.array([0.02], np.float32)
    c["seedRadius"] = 2.5
    cases["riem2_radius"] = c
    c = dict(cases["iso2"])
    for k in ("tips", "sensitivity", "seedValues"):
        c.pop(k, None)
    c["seeds"] = np.array([[0.37, 0.3]], np.float32)
    c["seedRadius"] = 2.0
    cases["iso2_radius"] = c
    # source factorisation (factoringRadius), seeds spread over the default radius 2
    c = dict(cases["riem2_radius"])
    c.pop("seedRadius")
    c["factoringRadius"] = 10.0
    c["tips"] = np.array([[0.2, 0.35], [0.8, 1.1], [0.6, 0.5]], np.float32)
    cases["riem2_factor"] = c
    c = dict(cases["iso2_radius"])
    c.pop("seedRadius")
    c["factoringRadius"] = 12.0
    cases["iso2_factor"] = c
    # second order scheme (order: 2)
    for key in ("riem2", "iso2", "riem3"):
        c = {k: v for k, v in cases[key].items() if k != "sensitivity"}
        c["order"] = 2
        cases[key + "_order2"] = c
    # tips a few pixels from the seeds, with the PastSeed test delayed by 20 steps:
    # the first four stop as PastSeed within a few steps without the delay
    c = {k: v for k, v in cases["riem2"].items() if k != "sensitivity"}
    c["pastseed_delay"] = 20
    c["tips"] = np.array([[0.1958, 0.2319], [0.6943, 0.9547], [0.6748, 0.8182], [0.4959, 0.5293],
                          [0.25, 0.3], [0.7, 0.95]], np.float32)
    cases["riem2_pastseed"] = c
    # walls (obstacles), with a gap, a one-pixel diagonal wall (leaky for diagonal
    # offsets, as the reference's visibility test is) and a tip inside a wall
    c = {k: v for k, v in cases["riem2"].items() if k != "sensitivity"}
    w = np.zeros((61, 77), bool)
    w[25, 5:70] = True
    w[25, 40:44] = False
    for i in range(35, 56):
        w[i, i + 10] = True
    c["walls"] = w
    c["tips"] = np.array([[0.418, 0.3], [0.1, 0.5], [0.6, 0.2], [0.3, 1.1], [0.9, 0.7]], np.float32)
    cases["riem2_walls"] = c
    c = {k: v for k, v in cases["iso2"].items() if k != "sensitivity"}
    w = np.zeros((70, 53), bool)
    w[10:65, 26] = True
    w[40:43, 26] = False
    c["walls"] = w
    cases["iso2_walls"] = c
    c = {k: v for k, v in cases["riem3"].items() if k != "sensitivity"}
    w = np.zeros((20, 22, 19), bool)
    w[:, 14, :] = True
    w[8:12, 14, 6:10] = False
    c["walls"] = w
    c["wallDistBound"] = 3
    c["tips"] = np.array([[0.5, 0.95, 0.5], [0.2, 0.3, 0.8]], np.float32)
    cases["riem3_walls"] = c
    # forward AD inputs (drawn last, so that the inputs above do not change):
    # two variations of the cost, and of the seed values
    for key in ("iso2", "riem2", "riem3"):
        cc = cases[key]
        shp = tuple(int(s) for s in cc["dims"])
        cv = np.stack([smooth_noise(rng, shp, 2.0), np.zeros(shp)], -1).astype(np.float32)
        cv[..., 1].reshape(-1)[rng.choice(int(np.prod(shp)), 3, replace=False)] = 1.0
        cc["costVariation"] = cv
        cc["seedValueVariation"] = np.ascontiguousarray(rng.uniform(-1, 1, (len(cc["seeds"]), 2)).T).astype(np.float32)
    # Diagonal models (axis costs per point), with their own random stream
    rng = np.random.default_rng(4321)
    sh = (70, 53)
    c = dict(model="Diagonal2", **rect(sh, 1.0 / 70))
    c["metric"] = np.stack([np.exp(0.4 * smooth_noise(rng, sh, 3.0)), 2.0 * np.exp(0.4 * smooth_noise(rng, sh, 3.0))],
                           -1).astype(np.float32)  # HFM layout (*shape, ndim): the costs per axis
    c["cost"] = np.exp(0.3 * smooth_noise(rng, sh, 4.0)).astype(np.float32)
    c["seeds"] = np.array([[0.31, 0.22], [0.72, 0.55]], np.float32)
    c["seedValues"] = np.array([0.0, 0.05], np.float32)
    c["tips"] = rng.uniform(0.05, 0.7, (5, 2)).astype(np.float32)
    sens = np.zeros(sh + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(sh)), 5, replace=False)] = 1.0
    c["sensitivity"] = sens
    cases["diag2"] = c
    c = {k: v for k, v in cases["diag2"].items() if k not in ("sensitivity", "seedValues", "tips")}
    c["seeds"] = np.array([[0.37, 0.3]], np.float32)
    c["factoringRadius"] = 10.0
    cases["diag2_factor"] = c
    c = {k: v for k, v in cases["diag2"].items() if k != "sensitivity"}
    c["order"] = 2
    cases["diag2_order2"] = c
    c = {k: v for k, v in cases["diag2"].items() if k != "sensitivity"}
    w = np.zeros(sh, bool)
    w[10:65, 26] = True
    w[40:43, 26] = False
    c["walls"] = w
    cases["diag2_walls"] = c
    sh = (21, 18, 23)
    c = dict(model="Diagonal3", **rect(sh, 1.0 / 21))
    c["metric"] = np.stack([np.exp(0.4 * smooth_noise(rng, sh, 2.0)) for _ in range(3)], -1).astype(np.float32)
    c["seeds"] = np.array([[0.5, 0.4, 0.5]], np.float32)
    c["tips"] = rng.uniform(0.05, 0.8, (3, 3)).astype(np.float32)
    sens = np.zeros(sh + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(sh)), 5, replace=False)] = 1.0
    c["sensitivity"] = sens
    cases["diag3"] = c
    cc = cases["diag2"]
    cv = np.stack([smooth_noise(rng, sh2 := (70, 53), 2.0), np.zeros(sh2)], -1).astype(np.float32)
    cv[..., 1].reshape(-1)[rng.choice(70 * 53, 3, replace=False)] = 1.0
    cc["costVariation"] = cv
    cc["seedValueVariation"] = np.ascontiguousarray(rng.uniform(-1, 1, (2, 2)).T).astype(np.float32)
    # Rander models (Riemann metric plus a drift with |w|_{M^-1} < 1), own random stream
    rng = np.random.default_rng(8765)

    def rander(shape, nd, sigma, lam_max, wmax):
        m = riemann2_metric(rng, shape, sigma, lam_max) if nd == 2 else riemann3_metric(rng, shape, sigma, lam_max)
        M = np.moveaxis(m, (0, 1), (-2, -1)).astype(np.float64)
        w = np.stack([smooth_noise(rng, shape, sigma) for _ in range(nd)], -1)
        # scale the drift to a fraction of the unit ball of the dual norm: |w|_{M^-1} <= wmax
        wn = np.sqrt(np.einsum("...i,...ij,...j->...", w, np.linalg.inv(M), w))
        w = w / wn.max() * wmax
        flat = np.stack([M[..., i, j] for i in range(nd) for j in range(i + 1)], -1)
        return np.concatenate([flat, w], -1).astype(np.float32)  # HFM layout (*shape, symdim + ndim)
    sh = (61, 77)
    c = dict(model="Rander2", **rect(sh, 1.0 / 61))
    c["metric"] = rander(sh, 2, 6.0, 10.0, 0.7)
    c["seeds"] = np.array([[0.2, 0.3], [0.7, 0.9]], np.float32)
    c["seedValues"] = np.array([0.0, 0.1], np.float32)
    c["tips"] = rng.uniform(0.05, 0.95, (5, 2)).astype(np.float32) * np.array([1.0, 77 / 61], np.float32)
    sens = np.zeros(sh + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(sh)), 5, replace=False)] = 1.0
    c["sensitivity"] = sens
    cv = np.stack([smooth_noise(rng, sh, 2.0), np.zeros(sh)], -1).astype(np.float32)
    cv[..., 1].reshape(-1)[rng.choice(int(np.prod(sh)), 3, replace=False)] = 1.0
    c["costVariation"] = cv
    c["seedValueVariation"] = np.ascontiguousarray(rng.uniform(-1, 1, (2, 2)).T).astype(np.float32)
    cases["rand2"] = c
    c = {k: v for k, v in cases["rand2"].items() if k not in ("sensitivity", "costVariation", "seedValueVariation",
                                                              "seedValues")}
    c["seeds"] = np.array([[0.43, 0.61]], np.float32)
    c["factoringRadius"] = 8.0
    c["tips"] = c["tips"][:3]
    cases["rand2_factor"] = c
    c = {k: v for k, v in cases["rand2"].items() if k not in ("sensitivity", "costVariation", "seedValueVariation")}
    c["order"] = 2
    cases["rand2_order2"] = c
    c = {k: v for k, v in cases["rand2"].items() if k not in ("sensitivity", "costVariation", "seedValueVariation")}
    w = np.zeros(sh, bool)
    w[25, 5:70] = True
    w[25, 40:44] = False
    c["walls"] = w
    cases["rand2_walls"] = c
    c = {k: v for k, v in cases["rand2"].items() if k not in ("sensitivity", "costVariation", "seedValueVariation",
                                                              "tips")}
    c["multiprecision"] = True
    cases["rand2_mp"] = c
    sh = (20, 22, 19)
    c = dict(model="Rander3", **rect(sh, 1.0 / 20))
    c["metric"] = rander(sh, 3, 2.0, 6.0, 0.6)
    c["seeds"] = np.array([[0.45, 0.5, 0.48]], np.float32)
    c["tips"] = rng.uniform(0.05, 0.9, (3, 3)).astype(np.float32)
    sens = np.zeros(sh + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(sh)), 5, replace=False)] = 1.0
    c["sensitivity"] = sens
    cases["rand3"] = c
    # Riemann3 32^3 with the 200^3 workload's metric distribution (eigenvalues
    # log-uniform in [1, 25], orientations smoothed over 6 voxels in proportion),
    # one source, reverse sensitivity of 24 receivers: the largest 3D size the
    # host build of the reference's kernels solves in a few minutes; own stream
    rng = np.random.default_rng(3232)
    sh = (32, 32, 32)
    c = dict(model="Riemann3", **rect(sh, 1.0 / 32))
    m = riemann3_metric(rng, sh, 6.0 * 32 / 200 * 4, 25.0)
    c["metric"] = np.moveaxis(np.stack([m[i, j] for i in range(3) for j in range(i + 1)]), 0, -1)
    c["cost"] = np.exp(0.3 * smooth_noise(rng, sh, 3.0)).astype(np.float32)
    c["seeds"] = np.array([[0.5, 0.5, 0.5]], np.float32)
    sens = np.zeros(sh + (1,), np.float32)
    sens.reshape(-1)[rng.choice(int(np.prod(sh)), 24, replace=False)] = 1.0
    c["sensitivity"] = sens
    cases["riem3_32"] = c
    # source factorisation with multiprecision (the reference composes the two)
    for key in ("riem2_factor", "iso2_factor"):
        c = {k: v for k, v in cases[key].items() if k not in ("tips", "sensitivity")}
        c["multiprecision"] = True
        cases[key + "_mp"] = c
    c = {k: v for k, v in cases["riem3"].items() if k not in ("tips", "sensitivity")}
    c["seeds"] = np.array([[0.45, 0.5, 0.48]], np.float32)
    c["factoringRadius"] = 5.0
    c["multiprecision"] = True
    cases["riem3_factor_mp"] = c
    # the second order scheme with source factorisation, and with multiprecision
    for key in ("riem2_factor", "iso2_factor"):
        c = {k: v for k, v in cases[key].items() if k not in ("tips", "sensitivity")}
        c["order"] = 2
        cases[key.replace("_factor", "_order2_factor")] = c
    c = {k: v for k, v in cases["riem3_factor_mp"].items() if k != "multiprecision"}
    c["order"] = 2
    cases["riem3_order2_factor"] = c
    for key in ("riem2_order2", "iso2_order2", "riem3_order2"):
        c = {k: v for k, v in cases[key].items() if k not in ("tips", "sensitivity")}
        c["multiprecision"] = True
        cases[key + "_mp"] = c
    for key in ("riem2_order2_factor", "iso2_order2_factor", "riem3_order2_factor"):
        c = dict(cases[key])
        c["multiprecision"] = True
        cases[key + "_mp"] = c
    return cases


def run_case(name, case):
    pipe = RefPipeline(case)
    if "traits" in case:
        tr = case["traits"]
        assert pipe.model == "Isotropic2" and tuple(tr["shape_i"]) == (8, 8) and tr["niter_i"] == 16
        pipe.md = dict(pipe.md, shape_i=(8, 8), niter_i=16, tag="iso2s8")
        pipe.shape_i = pipe.md["shape_i"]
        pipe.size_i = int(np.prod(pipe.shape_i))
        pipe.shape_o = tuple(int(x) for x in pipe.fd.round_up_ratio(np.array(pipe.shape), np.array(pipe.shape_i)))
        pipe.size_o = int(np.prod(pipe.shape_o))
    pipe.setup()
    pipe.solve()
    out = dict(values=pipe.values().astype(np.float32), niter_o=pipe.niter_o, tile_visits=pipe.tile_visits,
               atol=pipe.atol, rtol=pipe.rtol)
    if pipe.wall_b is not None:
        out["wall_dist"] = pipe.wall_grid
    if not pipe.multip:
        pipe.flow()
        out["values_after_flow"] = pipe.values().astype(np.float32)
        out["flow_vector"] = np.stack([pipe.bsq(v) for v in pipe.fv]).astype(np.float32)
        out["flow_weightsum"] = pipe.bsq(pipe.fws).astype(np.float32)
        if pipe.flow_norm is not None:  # hfmOut['flow'] of a drift model: normalised, physical units
            h = pipe.h.reshape((-1,) + (1,) * pipe.ndim)
            out["flow_export"] = (out["flow_vector"] / pipe.flow_norm * -h).astype(np.float32)
        # exportActiveNeighs: positive flow weights as bits (cuda/Update.h:187,206)
        out["activeNeighs"] = sum((pipe.bsq(w) > 0).astype(np.int32) << k for k, w in enumerate(pipe.fw))
        if "tips" in case:
            geos, stops, eucl = pipe.geodesics(case["tips"], int(case.get("pastseed_delay", 0)))
            out["geodesic_lengths"] = np.array([g.shape[1] for g in geos], np.int32)
            out["geodesics_concat"] = np.concatenate(geos, axis=1).astype(np.float32)
            out["geodesic_stopping_criteria"] = np.array(stops)
            out["eucl"] = eucl
        if "costVariation" in case:
            out["valueVariation"] = pipe.forward_ad(case["costVariation"], case["seedValueVariation"]).astype(
                np.float32)
        if "sensitivity" in case:
            cs, ss = pipe.reverse_ad(case["sensitivity"])
            out["costSensitivity"] = cs.astype(np.float32)
            out["seedValueSensitivity"] = ss.astype(np.float32)
    return out


def selling_fixture(rng, nd, n):
    """Reference kernel decomposition (fp32) and agd.Selling (fp64) of random SPD tensors."""
    from agd import Selling
    if nd == 2:
        th = rng.uniform(0, np.pi, n)
        lam = np.exp(rng.uniform(0, np.log(100), n))
        c, s = np.cos(th), np.sin(th)
        M = np.stack([np.stack([c * c + lam * s * s, c * s * (1 - lam)]),
                      np.stack([c * s * (1 - lam), s * s + lam * c * c])])
        flat = np.stack([M[0, 0], M[1, 0], M[1, 1]], -1).astype(np.float32)
    else:
        a = rng.standard_normal((n, 3, 3))
        q, _ = np.linalg.qr(a)
        ev = np.exp(rng.uniform(0, np.log(50), (n, 3)))
        Mm = q @ (ev[:, :, None] * np.swapaxes(q, 1, 2))
        M = np.moveaxis(Mm, 0, -1)
        flat = np.stack([Mm[:, i, j] for i in range(3) for j in range(i + 1)], -1).astype(np.float32)
    sd = nd * (nd + 1) // 2
    L = lib(f"libagdref_eik_riem{nd}.so")
    w = np.zeros((n, sd), np.float32)
    e = np.zeros((n, sd, nd), np.int32)
    L.agdref_selling(ptr(np.ascontiguousarray(flat)), n, ptr(w), ptr(e))
    M64 = np.zeros((nd, nd, n))
    k = 0
    for i in range(nd):
        for j in range(i + 1):
            M64[i, j] = flat[:, k]
            M64[j, i] = flat[:, k]
            k += 1
    cw, ce = Selling.Decomposition(M64)
    return dict(m=flat, ref_w=w, ref_e=e, agd_w=np.moveaxis(cw, -1, 0), agd_e=np.moveaxis(ce, -1, 0).transpose(0, 2, 1).astype(np.int32))


def save(name, case, out):
    d = {}
    for k, v in case.items():
        if k == "traits":
            d["in_traits_shape_i"] = np.array(v["shape_i"], np.int32)
            d["in_traits_niter_i"] = np.int32(v["niter_i"])
        elif k == "model":
            d["in_model"] = np.array(v)
        else:
            d["in_" + k] = np.asarray(v)
    for k, v in out.items():
        d["out_" + k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("AGD_REFERENCE") or
                    os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                                 "..", "reference"))
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    sys.path.insert(0, args.ref)
    cases = make_cases()
    for name, case in cases.items():
        if args.only and name != args.only:
            continue
        out = run_case(name, case)
        save(name, case, out)
        print(name, "niter_o", out["niter_o"], "visits", out["tile_visits"],
              "stops", list(out.get("geodesic_stopping_criteria", [])))
    if not args.only or args.only.startswith("selling"):
        rng = np.random.default_rng(99)
        for nd in (2, 3):
            f = selling_fixture(rng, nd, 3000)
            np.savez_compressed(os.path.join(HERE, f"selling{nd}.npz"), **f)
            print("selling", nd)


if __name__ == "__main__":
    main()
