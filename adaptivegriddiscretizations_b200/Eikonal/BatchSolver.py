"""Repeated batched solves of one problem configuration (the serving path).

A template dictIn fixes the model, the grid, the tile traits, the tolerances and
the solver options (and, optionally, obstacles shared by every instance); every
submission brings the per-instance data of a batch (metrics or costs, seeds,
seed values, optionally obstacles) as arrays with a leading batch axis.
Device buffers and the solver plan are made once.  A submission queues on its
own CUDA stream: the upload of the host inputs (without blocking the host when
they are page-locked), two batched preparation kernels (agd_prep_batch), the
persistent solve (agd_plan_run), the reordering of the values into grid order
(agd_block_squeeze) and, when a host buffer is given, their copy back.  Buffer
sets alternate, so the host submits batch k+1 while the device solves batch k.

The reference solves one dictIn per Run() call (agd/Eikonal/HFM_CUDA/__init__.py:10-25)
and has no counterpart of this class; the values are the ones RunGPU returns for
the same inputs (same keys, defaults and tolerances, read from the template by
the Interface of HFM_CUDA).  Only the values are produced: flow, geodesics and
sensitivities go through RunGPU / RunBatch.
"""
import ctypes
import warnings

import numpy as np
import torch

from .. import _lib
from .HFM_CUDA import Interface, _FLOAT_RES


class _Buffers:
    """Device buffers, plan workspace and stream of one in-flight batch."""

    def __init__(self, solver):
        s = solver
        self.stream = torch.cuda.Stream()
        with torch.cuda.stream(self.stream):  # owned by this stream for the allocator
            dev = dict(dtype=torch.float32, device="cuda")
            self.geom = torch.empty((s.batch, s.nmet * s.size_tot), **dev) if s.nmet else None
            self.rhs = torch.empty((s.batch, s.size_tot), **dev)
            self.values = torch.empty((s.batch, s.size_tot), **dev)
            self.seedbits = torch.empty((s.batch, s.size_tot // 8), dtype=torch.uint8, device="cuda")
            self.out = torch.empty((s.batch,) + s.shape, **dev)
            self.stats = torch.zeros((s.batch, 2), dtype=torch.int64, device="cuda")
            self.bad = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.stats_host = torch.empty((s.batch, 2), dtype=torch.int64).pin_memory()
        self.bad_host = torch.empty(1, dtype=torch.int32).pin_memory()
        self.metric = self.cost = self.seed_index = self.seed_values = None  # staging, made on first use
        self.release = None  # tile release epochs (batch, tiles) uint16, made on first use
        self.wall_dist = None  # per-instance wall distances (batch, size_tot) uint8, made on first use
        self.trigger = None  # first tiles with walls (batch, tiles) uint8, made on first use
        self.plan = None
        self.plan_key = None
        self.ws = None
        self.job = None

    def staging(self, name, shape, dtype=torch.float32):
        """Device staging tensor for an input, reused while its shape holds."""
        t = getattr(self, name, None)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            with torch.cuda.stream(self.stream):
                t = torch.empty(shape, dtype=dtype, device="cuda")
            setattr(self, name, t)
        return t


class SolverJob:
    """A batch submitted to a BatchSolver; `result()` waits for it."""

    def __init__(self, solver, buf, out, dev_out=None):
        self.solver, self.buf, self.out, self.dev_out = solver, buf, out, dev_out
        self.event = torch.cuda.Event()
        self.event.record(buf.stream)
        self.stream = buf.stream
        self._done = False
        self.niter_o = self.tile_visits = None

    def done(self):
        return self.event.query()

    def result(self):
        """Values of the batch, shape (batch, *grid shape): the host buffer given to
        submit(), else a device tensor: its own with submit(fresh_out=True), or
        the buffer set's, valid until the set is reused (after the solver's
        `nbuffers` next submissions)."""
        self.event.synchronize()
        if not self._done:
            self._done = True
            s = self.buf.stats_host.numpy()
            self.niter_o = (s[:, 0] & 0xffffffff).astype(np.int64)
            status = ((s[:, 0] >> 32) & 0xffffffff).astype(np.int64)
            self.tile_visits = s[:, 1].copy()
            if int(self.buf.bad_host[0]):
                raise ValueError("Seeds outside the domain")
            bad = np.nonzero(status & ~_lib.AGD_STATUS_NOT_CONVERGED)[0]
            if len(bad):
                raise _lib.AgdError(int(status[bad[0]]), f"eikonal solve failed on the device (instance {bad[0]})")
            nc = np.nonzero(status & _lib.AGD_STATUS_NOT_CONVERGED)[0]
            if len(nc):
                msg = f"{len(nc)} instance(s) did not reach convergence after {self.solver.nitermax_o} iterations"
                if self.solver.raiseOnNonConvergence:
                    raise ValueError(msg)
                warnings.warn(msg)
        if self.out is not None:
            return self.out
        if self.dev_out is not None:
            # (made on the buffer set's stream: the caller's stream uses it from now on)
            self.dev_out.record_stream(torch.cuda.current_stream())
            return self.dev_out
        return self.buf.out


class BatchSolver:
    """Solves batches of `batch` instances of the configuration of `template`.

    template: a dictIn whose keys (model, dims/gridScale(s)/origin, traits,
    tol/atol/rtol, nitermax_o, fim_front_width, walls, wallDistBound, ...) apply
    to every instance; it may hold data of one instance (metric, cost, seeds),
    which is read only to check the keys.  submit(metric=, cost=, seeds=,
    seedValues=, walls=, out=) takes arrays with a leading batch axis: metric
    (batch, *shape, k) in HFM packing (Riemann: k = symdim; Diagonal: the costs
    per axis, k = ndim; Rander: metric then drift, k = symdim + ndim), cost
    (batch, *shape) (required by Isotropic models, optional for the others),
    seeds (batch, nseeds, ndim) points, seedValues (batch, nseeds), walls
    (batch, *shape) booleans (instead of the template's walls).  Host tensors
    are copied in (page-locked ones without blocking), device tensors are read
    in place."""

    _MODELS = ("Riemann", "Isotropic", "Diagonal", "Rander")

    def __init__(self, template, batch, nbuffers=2, launch=None):
        if batch < 1 or nbuffers < 1:
            raise ValueError("batch and nbuffers must be positive")
        model = str(template["model"])
        if "metric" not in template and "dualMetric" not in template and model[:-1] in ("Riemann", "Diagonal", "Rander"):
            # the configuration needs no data: a constant metric stands in for the check of the keys
            template = template.copy()
            nd = int(model[-1])
            eye = np.eye(nd, dtype=np.float32)[np.tril_indices(nd)]
            template["metric"] = {"Riemann": eye, "Diagonal": np.ones(nd, np.float32),
                                  "Rander": np.concatenate([eye, np.zeros(nd, np.float32)])}[model[:-1]]
        itf = Interface(template)
        itf.SetKernelTraits()
        itf.SetGeometry()
        if itf.multiprecision:
            raise NotImplementedError("BatchSolver: multiprecision instances go through RunBatch")
        for key in ("tips", "sensitivity", "exportGeodesicFlow", "seedRadius", "speed", "dualMetric"):
            if key in template and template[key] is not None and template[key] is not False:
                raise NotImplementedError(f"BatchSolver: key {key!r} is not available on the batched path")
        self.template = template
        self.batch, self.nbuffers = int(batch), int(nbuffers)
        self.model = itf.model
        if itf.model_ not in self._MODELS:
            raise NotImplementedError(f"BatchSolver: model {itf.model} goes through RunGPU / RunBatch")
        self.model_code = {"Riemann": _lib.AGD_MODEL_RIEMANN, "Isotropic": _lib.AGD_MODEL_ISOTROPIC,
                           "Diagonal": _lib.AGD_MODEL_DIAGONAL, "Rander": _lib.AGD_MODEL_RANDER}[itf.model_]
        self.riemann = itf.model_ == "Riemann"
        self.ndim = itf.ndim
        self.symdim = self.ndim * (self.ndim + 1) // 2
        # metric floats per point (and geometry planes)
        self.nmet = {"Riemann": self.symdim, "Isotropic": 0, "Diagonal": self.ndim,
                     "Rander": self.symdim + self.ndim}[itf.model_]
        self.shape, self.shape_i = tuple(itf.shape), tuple(itf.shape_i)
        self.size_tot = itf.size_tot
        self.ntiles = self.size_tot // int(np.prod(self.shape_i))
        self.h = np.asarray(itf.h, np.float32)
        bottom, _ = template.corners
        self.start = (bottom + 0.5 * self.h).astype(np.float32)
        self.niter_i, self.fim_front_width, self.nitermax_o = itf.niter_i, itf.fim_front_width, itf.nitermax_o
        self.flags = {"adaptive_gauss_siedel_iteration": _lib.AGD_FLAG_SOLVER_AGSI,
                      "global_iteration": _lib.AGD_FLAG_SOLVER_GLOBAL}.get(itf.solver, 0)
        self.raiseOnNonConvergence = itf.raiseOnNonConvergence
        self.rtol = itf.rtol
        # a tolerance given by the user holds for every instance; otherwise the
        # default follows each instance's mean cost, as for RunGPU
        self.fixed_atol = itf.atol if ("atol" in template or "tol" in template) else None
        self.launch = launch
        self.c_shape = (ctypes.c_int * 3)(*self.shape, *([1] * (3 - self.ndim)))
        self.c_shape_i = (ctypes.c_int * 3)(*self.shape_i, *([1] * (3 - self.ndim)))
        # obstacles of the template, shared by every instance: mask and wall distances made once
        self.wallDistBound = int(template["wallDistBound"]) if "wallDistBound" in template else 10
        if not 0 <= self.wallDistBound <= 254:
            raise ValueError("wallDistBound must lie in [0, 254]")
        self.walls = self.wall_dist = None
        if getattr(itf, "walls", None) is not None:
            self.walls = itf.walls  # uint8 device tensor, grid layout
            self.wall_dist = torch.empty(self.size_tot, dtype=torch.uint8, device="cuda")
            tmp = torch.empty(2 * int(np.prod(self.shape)), dtype=torch.uint8, device="cuda")
            _lib.check(_lib.lib().agd_prep_walls(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self.walls),
                                                 self.wallDistBound, _lib.ptr(self.wall_dist), _lib.ptr(tmp), None,
                                                 None, _lib.stream_ptr()), "walls")
            torch.cuda.current_stream().synchronize()
        self._bufs = [_Buffers(self) for _ in range(self.nbuffers)]
        self._next = 0
        self.submitted = 0

    # ------------------------------------------------------------------ input --
    def _stage(self, buf, name, x, shape, dtype=torch.float32):
        """Device tensor holding x (batch-leading array), in place when already on the device."""
        if not isinstance(x, torch.Tensor):
            x = torch.from_numpy(np.ascontiguousarray(np.asarray(x), dtype=np.float32 if dtype == torch.float32
                                                      else np.int32))
        if tuple(x.shape) != tuple(shape):
            raise ValueError(f"{name} has shape {tuple(x.shape)}, expected {tuple(shape)}")
        if x.is_cuda:
            return x.to(dtype).contiguous()
        d = buf.staging(name, shape, dtype)
        d.copy_(x.to(dtype), non_blocking=x.is_pinned())
        return d

    def _atol(self, cost):
        if self.fixed_atol is not None:
            return np.full(self.batch, self.fixed_atol, np.float32)
        if cost is None:
            return np.full(self.batch, np.float32(1.0 * _FLOAT_RES * 5.0), np.float32)
        c = cost if isinstance(cost, torch.Tensor) else torch.from_numpy(np.asarray(cost, np.float32))
        mean = torch.nanmean(c.reshape(self.batch, -1).float(), dim=1).cpu().numpy().astype(np.float64)
        return (mean * _FLOAT_RES * 5.0).astype(np.float32)

    def _plan(self, buf, atol, gated=False, walls=None):
        """The plan of the buffer set; walls: None, "shared" (the template's) or
        "batch" (per-instance wall distances in buf.wall_dist)."""
        key = (atol.tobytes(), gated, walls)
        if buf.plan is not None and buf.plan_key == key:
            return
        L = _lib.lib()
        arr = (_lib.AgdInstance * self.batch)()
        for i in range(self.batch):
            inst = arr[i]
            inst.model = self.model_code
            inst.ndim = self.ndim
            for k in range(3):
                inst.shape[k] = self.c_shape[k]
                inst.shape_i[k] = self.c_shape_i[k]
                inst.iso_weights[k] = float(self.h[k]) ** -2 if k < self.ndim else 0.0
            inst.niter_i, inst.fim_front_width, inst.nitermax_o = self.niter_i, self.fim_front_width, self.nitermax_o
            inst.flags = self.flags
            inst.atol, inst.rtol = float(atol[i]), float(self.rtol)
            inst.values = buf.values[i].data_ptr()
            inst.geom = buf.geom[i].data_ptr() if self.nmet else None
            inst.rhs = buf.rhs[i].data_ptr()
            inst.seedbits = buf.seedbits[i].data_ptr()
            if gated:
                inst.release = buf.release[i].data_ptr()
            if walls is not None:
                inst.wall_dist = (self.wall_dist if walls == "shared" else buf.wall_dist[i]).data_ptr()
                inst.trigger = buf.trigger[i].data_ptr()
        plan = ctypes.c_void_p()
        _lib.check(L.agd_plan_create(arr, self.batch, ctypes.byref(plan)), "plan")
        if buf.plan is not None:
            L.agd_plan_destroy(buf.plan)
        buf.plan = plan
        buf.plan_key = key
        nbytes = int(L.agd_plan_workspace_bytes(plan))
        if buf.ws is None or buf.ws.numel() < nbytes:
            with torch.cuda.stream(buf.stream):
                buf.ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        _lib.check(L.agd_plan_upload(plan, _lib.ptr(buf.ws), nbytes, _lib.stream_ptr(buf.stream)), "upload")

    def _seed_index(self, buf, seeds):
        """(batch, nseeds, ndim) grid indices of the seed points, rounded as the
        reference does (PointFromIndex(., to=True), then np.round)."""
        if isinstance(seeds, torch.Tensor) and seeds.is_cuda:
            if seeds.dim() != 3 or seeds.shape[0] != self.batch or seeds.shape[2] != self.ndim:
                raise ValueError(f"seeds must have shape (batch, nseeds, {self.ndim})")
            if getattr(self, "_start_h", None) is None:  # made once: a copy from host memory blocks the host
                self._start_h = (torch.as_tensor(self.start, device="cuda"), torch.as_tensor(self.h, device="cuda"))
            start, h = self._start_h
            return torch.round((seeds.float() - start) / h).to(torch.int32).contiguous()  # checked on the device
        s = seeds.numpy() if isinstance(seeds, torch.Tensor) else np.asarray(seeds, np.float32)
        s = s.astype(np.float32, copy=False)
        if s.ndim != 3 or s.shape[0] != self.batch or s.shape[2] != self.ndim:
            raise ValueError(f"seeds must have shape (batch, nseeds, {self.ndim})")
        idx = np.round((s - self.start) / self.h).astype(np.int32)
        inside = np.all((idx >= 0) & (idx < np.array(self.shape)), axis=2)
        if not np.all(inside):
            raise ValueError(f"Seeds outside the domain: {s[~inside].tolist()}")
        host = torch.from_numpy(idx).pin_memory()
        d = buf.staging("seed_index", idx.shape, torch.int32)
        d.copy_(host, non_blocking=True)
        return d

    # ----------------------------------------------------------------- submit --
    def submit(self, metric=None, cost=None, seeds=None, seedValues=None, out=None, release=None, values=None,
               walls=None, fresh_out=False):
        """Queues one batch; returns a SolverJob.  out: optional host tensor
        (batch, *shape) float32 (page-locked for an asynchronous copy).
        walls: optional (batch, *shape) obstacle masks of the instances, in
        place of the template's (whose wall distances are made once).
        fresh_out: the values go to a device tensor of this submission's own
        (written by the reordering kernel right behind the solve), which stays
        valid when the buffer set is reused: no copy is needed afterwards,
        which would have to wait for the SMs behind the next batch's solve.
        release: optional device tensor (batch, tiles) of int16/uint16 tile
        release epochs (agd_instance.release; the learned schedule); values:
        optional device tensor (batch, tiles * tile size) of initial values in
        tile layout (a warm start: upper bounds of the solution, since values
        only decrease), instead of +inf."""
        if seeds is None:
            raise ValueError("Missing value for key seeds")
        if self.nmet and metric is None:
            raise ValueError("Missing value for key metric")
        if not self.nmet and cost is None:
            raise ValueError("Missing value for key cost")
        if not self.nmet and metric is not None:
            raise ValueError("Isotropic models take a cost, not a metric")
        if out is not None and (tuple(out.shape) != (self.batch,) + self.shape or out.dtype != torch.float32):
            raise ValueError(f"out must be a float32 tensor of shape {(self.batch,) + self.shape}")
        buf = self._bufs[self._next]
        self._next = (self._next + 1) % self.nbuffers
        if buf.job is not None:
            buf.job.event.synchronize()  # the previous batch of this buffer set is complete
        atol = self._atol(cost)
        user_stream = torch.cuda.current_stream()
        L = _lib.lib()
        with torch.cuda.stream(buf.stream):
            buf.stream.wait_stream(user_stream)  # device inputs made on the caller's stream
            ntiles = self.ntiles
            if release is not None:
                if tuple(release.shape) != (self.batch, ntiles) or release.dtype not in (torch.int16, torch.uint16):
                    raise ValueError(f"release must be a 16-bit tensor of shape {(self.batch, ntiles)}")
                if buf.release is None:
                    buf.release = torch.empty((self.batch, ntiles), dtype=torch.int16, device="cuda")
                buf.release.copy_(release.view(torch.int16))
            wmode, wmask = None, None
            if walls is not None:
                wmask = self._stage(buf, "walls_mask", walls if isinstance(walls, torch.Tensor)
                                    else np.asarray(walls, np.uint8), (self.batch,) + self.shape, torch.uint8)
                if buf.wall_dist is None:
                    buf.wall_dist = torch.empty((self.batch, self.size_tot), dtype=torch.uint8, device="cuda")
                    buf.walls_tmp = torch.empty(2 * self.batch * int(np.prod(self.shape)), dtype=torch.uint8,
                                                device="cuda")
                _lib.check(L.agd_prep_walls_batch(self.ndim, self.c_shape, self.c_shape_i, self.batch,
                                                  _lib.ptr(wmask), self.wallDistBound, _lib.ptr(buf.wall_dist),
                                                  _lib.ptr(buf.walls_tmp), _lib.stream_ptr(buf.stream)), "walls")
                wmode = "batch"
            elif self.walls is not None:
                wmode, wmask = "shared", self.walls
            if wmode is not None and buf.trigger is None:
                buf.trigger = torch.empty((self.batch, ntiles), dtype=torch.uint8, device="cuda")
            self._plan(buf, atol, gated=release is not None, walls=wmode)
            prep = _lib.AgdBatchPrep()
            prep.model = self.model_code
            prep.ndim, prep.n = self.ndim, self.batch
            for k in range(3):
                prep.shape[k], prep.shape_i[k] = self.c_shape[k], self.c_shape_i[k]
                prep.grid_scales[k] = float(self.h[k]) if k < self.ndim else 1.0
            keep = []
            if self.nmet:
                m = self._stage(buf, "metric", metric, (self.batch,) + self.shape + (self.nmet,))
                keep.append(m)
                prep.metric, prep.geom = m.data_ptr(), buf.geom.data_ptr()
            if wmode is not None:
                keep.append(wmask)
                prep.walls, prep.walls_shared = wmask.data_ptr(), int(wmode == "shared")
                prep.trigger = buf.trigger.data_ptr()
            if cost is not None:
                c = self._stage(buf, "cost", cost, (self.batch,) + self.shape)
                keep.append(c)
                prep.cost = c.data_ptr()
            idx = self._seed_index(buf, seeds)
            keep.append(idx)
            prep.seed_index, prep.nseeds = idx.data_ptr(), int(idx.shape[1])
            if seedValues is not None:
                v = self._stage(buf, "seed_values", seedValues, (self.batch, int(idx.shape[1])))
                keep.append(v)
                prep.seed_values = v.data_ptr()
            buf.bad.zero_()
            prep.rhs, prep.values = buf.rhs.data_ptr(), buf.values.data_ptr()
            prep.seedbits, prep.bad_seed = buf.seedbits.data_ptr(), buf.bad.data_ptr()
            st = _lib.stream_ptr(buf.stream)
            _lib.check(L.agd_prep_batch(ctypes.byref(prep), st), "prep_batch")
            if values is not None:
                if tuple(values.shape) != (self.batch, self.size_tot) or not values.is_cuda:
                    raise ValueError(f"values must be a device tensor of shape {(self.batch, self.size_tot)}")
                buf.values.copy_(values)
            lp = ctypes.byref(self.launch) if self.launch is not None else None
            _lib.check(L.agd_plan_run(buf.plan, _lib.ptr(buf.ws), buf.ws.numel(), _lib.ptr(buf.stats), lp, st),
                       "solve")
            dev_out = torch.empty_like(buf.out) if fresh_out and out is None else None
            target = dev_out if dev_out is not None else buf.out
            _lib.check(L.agd_block_squeeze(self.ndim, self.c_shape, self.c_shape_i, self.batch, _lib.ptr(buf.values),
                                           _lib.ptr(target), st), "block_squeeze")
            buf.stats_host.copy_(buf.stats, non_blocking=True)
            buf.bad_host.copy_(buf.bad, non_blocking=True)
            if out is not None:
                out.copy_(buf.out, non_blocking=True)
            for t in keep:  # inputs read in place on this stream stay alive until it gets past them
                if t.is_cuda:
                    t.record_stream(buf.stream)
            job = SolverJob(self, buf, out, dev_out)
        buf.job = job
        self.submitted += 1
        return job

    def solve(self, **kwargs):
        """submit(**kwargs).result()."""
        return self.submit(**kwargs).result()

    def __del__(self):
        try:
            L = _lib.lib()
            for b in self._bufs:
                if b.plan is not None:
                    b.stream.synchronize()
                    L.agd_plan_destroy(b.plan)
                    b.plan = None
        except Exception:  # noqa: BLE001
            pass
