"""GPU eikonal solver behind dictIn.Run() (the reference's HFM_CUDA package).

`RunGPU(hfmIn)` mirrors agd/Eikonal/HFM_CUDA/__init__.py:10-25 and the
Interface class of _Interface.py:23-174: every key is read through GetValue,
which records help texts, defaults, used and unused keys in
hfmOut['keys']; the same keys, defaults and errors as the reference are used
for the Isotropic2/3, Diagonal2/3, Riemann2/3 and Rander2/3 models.  The work is done by
libagd_b200.so through the C ABI of include/agd_b200.h:
  SetGeometry/SetArgs  -> agd_prep_geom(_diagonal), agd_block_expand, agd_prep_seeds,
                          agd_prep_walls
  Solve (FIM)          -> agd_plan_create / agd_plan_upload / agd_plan_run
  PostProcess (flow)   -> agd_flow
  GetGeodesics         -> agd_eucl_map, agd_geodesics
  SolveAD (reverse)    -> agd_reverse
"""
import ctypes
import math
import numbers
import warnings
from collections import OrderedDict

import numpy as np
import torch

from .. import _lib
from .. import Metrics

# Default traits (agd/Eikonal/HFM_CUDA/kernel_traits.py:61-88): shape_i, niter_i, fim_front_width.
DEFAULT_TRAITS = {
    "Riemann2": ((8, 8), 8, 4),
    "Riemann3": ((4, 4, 4), 4, 6),
    "Isotropic2": ((16, 16), 16, 4),
    "Isotropic3": ((4, 4, 4), 8, 4),
    "Diagonal2": ((16, 16), 16, 4),
    "Diagonal3": ((4, 4, 4), 8, 4),
    "Rander2": ((8, 8), 12, 8),
    "Rander3": ((4, 4, 4), 8, 8),
}
SUPPORTED_TILES = {2: {(8, 8), (16, 16)}, 3: {(4, 4, 4)}}
GEODESIC_CODES = ["Continue", "AtSeed", "InWall", "Stationnary", "PastSeed", "VanishingFlow"]
_FLOAT_RES = float(np.finfo(np.float32).resolution)


def RunGPU(hfmIn, *args, cache=None, **kwargs):
    """Runs the GPU eikonal solver.

    Main input: hfmIn, a dictIn.  Set hfmIn['verbosity'] to 1 or 2 to display
    information on the run (0 to silence it); hfmOut['keys']['help'] holds a
    short help for every key that was looked up."""
    if cache is not None:
        print("Warning : gpu eikonal solver does not support caching")
    return Interface(hfmIn).Run(*args, **kwargs)


def RunBatch(hfmIns, launch=None):
    """Solves several dictIn in one persistent launch (all of the same dimension).

    Each instance keeps its own model, tile shape, tolerances and options; the
    per-instance post-processing (flow, geodesics, sensitivities, outputs) is the
    same as RunGPU's.  Returns the list of outputs."""
    return SubmitBatch(hfmIns, launch=launch).result()


def SubmitBatch(hfmIns, launch=None):
    """Queues the preparation and the solve of several dictIn on the current
    CUDA stream and returns a BatchJob without waiting for the device.

    The host can meanwhile prepare the next batch: submitted on a second
    stream, its uploads and preparation kernels queue while this solve runs.
    `BatchJob.result()` gives what RunBatch returns.

    A batch of dictIn that differ only in their data (same model, grid, traits
    and options; metric or cost arrays of one shape, the same number of seeds)
    is prepared by one batched kernel (agd_prep_batch, as Eikonal.BatchSolver
    does) instead of instance by instance."""
    fast = _submit_uniform(hfmIns, launch)
    if fast is not None:
        return fast
    itfs = [Interface(h) for h in hfmIns]
    for it in itfs:
        it.SetKernelTraits()
        it.SetGeometry()
        it.SetArgs()
    plan = BatchPlan(itfs, launch=launch)
    plan.run()
    return BatchJob(plan)


# Keys that the batched preparation takes (anything else: instance by instance).
_UNIFORM_KEYS = {"model", "mode", "arrayOrdering", "verbosity", "dims", "gridScale", "gridScales", "origin",
                 "metric", "cost", "seeds", "seedValues", "exportValues", "tol", "atol", "rtol", "traits",
                 "nitermax_o", "fim_front_width", "raiseOnNonConvergence", "solver", "projective", "walls",
                 "wallDistBound"}
_UNIFORM_DATA = {"metric", "cost", "seeds", "seedValues"}
_uniform_solvers = OrderedDict()  # configuration -> (BatchSolver, key bookkeeping of one instance)


def _option(h, k):
    """A comparable host form of an option of a dictIn: small arrays from the
    host copy the dictIn keeps (no device read), None for large device arrays."""
    v = h.raw(k)
    if isinstance(v, (np.ndarray, torch.Tensor)):
        a = h.host(k) if not (isinstance(v, torch.Tensor) and v.is_cuda and v.numel() > 64) else None
        if a is None:
            return None
        a = np.ascontiguousarray(a)
        return ("array", a.shape, a.dtype.str, a.tobytes())
    if isinstance(v, dict):
        return ("dict", repr(sorted((kk, repr(vv)) for kk, vv in v.items())))
    if isinstance(v, (list, tuple)):
        return ("seq", repr(list(v)))
    return ("value", repr(v))


_SCALARS = (bool, int, float, str, type(None))


def _eq(x, y):
    """x == y for scalars of one type, with repr's float identity: -0.0 is
    not 0.0, and NaN is NaN."""
    if type(x) is float:
        return (x == y and math.copysign(1.0, x) == math.copysign(1.0, y)) or (x != x and y != y)
    return x == y


def _same_option(a, b):
    """True or False when a and b (raw option values of two dictIn) are
    scalars, lists/tuples of scalars of the same types element by element, or
    small numpy arrays: their equality, as _option's comparison would give it
    without building its host forms; None for anything else (compare by
    _option)."""
    if a is b:
        return True
    ta = type(a)
    if ta in _SCALARS:
        return ta is type(b) and _eq(a, b)
    if ta is np.ndarray:  # small host arrays (dims, gridScale, origin after SetRect): their bytes
        if type(b) is not np.ndarray or a.size > 64:
            return None
        return a.shape == b.shape and a.dtype.str == b.dtype.str and a.tobytes() == b.tobytes()
    if ta in (list, tuple) and type(b) is ta and len(a) == len(b):
        for x, y in zip(a, b):
            tx = type(x)
            if tx not in _SCALARS or tx is not type(y):
                return None
            if not _eq(x, y):
                return False
        return True
    return None


def _submit_uniform(hfmIns, launch):
    """The batched preparation path of SubmitBatch, or None when the dictIn do
    not qualify."""
    from .BatchSolver import BatchSolver
    B = len(hfmIns)
    if B < 2:
        return None
    h0 = hfmIns[0]
    model = h0.get("model")
    if model not in ("Riemann2", "Riemann3", "Isotropic2", "Isotropic3", "Diagonal2", "Diagonal3", "Rander2",
                     "Rander3"):
        return None
    keys0 = set(h0.keys())
    data = "cost" if model.startswith("Isotropic") else "metric"
    if not keys0 <= _UNIFORM_KEYS or data not in keys0 or "seeds" not in keys0:
        return None
    opts = sorted(keys0 - _UNIFORM_DATA - {"verbosity"})
    arrays = [k for k in ("metric", "cost", "seeds", "seedValues") if k in keys0]
    for k in arrays:
        if not isinstance(h0.raw(k), (np.ndarray, torch.Tensor)):
            return None
    shapes = {k: tuple(h0.raw(k).shape) for k in arrays}
    opt0 = tuple(_option(h0, k) for k in opts)
    if any(o is None for o in opt0):
        return None
    raw0 = [h0.raw(k) for k in opts]
    for h in hfmIns[1:]:
        if set(h.keys()) != keys0:
            return None
        for k, r0, o0 in zip(opts, raw0, opt0):
            same = _same_option(h.raw(k), r0)
            if same is None:
                same = _option(h, k) == o0
            if not same:
                return None
        for k in arrays:
            x = h.raw(k)
            if not isinstance(x, (np.ndarray, torch.Tensor)) or tuple(x.shape) != shapes[k]:
                return None
    cfg = (model, tuple(h0.shape), B, id(launch), tuple(zip(opts, opt0)), tuple(sorted(shapes.items())))
    entry = _uniform_solvers.get(cfg)
    if entry is None:
        solver = BatchSolver(h0, B, launch=launch)
        # the key bookkeeping of one instance, as RunGPU records it
        itf = Interface(h0)
        itf.SetKernelTraits()
        itf.SetGeometry()
        itf.SetArgs()
        itf.PostProcess()
        itf.SolveAD()
        itf.GetGeodesics()
        itf.FinalCheck()
        if itf.extractValues or itf.retself or itf.flow_needed:
            return None
        keys = itf.hfmOut["keys"]
        entry = (solver, keys, bool(h0.get("exportValues", False)))
        _uniform_solvers[cfg] = entry
        while len(_uniform_solvers) > 2:
            _uniform_solvers.popitem(last=False)
    else:
        _uniform_solvers.move_to_end(cfg)
    solver, keys, export = entry
    user = torch.cuda.current_stream()
    buf = solver._bufs[solver._next]
    if buf.job is not None:
        buf.job.event.synchronize()
    inputs = {}
    with torch.cuda.stream(buf.stream):
        buf.stream.wait_stream(user)
        for k in arrays:
            dev = buf.staging("u_" + k, (B,) + shapes[k], torch.float32)
            xs = [h.raw(k) for h in hfmIns]
            if all(isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32 for x in xs):
                torch.stack(xs, out=dev)  # one gather on the device
            elif all(isinstance(x, np.ndarray) for x in xs) and sum(x.size for x in xs) <= 1 << 20:
                # small host arrays (seeds, seed values): one page-locked upload
                dev.copy_(torch.from_numpy(np.stack(xs).astype(np.float32, copy=False)).pin_memory(), non_blocking=True)
            else:
                for i, x in enumerate(xs):
                    x = torch.from_numpy(np.asarray(x, np.float32)) if isinstance(x, np.ndarray) else x
                    dev[i].copy_(x, non_blocking=x.device.type == "cpu" and x.is_pinned() or x.is_cuda)
            inputs[k] = dev
    job = solver.submit(metric=inputs.get("metric"), cost=inputs.get("cost"), seeds=inputs["seeds"],
                        seedValues=inputs.get("seedValues"), fresh_out=export)
    return UniformBatchJob(job, keys, export, B)


class UniformBatchJob:
    """A batch of SubmitBatch prepared in one go; `result()` gives the list of
    outputs (values, stats and key bookkeeping per instance)."""

    def __init__(self, job, keys, export, n):
        self.job, self.keys, self.export, self.n = job, keys, export, n
        self.stream = job.stream
        self._outs = None

    def done(self):
        return self.job.done()

    def result(self):
        if self._outs is not None:
            return self._outs
        values = self.job.result()  # the submission's own tensor when exported (fresh_out)
        if not self.export:
            values = None
        outs = []
        for i in range(self.n):
            keys = {k: (list(v) if isinstance(v, list) else OrderedDict(v) if isinstance(v, dict) else v)
                    for k, v in self.keys.items()}
            stats = {"eikonal": {"niter_o": int(self.job.niter_o[i]), "time": None,
                                 "nupdate_o_total": int(self.job.tile_visits[i])},
                     "flow": {}, "geodesic": {}, "forwardAD": {}, "reverseAD": {}}
            out = {"keys": keys, "stats": stats, "solverGPUTime": None}
            if values is not None:
                out["values"] = values[i]
            outs.append(out)
        self._outs = outs
        return outs


class BatchJob:
    """A submitted batch.  The solver statistics come back to page-locked host
    memory and the solution values are rearranged into grid order on the
    submission stream right behind the solve, so that `result()` only waits
    for this batch even when later work is queued on other streams."""

    def __init__(self, plan):
        self.plan = plan
        self.stream = torch.cuda.current_stream()
        for it in plan.itfs:
            if it.hfmIn.get("exportValues", False) or it.hfmIn.get("extractValues", False):
                it.values  # noqa: B018  (queues the squeeze; the tensor is cached)
        self.stats_host = torch.empty(tuple(plan.stats.shape), dtype=plan.stats.dtype).pin_memory()
        self.stats_host.copy_(plan.stats, non_blocking=True)
        self.event = torch.cuda.Event()
        self.event.record(self.stream)
        self._outs = None

    def done(self):
        """True once the device has finished the solve (does not block)."""
        return self.event.query()

    def result(self):
        """Waits for the solve, checks its status and returns the outputs (a list,
        in submission order); post-processing runs on the submission stream."""
        if self._outs is not None:
            return self._outs
        self.event.synchronize()
        with torch.cuda.stream(self.stream):
            self.plan.finish(self.stats_host.numpy())
            outs = []
            for it in self.plan.itfs:
                it.PostProcess()
                it.SolveAD()
                it.GetGeodesics()
                it.FinalCheck()
                if it.extractValues or it.retself:
                    r = [it.hfmOut]
                    if it.extractValues:
                        r.insert(0, it.values)
                    if it.retself:
                        r.append(it)
                    outs.append(r)
                else:
                    outs.append(it.hfmOut)
        self._outs = outs
        return outs


class BatchPlan:
    """A plan over prepared Interfaces: device workspace, descriptors uploaded
    once, and `run()` that only enqueues device work (graph capturable)."""

    def __init__(self, itfs, launch=None):
        L = _lib.lib()
        self.itfs = itfs
        self.n = len(itfs)
        arr = (_lib.AgdInstance * self.n)(*[it.instance() for it in itfs])
        self._arr = arr
        self.plan = ctypes.c_void_p()
        _lib.check(L.agd_plan_create(arr, self.n, ctypes.byref(self.plan)), "plan")
        self.nbytes = int(L.agd_plan_workspace_bytes(self.plan))
        self.ws = torch.empty(self.nbytes, dtype=torch.uint8, device="cuda")
        self.stats = torch.zeros((self.n, 2), dtype=torch.int64, device="cuda")
        self.launch = launch
        _lib.check(L.agd_plan_upload(self.plan, _lib.ptr(self.ws), self.nbytes, _lib.stream_ptr()), "upload")
        self.grid_updates_per_visit = [it.size_i for it in itfs]

    def run(self, stream=None):
        L = _lib.lib()
        lp = ctypes.byref(self.launch) if self.launch is not None else None
        _lib.check(L.agd_plan_run(self.plan, _lib.ptr(self.ws), self.nbytes, _lib.ptr(self.stats), lp,
                                  _lib.stream_ptr(stream)), "solve")

    def read_stats(self, s=None):
        """(niter_o, status, tile_visits) per instance, from the device statistics
        or from a host copy of them."""
        if s is None:
            s = self.stats.cpu().numpy()
        return (s[:, 0] & 0xffffffff).astype(np.int64), ((s[:, 0] >> 32) & 0xffffffff).astype(np.int64), s[:, 1]

    def finish(self, stats_host=None):
        niter, status, visits = self.read_stats(stats_host)
        for i, it in enumerate(self.itfs):
            it.tile_visits = int(visits[i])
            it.stats["eikonal"].update({"niter_o": int(niter[i]), "time": None, "nupdate_o_total": int(visits[i]),
                                        "grid_updates": int(visits[i]) * it.size_i})
            st = int(status[i])
            if st & ~_lib.AGD_STATUS_NOT_CONVERGED:
                raise _lib.AgdError(st, f"eikonal solve failed on the device (instance {i})")
            if st & _lib.AGD_STATUS_NOT_CONVERGED:
                msg = f"Instance {i} did not reach convergence after {it.nitermax_o} iterations"
                if it.raiseOnNonConvergence:
                    raise ValueError(msg)
                it.Warn(msg)

    def __del__(self):
        try:
            _lib.lib().agd_plan_destroy(self.plan)
        except Exception:  # noqa: BLE001
            pass


def _to_tensor(x, dtype=torch.float32):
    if isinstance(x, torch.Tensor):
        # a copy from page-locked host memory is queued without waiting for it
        return x.to(device="cuda", dtype=dtype, non_blocking=x.is_pinned())
    return torch.as_tensor(np.asarray(x, dtype=np.float32 if dtype == torch.float32 else None), device="cuda",
                           dtype=dtype)


class Interface:
    """Carries out the work of RunGPU (agd/Eikonal/HFM_CUDA/_Interface.py:23-174)."""

    def __init__(self, hfmIn):
        self.hfmIn = hfmIn
        if hfmIn["arrayOrdering"] != "RowMajor":
            raise ValueError("Only RowMajor indexing supported")
        self.hfmOut = {"keys": {
            "used": ["origin", "arrayOrdering", "dims", "mode", "projective"],
            "default": OrderedDict(),
            "visited": [],
            "help": OrderedDict(),
            "kernelStats": OrderedDict(),
        }}
        self.verbosity = 1
        self.verbosity = self.GetValue("verbosity", default=1,
                                       help="Choose the amount of detail displayed on the run")
        self.clear_hfmIn = self.GetValue("clear_hfmIn", default=False,
                                         help="Delete hfmIn member fields. (May save memory.)")
        self.model = self.GetValue("model", help="Minimal path model to be solved.")
        if self.model not in DEFAULT_TRAITS:
            raise ValueError(f"Unsupported model {self.model!r}; supported: {sorted(DEFAULT_TRAITS)}")
        self.ndim = len(np.asarray(hfmIn.host("dims")).reshape(-1))
        if self.ndim != int(self.model[-1]):
            raise ValueError(f"Model {self.model} expects {self.model[-1]} dimensions, got dims of length {self.ndim}")
        self.stats = {"eikonal": {}, "flow": {}, "geodesic": {}, "forwardAD": {}, "reverseAD": {}}

    @property
    def model_(self):
        return self.model[:-1]

    # ------------------------------------------------------------- keys ---
    def HasValue(self, key):
        self.hfmOut["keys"]["visited"].append(key)
        return key in self.hfmIn

    def GetValue(self, key, default="_None", verbosity=2, array_float=False, help="Sorry : no help for this key"):
        """Value of a key, with the reference's bookkeeping (_Interface.py:80-122)."""
        assert key not in self.hfmOut["keys"]["help"]
        self.hfmOut["keys"]["help"][key] = help
        self.hfmOut["keys"]["default"][key] = default
        if key in self.hfmIn:
            self.hfmOut["keys"]["used"].append(key)
            value = self.hfmIn[key]
            if array_float is False:
                return value
            value = _to_tensor(value)
            if isinstance(array_float, tuple):
                shapeRef, shape = array_float, tuple(value.shape)
                if len(shapeRef) != len(shape):
                    raise ValueError(f"Field {key} has incorrect number of dimensions. "
                                     f"Expected shape {shapeRef}, found {shape}")
                for sRef, s in zip(shapeRef, shape):
                    if sRef not in (-1, s):
                        raise ValueError(f"Field {key} has incorrect dimensions. "
                                         f"Expected shape {shapeRef}, found {shape}")
            return value
        elif isinstance(default, str) and default == "_None":
            raise ValueError(f"Missing value for key {key}")
        else:
            if verbosity <= self.verbosity:
                if isinstance(default, str) and default == "_Dummy":
                    print(f"see out['keys']['default'][{key}] for default")
                else:
                    print(f"key {key} defaults to {default}")
            if isinstance(default, numbers.Number) and array_float is not False:
                default = _to_tensor(default)
            return default

    def Warn(self, msg):
        if self.verbosity >= -1:
            print("---- Warning ----\n", msg, "\n-----------------\n")

    # -------------------------------------------------------------- run ---
    def Run(self):
        self.SetKernelTraits()
        self.SetGeometry()
        self.SetArgs()
        self.Solve()
        self.PostProcess()
        self.SolveAD()
        self.GetGeodesics()
        self.FinalCheck()
        if self.extractValues or self.retself:
            retval = [self.hfmOut]
            if self.extractValues:
                retval.insert(0, self.values)
            if self.retself:
                retval.append(self)
            return retval
        return self.hfmOut

    def SetKernelTraits(self):
        """Traits (agd/Eikonal/HFM_CUDA/_Kernel.py:23-92)."""
        si, niter, front = DEFAULT_TRAITS[self.model]
        traits = {"shape_i": si, "niter_i": niter}
        given = self.GetValue("traits", default=dict(traits),
                              help="Optional trait parameters for the eikonal kernel "
                                   "('auto': tile shape and niter_i chosen by timed trial solves, cached)")
        if isinstance(given, str):
            if given != "auto":
                raise ValueError(f"traits must be a dict or 'auto', got {given!r}")
            traits.update(self._autotune())
        else:
            traits.update(given)
        self.shape_i = tuple(int(s) for s in traits["shape_i"])
        self.niter_i = int(traits["niter_i"])
        if self.shape_i not in SUPPORTED_TILES[self.ndim]:
            raise ValueError(f"Unsupported shape_i {self.shape_i} for {self.model}; "
                             f"built tile shapes: {sorted(SUPPORTED_TILES[self.ndim])}")
        self.traits = traits
        self.values_float64 = self.GetValue("values_float64", default=False,
                                            help="Export values using the float64 data type")
        self.multiprecision = self.values_float64 or self.GetValue(
            "multiprecision", default=False, help="Use multiprecision arithmetic, to improve accuracy")
        self.factoringRadius = float(self.GetValue("factoringRadius", default=0,
                                                   help="Use source factorization, to improve accuracy"))
        order = self.GetValue("order", default=1, help="Use second order scheme to improve accuracy")
        if order not in {1, 2}:
            raise ValueError(f"Unsupported scheme order {order}")
        self.order = int(order)
        self.order2_threshold = 0.0
        if order == 2:
            self.order2_threshold = float(self.GetValue(  # _Kernel.py:310-314
                "order2_threshold", 0.3,
                help="Relative threshold on second order differences / first order difference,"
                     "beyond which the second order scheme deactivates"))
        solver = self.GetValue("solver", default="FIM",
                               help="Choice of fixed point solver (AGSI, global_iteration)")
        alt = {"FIM": "fast_iterative_method", "AGSI": "adaptive_gauss_siedel_iteration"}
        self.solver = alt.get(solver, solver)
        if self.solver not in ("fast_iterative_method", "adaptive_gauss_siedel_iteration", "global_iteration"):
            raise ValueError(f"Unrecognized solver : {self.solver}")
        self.fim_front_width = int(self.GetValue(
            "fim_front_width", default=front,
            help="Dictates the max front width in the FIM variant.\n(original FIM : 2. Must be >=2.)"))
        if not 2 <= self.fim_front_width <= 255:
            raise ValueError("fim_front_width must be an integer in [2, 255]")
        self.nitermax_o = int(self.GetValue("nitermax_o", default=2000,
                                            help="Maximum number of iterations of the solver"))
        self.raiseOnNonConvergence = self.GetValue("raiseOnNonConvergence", default=True,
                                                   help="Raise an exception if a solver fails to converge")
        self.size_i = int(np.prod(self.shape_i))

    def _autotune(self):
        """Traits of traits='auto': the cached choice for this model and grid size
        on this device, else the fastest of the candidates of Autotune.py in
        trial solves of this very problem (solve time by CUDA events)."""
        from .Autotune import Autotuner, bucket_key, candidates
        key = bucket_key(self.model, self.hfmIn.shape, 1, torch.cuda.get_device_name())

        def run(tr):
            h = self.hfmIn.copy()
            h["traits"], h["verbosity"] = dict(tr), 0
            for k in ("tips", "sensitivity", "costVariation", "seedValueVariation", "exportGeodesicFlow",
                      "exportActiveNeighs"):
                h.store.pop(k, None)
            it = Interface(h)
            try:
                it.SetKernelTraits()
                it.SetGeometry()
                it.SetArgs()
                it.Solve()
            except (ValueError, _lib.AgdError):
                return float("inf")
            return it.stats["eikonal"]["time"]

        choice, trials = Autotuner().choose(key, run, candidates(self.model))
        self.stats["autotune"] = {"key": key, "traits": {k: list(v) if isinstance(v, tuple) else v
                                                        for k, v in choice.items()},
                                  "cached": trials is None}
        return choice

    def SetGeometry(self):
        """Domain, metric and cost (agd/Eikonal/HFM_CUDA/_SetGeometry.py:16-282)."""
        L = _lib.lib()
        self.shape = self.hfmIn.shape
        if any(s <= 0 for s in self.shape):
            raise ValueError(f"Invalid domain shape {self.shape}")
        self.shape_o = tuple((s + i - 1) // i for s, i in zip(self.shape, self.shape_i))
        self.size_o = int(np.prod(self.shape_o))
        self.size_tot = self.size_o * self.size_i
        if "gridScale" in self.hfmIn:
            self.GetValue("gridScale", help="Scale of the computational grid")
        else:
            self.GetValue("gridScales", array_float=(self.ndim,), help="Axis independent scales of the computational grid")
        self.h = np.asarray(self.hfmIn.gridScales, np.float32).reshape(-1)
        self.c_shape = (ctypes.c_int * 3)(*self.shape, *([1] * (3 - self.ndim)))
        self.c_shape_i = (ctypes.c_int * 3)(*self.shape_i, *([1] * (3 - self.ndim)))
        self.stream = _lib.stream_ptr()

        if self.model_ == "Riemann":
            metric = self.GetValue("metric", default=None, verbosity=3, help="Metric of the minimal path model")
            dual = self.GetValue("dualMetric", default=None, verbosity=3,
                                 help="Dual metric of the minimal path model")
            if metric is None and dual is None:
                raise ValueError("Missing value for key metric")
            src, is_dual = (metric, 0) if metric is not None else (dual, 1)
            self._metric_is_dual = bool(is_dual)
            flat = _metric_hfm(src, self.ndim)
            symdim = self.ndim * (self.ndim + 1) // 2
            bcast = 1 if flat.dim() == 1 else 0
            if not bcast and tuple(flat.shape[:-1]) != self.shape:
                raise ValueError("Inconsistent dimensions for geometry data. "
                                 "It should match (the last coordinates of) domain shape.")
            self._metric_flat = flat.contiguous()
            self.geom = torch.empty(symdim * self.size_tot, dtype=torch.float32, device="cuda")
            hs = (ctypes.c_double * 3)(*[float(x) for x in self.h], *([1.0] * (3 - self.ndim)))
            _lib.check(L.agd_prep_geom(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self._metric_flat), bcast,
                                       is_dual, hs, _lib.ptr(self.geom), self.stream), "prep_geom")
        elif self.model_ == "Rander":  # geom = metric.flatten(inverse_m=True) (_SetGeometry.py:138-139)
            metric = self.GetValue("metric", default=None, verbosity=3, help="Metric of the minimal path model")
            dual = self.GetValue("dualMetric", default=None, verbosity=3,
                                 help="Dual metric of the minimal path model")
            if metric is None and dual is None:
                raise ValueError("Missing value for key metric")
            src, is_dual = (metric, 0) if metric is not None else (dual, 1)
            self._metric_is_dual = bool(is_dual)
            flat = _rander_hfm(src, self.ndim)
            bcast = 1 if flat.dim() == 1 else 0
            if not bcast and tuple(flat.shape[:-1]) != self.shape:
                raise ValueError("Inconsistent dimensions for geometry data. "
                                 "It should match (the last coordinates of) domain shape.")
            self._metric_flat = flat.contiguous()
            symdim = self.ndim * (self.ndim + 1) // 2
            self.geom = torch.empty((symdim + self.ndim) * self.size_tot, dtype=torch.float32, device="cuda")
            hs = (ctypes.c_double * 3)(*[float(x) for x in self.h], *([1.0] * (3 - self.ndim)))
            _lib.check(L.agd_prep_geom_rander(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self._metric_flat),
                                              bcast, is_dual, hs, _lib.ptr(self.geom), self.stream),
                       "prep_geom_rander")
        elif self.model_ == "Diagonal":  # geom = dualMetric.costs**2 (_SetGeometry.py:134-135)
            metric = self.GetValue("metric", default=None, verbosity=3, help="Metric of the minimal path model")
            dual = self.GetValue("dualMetric", default=None, verbosity=3,
                                 help="Dual metric of the minimal path model")
            if metric is None and dual is None:
                raise ValueError("Missing value for key metric")
            src, is_dual = (metric, 0) if metric is not None else (dual, 1)
            self._metric_is_dual = bool(is_dual)
            costs = _costs_hfm(src, self.ndim)
            bcast = 1 if costs.dim() == 1 else 0
            if not bcast and tuple(costs.shape[:-1]) != self.shape:
                raise ValueError("Inconsistent dimensions for geometry data. "
                                 "It should match (the last coordinates of) domain shape.")
            self._metric_flat = costs.contiguous()
            self.geom = torch.empty(self.ndim * self.size_tot, dtype=torch.float32, device="cuda")
            hs = (ctypes.c_double * 3)(*[float(x) for x in self.h], *([1.0] * (3 - self.ndim)))
            _lib.check(L.agd_prep_geom_diagonal(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self._metric_flat),
                                                bcast, is_dual, hs, _lib.ptr(self.geom), self.stream),
                       "prep_geom_diagonal")
        else:
            self.geom = None

        self.exportGeodesicFlow = self.GetValue("exportGeodesicFlow", default=False,
                                                help="Export the upwind geodesic flow (direction of the geodesics)")
        self.tips = self.GetValue("tips", default=None, array_float=(-1, self.ndim),
                                  help="Tips from which to compute the minimal geodesics")
        self.hasTips = self.tips is not None

        mean_cost = None
        if self.HasValue("speed"):
            cost = 1.0 / self.GetValue("speed", array_float=True, help="speed = 1/cost (scales the metric, accepts AD)")
        else:
            cost = self.GetValue("cost", array_float=True, default=None,
                                 help="cost = 1/speed (scales the metric, accepts AD)")
            if cost is None:
                cost = torch.ones((), dtype=torch.float32, device="cuda")
                mean_cost = 1.0
        cost = cost.to(torch.float32)
        if cost.dim() != 0 and tuple(cost.shape) != self.shape:
            raise ValueError(f"Field cost has incorrect dimensions. Found {tuple(cost.shape)}, "
                             f"whereas domain has shape {self.shape}")
        self.cost = cost
        # forward AD (_SetGeometry.py:231-233): the cost's first order variations, (*shape, n)
        cv = self.GetValue("costVariation", default=None, help="First order variation of the cost function")
        if cv is not None:
            cv = _to_tensor(cv)
            if cv.dim() != self.ndim + 1 or tuple(cv.shape[:-1]) != self.shape:
                raise ValueError(f"costVariation has shape {tuple(cv.shape)}; expected {self.shape} + (n,)")
        self.costVariation = cv
        if self.HasValue("atol") and self.HasValue("rtol"):
            tol = None
        else:
            tol = self.GetValue("tol", default="_Dummy", array_float=tuple(),
                                help="Convergence tolerance for the fixed point solver (determines atol, rtol)")
            if isinstance(tol, str) and tol == "_Dummy":
                if mean_cost is None:
                    mean_cost = float(torch.nanmean(cost.float())) if cost.dim() else float(cost)
                tol = np.float32(mean_cost * _FLOAT_RES * 5.0)
                self.hfmOut["keys"]["default"]["tol"] = np.float32(tol)
            else:
                tol = float(tol)
        self.atol = float(self.GetValue("atol", default=tol, array_float=tuple(),
                                        help="Absolute convergence tolerance for the fixed point solver"))
        self.rtol = float(self.GetValue("rtol", default=0.0 if self.multiprecision else _FLOAT_RES * 5.0,
                                        array_float=tuple(),
                                        help="Relative convergence tolerance for the fixed point solver"))
        if self.multiprecision:
            # a power of two well below the grid scale (_SetGeometry.py:52-56)
            hmin = float(np.min(self.h))
            self.multip_step = float(2.0 ** np.floor(np.log2(hmin / 10)))
            self.multip_max = float(np.iinfo(np.int32).max * self.multip_step / 2)
        # obstacles (_SetGeometry.py:262-280): distance map by agd_prep_walls in SetArgs
        walls = self.GetValue("walls", default=None, help="Obstacles in the domain")
        self.walls = self.wall_dist = None
        if walls is not None:
            w = _to_tensor(walls, torch.bool)
            if tuple(w.shape) != self.shape:
                w = w.expand(self.shape)
            self.walls = w.to(torch.uint8).contiguous()
            self.wallDistBound = int(self.GetValue(
                "wallDistBound", default=10,
                help="Bound on the computed distance to the obstacles.\n"
                     "(Ideally a sharp upper bound on the stencil width.)"))
            if not 0 <= self.wallDistBound <= 254:
                raise ValueError("wallDistBound must lie in [0, 254]")
            self.wall_dist = torch.empty(self.size_tot, dtype=torch.uint8, device="cuda")

    def SetArgs(self):
        """Initial values, rhs, seeds (agd/Eikonal/HFM_CUDA/_SetArgs.py:8-177)."""
        L = _lib.lib()
        values = self.GetValue("values", default=None, array_float=self.shape,
                               help="Initial values for the eikonal solver")
        self.activateAll = bool(self.GetValue(
            "activateAll", default=False,
            help="Visit every tile at the first iteration (for warm starts from an upper bound of the "
                 "solution; by default only the tiles holding seeds are active at first)"))
        self.values_t = torch.empty(self.size_tot, dtype=torch.float32, device="cuda")
        if values is None:
            self.values_t.fill_(math.inf)
        else:
            v = values.contiguous().float()
            _lib.check(L.agd_block_expand(self.ndim, self.c_shape, self.c_shape_i, 1, _lib.ptr(v), 0,
                                          ctypes.c_float(math.inf), _lib.ptr(self.values_t), self.stream),
                       "values")
        self._values = None
        self.valuesq_t = self.values_next_t = self.valuesq_next_t = None
        if self.multiprecision:  # _SetArgs.py:168-177
            self.valuesq_t = torch.zeros(self.size_tot, dtype=torch.int32, device="cuda")
            self.values_next_t = torch.empty_like(self.values_t)
            self.valuesq_next_t = torch.empty_like(self.valuesq_t)
        self.rhs_t = torch.empty(self.size_tot, dtype=torch.float32, device="cuda")
        c = self.cost.contiguous()
        _lib.check(L.agd_block_expand(self.ndim, self.c_shape, self.c_shape_i, 1, _lib.ptr(c.reshape(-1)),
                                      1 if c.dim() == 0 else 0, ctypes.c_float(math.inf), _lib.ptr(self.rhs_t),
                                      self.stream), "rhs")
        seeds = self.GetValue("seeds", default=None, array_float=(-1, self.ndim),
                              help="Points from where the front propagation starts")
        self.reverseAD = self.HasValue("sensitivity")
        if seeds is None:
            raise ValueError("Missing value for key seeds (trigger-only fronts are not available in this build)")
        seedValues = self.GetValue("seedValues", default=torch.zeros(len(seeds), device="cuda"),
                                   array_float=(len(seeds),), help="Initial value for the front propagation")
        # (n, nseeds), as the reference (_SetArgs.py:30-33)
        sv = self.GetValue("seedValueVariation", default=None, array_float=(-1, len(seeds)),
                           help="First order variation of the seed values")
        if sv is not None:
            if self.costVariation is not None and sv.shape[0] != self.costVariation.shape[-1]:
                raise ValueError("costVariation and seedValueVariation have different numbers of variations")
        self.seedValueVariation = sv
        self.forwardAD = self.costVariation is not None or sv is not None
        seedRadius = float(self.GetValue(
            "seedRadius", default=2.0 if self.factoringRadius else 0.0,
            help="Spread the seeds over a radius given in pixels, so as to improve accuracy."))
        seeds_h = self.hfmIn.host("seeds").reshape(-1, self.ndim)
        ci = self.hfmIn.PointFromIndex(seeds_h, to=True)
        self.factor = None
        if self.factoringRadius:  # single seed only (_Kernel.py:301-308)
            if len(ci) != 1:
                raise ValueError("factoringRadius needs a single seed (as the reference)")
            m0 = self._seed_metric(np.asarray(ci[0], np.float64))
            nd = self.ndim
            fm = ([m0[i, j] for i in range(nd) for j in range(i + 1)] if self.model_ in ("Riemann", "Rander")
                  else list(np.diag(m0)))
            self.factor = (self.factoringRadius ** 2, np.asarray(ci[0], np.float64), np.asarray(fm, np.float64))
        if seedRadius:
            if len(ci) != 1:
                raise ValueError("seedRadius spreads a single seed (as the reference's SetRHS does)")
            idx, vals = self._spread_seed(ci[0], float(_host_scalar(seedValues[0])), seedRadius)
            seedValues = torch.as_tensor(vals, dtype=torch.float32, device="cuda")
            self.seed_owner = np.zeros(len(idx), np.int64)  # every spread point comes from seed 0
        else:
            idx = np.round(ci).astype(np.int64)
            inside = np.all((idx >= 0) & (idx < np.array(self.shape)), axis=1)
            if not np.all(inside):
                raise ValueError(f"Seeds outside the domain: {np.asarray(seeds_h)[~inside].tolist()}")
            self.seed_owner = np.arange(len(idx))
        self.nseeds_in = len(ci)
        self.seedIndices = idx
        self.seed_values = seedValues.contiguous().float()
        self.seed_idx_t = torch.from_numpy(idx.astype(np.int32)).pin_memory().to("cuda", non_blocking=True)
        self.seedbits = torch.empty(self.size_tot // 8, dtype=torch.uint8, device="cuda")
        # with walls, the first tiles are those of the seeds alone (_SetArgs.py:119-126)
        self.trigger_t = None if self.walls is None else torch.zeros(self.size_o, dtype=torch.uint8, device="cuda")
        _lib.check(L.agd_prep_seeds(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self.seed_idx_t),
                                    _lib.ptr(self.seed_values), len(idx), _lib.ptr(self.rhs_t),
                                    _lib.ptr(self.seedbits), _lib.ptr(self.trigger_t), self.stream), "seeds")
        if self.walls is not None:  # walls: seeds of value +inf, after the seeds
            tmp = torch.empty(2 * int(np.prod(self.shape)), dtype=torch.uint8, device="cuda")
            _lib.check(L.agd_prep_walls(self.ndim, self.c_shape, self.c_shape_i, _lib.ptr(self.walls),
                                        self.wallDistBound, _lib.ptr(self.wall_dist), _lib.ptr(tmp),
                                        _lib.ptr(self.rhs_t), _lib.ptr(self.seedbits), self.stream), "walls")

    def _rander_parts(self, pts=None):
        """Rander metric (M, w) with the grid scales applied (index units, no
        cost), float64 host arrays, at the grid points pts (k, ndim) or at every
        point (pts None): the dual metric is turned into the metric first."""
        nd = self.ndim
        sd = nd * (nd + 1) // 2
        fm = self._metric_flat.reshape(-1, sd + nd)
        if pts is not None:
            flat = torch.as_tensor(np.ravel_multi_index(np.asarray(pts).T, self.shape), device="cuda")
            fm = fm[flat] if fm.shape[0] > 1 else fm.expand(len(pts), sd + nd)
        fm = fm.double().cpu().numpy()
        M = np.zeros((len(fm), nd, nd))
        k = 0
        for i in range(nd):
            for j in range(i + 1):
                M[:, i, j] = M[:, j, i] = fm[:, k]
                k += 1
        w = fm[:, sd:]
        h = self.h.astype(np.float64)
        if self._metric_is_dual:  # dualMetric.with_speeds(h), then dual() (rander.py:35-39)
            M, w = M / np.outer(h, h), w / h
            s_ = np.linalg.inv(M - w[:, :, None] * w[:, None, :])
            om = np.einsum("kij,kj->ki", s_, w)
            return (1 + (w * om).sum(-1))[:, None, None] * s_, -om
        return M * np.outer(h, h), w * h

    def _cost_metrics(self, pts, drift=False):
        """The metric with the grid scales and the cost applied (index units;
        Interface.CostMetric, _Interface.py:202-211) at the grid points pts
        (k, ndim): (k, ndim, ndim) float64 (the quadratic part for Rander), and
        the cost there; with drift, also the Rander drift (k, ndim) (zero for
        the other models)."""
        nd = self.ndim
        flat = torch.as_tensor(np.ravel_multi_index(np.asarray(pts).T, self.shape), device="cuda")
        cost = self.cost.reshape(-1)[flat] if self.cost.dim() else self.cost.expand(len(pts))
        cost = cost.double().cpu().numpy()
        if self.model_ == "Rander":  # Rander.with_cost: (c^2 M, c w)
            M, w = self._rander_parts(pts)
            M = cost[:, None, None] ** 2 * M
            return (M, cost, cost[:, None] * w) if drift else (M, cost)
        if drift:
            M, c = self._cost_metrics(pts)
            return M, c, np.zeros((len(pts), nd))
        h = self.h.astype(np.float64)
        if self.model_ == "Isotropic":  # Diagonal(ones).with_costs(h).with_cost(cost)
            return np.einsum("ki,ij->kij", (cost[:, None] * h) ** 2, np.eye(nd)), cost
        if self.model_ == "Diagonal":  # Diagonal(costs).with_costs(h).with_cost(cost)
            fc = self._metric_flat.reshape(-1, nd)
            fc = (fc[flat] if fc.shape[0] > 1 else fc.expand(len(pts), nd)).double().cpu().numpy()
            if self._metric_is_dual:
                fc = 1.0 / fc
            return np.einsum("ki,ij->kij", (fc * cost[:, None] * h) ** 2, np.eye(nd)), cost
        sd = nd * (nd + 1) // 2
        fm = self._metric_flat.reshape(-1, sd)
        fm = (fm[flat] if fm.shape[0] > 1 else fm.expand(len(pts), sd)).double().cpu().numpy()
        M = np.zeros((len(pts), nd, nd))
        k = 0
        for i in range(nd):
            for j in range(i + 1):
                M[:, i, j] = M[:, j, i] = fm[:, k]
                k += 1
        if self._metric_is_dual:
            M = np.linalg.inv(M)
        return cost[:, None, None] ** 2 * M * np.outer(h, h), cost

    def _seed_metric(self, seed):
        """The cost metric at a seed (continuous index coordinates), interpolated
        multilinearly like the reference's set_interpolation: its entries
        (Riemann), or the costs c*h of the diagonal metric (Isotropic)."""
        import itertools
        nd = self.ndim
        shape = np.array(self.shape)
        lo = np.clip(np.floor(seed).astype(np.int64), 0, shape - 1)
        bits = np.array(list(itertools.product((0, 1), repeat=nd)))
        corners = np.minimum(lo + bits, shape - 1)
        frac = np.clip(seed - lo, 0.0, 1.0)
        wc = np.prod(np.where(bits == 1, frac, 1.0 - frac), axis=1)
        m, cost = self._cost_metrics(corners)
        if self.model_ in ("Riemann", "Rander"):
            return np.tensordot(wc, m, axes=1)
        # diagonal metrics: the costs c*h per axis are interpolated, then squared
        return np.diag(np.dot(wc, np.sqrt(np.diagonal(m, axis1=1, axis2=2))) ** 2)

    def _seed_drift(self, seed):
        """The drift of the cost metric at a seed, interpolated multilinearly
        (zero for the models without drift)."""
        import itertools
        nd = self.ndim
        shape = np.array(self.shape)
        lo = np.clip(np.floor(seed).astype(np.int64), 0, shape - 1)
        bits = np.array(list(itertools.product((0, 1), repeat=nd)))
        corners = np.minimum(lo + bits, shape - 1)
        frac = np.clip(seed - lo, 0.0, 1.0)
        wc = np.prod(np.where(bits == 1, frac, 1.0 - frac), axis=1)
        return wc @ self._cost_metrics(corners, drift=True)[2]

    def _spread_seed(self, seed, seed_value, r):
        """SetRHS's seed spreading (agd/Eikonal/HFM_CUDA/_SetArgs.py:46-75): the grid
        points closer than r (index units, inside the domain) to the seed become
        seeds with value seed_value + (|d|_{M(seed)} + |d|_{M(x)}) / 2, d = x - seed,
        M the cost metric (_cost_metrics), interpolated at the seed (_seed_metric)."""
        nd = self.ndim
        seed = np.asarray(seed, np.float64)
        shape = np.array(self.shape)
        aX = [np.arange(int(np.floor(c - r)), int(np.ceil(c + r) + 1)) for c in seed]
        neigh = np.stack(np.meshgrid(*aX, indexing="ij"), axis=-1).reshape(-1, nd)
        neigh = neigh[np.linalg.norm(neigh - seed, axis=-1) < r]
        neigh = neigh[np.all((-0.5 <= neigh) & (neigh < shape - 0.5), axis=-1)]
        m1, _, w1 = self._cost_metrics(neigh, drift=True)
        m0 = self._seed_metric(seed)
        w0 = self._seed_drift(seed)
        d = neigh - seed  # Rander norms add the drift term <w, d>
        n0 = np.sqrt(np.einsum("ki,ij,kj->k", d, m0, d)) + d @ w0
        n1 = np.sqrt(np.einsum("ki,kij,kj->k", d, m1, d)) + np.einsum("ki,ki->k", d, w1)
        return neigh.astype(np.int64), (seed_value + 0.5 * (n0 + n1)).astype(np.float32)

    def instance(self):
        inst = _lib.AgdInstance()
        inst.model = {"Riemann": _lib.AGD_MODEL_RIEMANN, "Diagonal": _lib.AGD_MODEL_DIAGONAL,
                      "Rander": _lib.AGD_MODEL_RANDER}.get(self.model_, _lib.AGD_MODEL_ISOTROPIC)
        inst.ndim = self.ndim
        for k in range(3):
            inst.shape[k] = self.shape[k] if k < self.ndim else 1
            inst.shape_i[k] = self.shape_i[k] if k < self.ndim else 1
            inst.iso_weights[k] = float(self.h[k]) ** -2 if k < self.ndim else 0.0
        inst.niter_i = self.niter_i
        inst.fim_front_width = self.fim_front_width
        inst.nitermax_o = self.nitermax_o
        inst.flags = (_lib.AGD_FLAG_ACTIVATE_ALL if self.activateAll else 0) | {
            "adaptive_gauss_siedel_iteration": _lib.AGD_FLAG_SOLVER_AGSI,
            "global_iteration": _lib.AGD_FLAG_SOLVER_GLOBAL}.get(getattr(self, "solver", ""), 0)
        inst.atol, inst.rtol = self.atol, self.rtol
        inst.values = self.values_t.data_ptr()
        if self.multiprecision:
            inst.multip_step, inst.multip_max = self.multip_step, self.multip_max
            inst.valuesq = self.valuesq_t.data_ptr()
            inst.values_next = self.values_next_t.data_ptr()
            inst.valuesq_next = self.valuesq_next_t.data_ptr()
        inst.geom = self.geom.data_ptr() if self.geom is not None else None
        inst.rhs = self.rhs_t.data_ptr()
        inst.seedbits = self.seedbits.data_ptr()
        if getattr(self, "trigger_t", None) is not None:
            inst.trigger = self.trigger_t.data_ptr()
        if getattr(self, "wall_dist", None) is not None:
            inst.wall_dist = self.wall_dist.data_ptr()
        if getattr(self, "release_t", None) is not None:  # tile release epochs (learned schedule)
            inst.release = self.release_t.data_ptr()
        inst.order2_threshold = getattr(self, "order2_threshold", 0.0)
        if getattr(self, "factor", None) is not None:
            r2, origin, fm = self.factor
            inst.factor_radius2 = float(r2)
            for k in range(self.ndim):
                inst.factor_origin[k] = float(origin[k])
            for k in range(len(fm)):
                inst.factor_metric[k] = float(fm[k])
        return inst

    def Solve(self):
        """The eikonal solve (agd/Eikonal/HFM_CUDA/_solvers.py:15-57)."""
        L = _lib.lib()
        inst = self.instance()
        plan = ctypes.c_void_p()
        _lib.check(L.agd_plan_create(ctypes.byref(inst), 1, ctypes.byref(plan)), "plan")
        try:
            nbytes = L.agd_plan_workspace_bytes(plan)
            ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            stats = torch.zeros(2, dtype=torch.int64, device="cuda")
            _lib.check(L.agd_plan_upload(plan, _lib.ptr(ws), nbytes, self.stream), "upload")
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            _lib.check(L.agd_plan_run(plan, _lib.ptr(ws), nbytes, _lib.ptr(stats), None, self.stream), "solve")
            stop.record()
            stop.synchronize()
        finally:
            L.agd_plan_destroy(plan)
        s = stats.cpu().numpy()
        niter_o = int(s[0] & 0xffffffff)
        status = int((s[0] >> 32) & 0xffffffff)
        self.tile_visits = int(s[1])
        t = start.elapsed_time(stop) / 1000.0
        self.stats["eikonal"].update({"niter_o": niter_o, "time": t, "nupdate_o_total": self.tile_visits,
                                      "grid_updates": self.tile_visits * self.size_i})
        if status & ~_lib.AGD_STATUS_NOT_CONVERGED:
            raise _lib.AgdError(status, "eikonal solve failed on the device")
        if status & _lib.AGD_STATUS_NOT_CONVERGED:
            msg = (f"Solver fast_iterative_method for kernel eikonal did not reach convergence after "
                   f"maximum allowed number {self.nitermax_o} of iterations")
            if self.raiseOnNonConvergence:
                raise ValueError(msg)
            self.Warn(msg)
        self._values = None

    def combine_multiprecision(self):
        """values + valuesq * multip_step (_PostProcess.py:19-36): float64 output if
        values_float64, and float32 values for the flow, geodesics and adjoint."""
        if not self.multiprecision or getattr(self, "_combined", False):
            return
        if self.values_float64:
            u = self.squeeze(self.values_t)
            q = self.squeeze(self.valuesq_t.float())  # |uq| < 2^24 is exact in float32
            self._values64 = u.double() + q.double() * self.multip_step
        self.values_t = self.values_t + self.valuesq_t.float() * np.float32(self.multip_step)
        self._combined = True
        self._values = None

    def squeeze(self, t, nplanes=1):
        L = _lib.lib()
        out = torch.empty((nplanes,) + self.shape, dtype=torch.float32, device="cuda")
        _lib.check(L.agd_block_squeeze(self.ndim, self.c_shape, self.c_shape_i, nplanes, _lib.ptr(t),
                                       _lib.ptr(out), self.stream), "block_squeeze")
        return out if nplanes > 1 else out[0]

    @property
    def values(self):
        self.combine_multiprecision()
        if self.multiprecision and self.values_float64:
            return self._values64
        if self._values is None:
            self._values = self.squeeze(self.values_t)
        return self._values

    def PostProcess(self):
        """Upwind flow, if needed (agd/Eikonal/HFM_CUDA/_PostProcess.py:46-95)."""
        self.combine_multiprecision()
        self.exportActiveNeighs = bool(self.GetValue(
            "exportActiveNeighs", default=False,
            help="Export which finite differences are active, and the min/max index."))
        self.flow_needed = (self.reverseAD or self.forwardAD or self.hasTips or self.exportGeodesicFlow
                            or self.exportActiveNeighs)
        self.flow_normalization = None
        if not self.flow_needed:
            return
        L = _lib.lib()
        nact = self.ndim * (self.ndim + 1) // 2 if self.model_ in ("Riemann", "Rander") else self.ndim
        self.nact = nact
        self.flow_vector = torch.empty(self.ndim * self.size_tot, dtype=torch.float32, device="cuda")
        self.flow_weightsum = torch.empty(self.size_tot, dtype=torch.float32, device="cuda")
        self.flow_weights = self.flow_indices = None
        if self.reverseAD or self.forwardAD or self.exportActiveNeighs:
            self.flow_weights = torch.empty(nact * self.size_tot, dtype=torch.float32, device="cuda")
            self.flow_indices = torch.empty(nact * self.size_tot, dtype=torch.int32, device="cuda")
        inst = self.instance()
        _lib.check(L.agd_flow(ctypes.byref(inst), _lib.ptr(self.flow_vector), _lib.ptr(self.flow_weightsum),
                              _lib.ptr(self.flow_weights), _lib.ptr(self.flow_indices), self.stream), "flow")
        # drift models: the flow is normalised by the metric norm of -flow at the
        # non-seed points (_PostProcess.py:80-88), for the export and for AD
        if self.model_ == "Rander" and (self.exportGeodesicFlow or self.forwardAD or self.reverseAD):
            fv = self.squeeze(self.flow_vector, self.ndim)
            M, w = self._rander_parts()
            M = torch.as_tensor(M, device="cuda").reshape(self.shape + (self.ndim, self.ndim)) \
                if len(M) > 1 else torch.as_tensor(M[0], device="cuda")
            w = torch.as_tensor(w, device="cuda").reshape(self.shape + (self.ndim,)) \
                if len(w) > 1 else torch.as_tensor(w[0], device="cuda")
            v = -torch.movedim(fv, 0, -1).double()
            n = torch.sqrt(torch.einsum("...i,...ij,...j->...", v, M.expand(v.shape + (self.ndim,)), v)) + \
                (w.expand(v.shape) * v).sum(-1)
            self.flow_normalization = torch.where(self._seed_tags(), torch.ones_like(n), n).float()
        if self.exportGeodesicFlow:
            fv = self.squeeze(self.flow_vector, self.ndim)
            if self.flow_normalization is not None:
                fv = fv / self.flow_normalization
            h = torch.as_tensor(self.h, device="cuda").reshape((self.ndim,) + (1,) * self.ndim)
            self.hfmOut["flow"] = fv * (-h)
        if self.exportActiveNeighs:
            # bit k: the k-th finite difference has a positive flow weight; the mix
            # index above the nact bits is 0 for these models (cuda/Update.h:187,206)
            fw = self.squeeze(self.flow_weights, nact).reshape((nact,) + self.shape)
            bits = torch.zeros(self.shape, dtype=torch.int32, device="cuda")
            for k in range(nact):
                bits |= (fw[k] > 0).to(torch.int32) << k
            self.hfmOut["activeNeighs"] = bits

    def _seed_tags(self):
        """Seeds and walls, grid layout (the reference's seedTags)."""
        tags = torch.zeros(self.shape, dtype=torch.bool, device="cuda")
        tags[tuple(torch.as_tensor(self.seedIndices.T, device="cuda").long())] = True
        if getattr(self, "walls", None) is not None:
            tags |= self.walls.bool()
        return tags

    def SolveAD(self):
        """Forward and reverse differentiation (agd/Eikonal/HFM_CUDA/_PostProcess.py:155-219)."""
        if self.forwardAD:
            self._forward_ad()
        if not self.reverseAD:
            return
        sens = self.GetValue("sensitivity", help="Reverse automatic differentiation")
        sens = _to_tensor(sens)
        if tuple(sens.shape[:-1]) != self.shape:
            raise ValueError(f"Reverse AD rhs shape {tuple(sens.shape)} does not start with {self.shape}")
        allS = self.reverse_columns(sens)
        pos = tuple(torch.as_tensor(self.seedIndices.T, device="cuda").long())
        seedS = allS[pos].clone()
        allS[pos] = 0
        if self.flow_normalization is not None:  # drift models (_PostProcess.py:213-214)
            allS = allS / self.flow_normalization[..., None]
        self.hfmOut["costSensitivity"] = allS
        if self.nseeds_in != len(self.seedIndices):  # spread seeds: each depends on its seed with weight 1
            owner = torch.as_tensor(self.seed_owner, device="cuda")
            seedS = torch.zeros((self.nseeds_in, seedS.shape[1]), dtype=seedS.dtype,
                                device="cuda").index_add_(0, owner, seedS)
        self.hfmOut["seedValueSensitivity"] = seedS

    def _linear_columns(self, rhs, reverse):
        """Solves the transposed (reverse) or plain (forward) linear system of the
        flow pass's weights for each column of rhs (*shape, n), grid layout;
        returns the unknowns (*shape, n).  Tolerances: rtol = 5 float32
        resolutions, atol = rtol * mean |rhs| (_PostProcess.py:155-219)."""
        L = _lib.lib()
        inst = self.instance()
        nbytes = L.agd_reverse_workspace_bytes(ctypes.byref(inst))
        ws = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device="cuda")
        stats = torch.zeros(2, dtype=torch.int64, device="cuda")
        rtol = _FLOAT_RES * 5.0
        fn = L.agd_reverse if reverse else L.agd_forward
        name = "reverse" if reverse else "forward"
        out = []
        for r in range(rhs.shape[-1]):
            col = rhs[..., r].contiguous()
            r_t = torch.empty(self.size_tot, dtype=torch.float32, device="cuda")
            _lib.check(L.agd_block_expand(self.ndim, self.c_shape, self.c_shape_i, 1, _lib.ptr(col), 0,
                                          ctypes.c_float(0.0), _lib.ptr(r_t), self.stream), name + " rhs")
            fin = col[torch.isfinite(col)]
            atol = float(rtol * fin.abs().mean()) if fin.numel() else 0.0
            x = torch.empty(self.size_tot, dtype=torch.float32, device="cuda")
            _lib.check(fn(ctypes.byref(inst), _lib.ptr(self.flow_weights), _lib.ptr(self.flow_indices),
                          _lib.ptr(self.flow_weightsum), _lib.ptr(r_t), _lib.ptr(x), ctypes.c_float(atol),
                          ctypes.c_float(rtol), _lib.ptr(ws), int(nbytes), _lib.ptr(stats), None, self.stream), name)
            st = stats.cpu().numpy()
            status = int((st[0] >> 32) & 0xffffffff)
            if status:
                raise _lib.AgdError(status, f"{name} linear solve failed on the device")
            self.stats["reverseAD" if reverse else "forwardAD"] = {"niter_o": int(st[0] & 0xffffffff),
                                                                   "nupdate_o_total": int(st[1])}
            out.append(self.squeeze(x))
        return torch.stack(out, dim=-1)

    def reverse_columns(self, sens):
        """Adjoint unknowns lam (*shape, n) of the right-hand sides sens (*shape, n):
        diag lam - W^T lam = sens, from the flow of the last PostProcess (no
        key is read; seeds are not zeroed)."""
        return self._linear_columns(sens, reverse=True)

    def forward_columns(self, rhs):
        """Variations du (*shape, n) of the right-hand sides rhs (*shape, n):
        diag du - W du = rhs, from the flow of the last PostProcess."""
        return self._linear_columns(rhs, reverse=False)

    def _forward_ad(self):
        """valueVariation (*shape, n): the linearised solve with the right-hand side
        cost * costVariation, and seedValueVariation at the seeds
        (_PostProcess.py:181-191).  The reference returns the values as a dense AD
        array with these coefficients; they are the hfmOut key valueVariation here."""
        cv, sv = self.costVariation, self.seedValueVariation
        n = cv.shape[-1] if cv is not None else sv.shape[0]
        if cv is None:
            cv = torch.zeros(self.shape + (n,), dtype=torch.float32, device="cuda")
        value = (self.cost.expand(self.shape) if self.cost.dim() == 0 else self.cost).clone()
        pos = tuple(torch.as_tensor(self.seedIndices.T, device="cuda").long())
        value[pos] = self.seed_values.to(value.dtype)
        rhs_all = cv * value[..., None]
        rhs_all[pos] = sv.T[torch.as_tensor(self.seed_owner, device="cuda")] if sv is not None else 0.0
        if self.walls is not None:  # the walls' right-hand side +inf does not vary
            rhs_all[self.walls.bool()] = 0.0
        if self.flow_normalization is not None:  # drift models (_PostProcess.py:185)
            rhs_all = rhs_all * self.flow_normalization[..., None]
        self.hfmOut["valueVariation"] = self.forward_columns(rhs_all)

    def GetGeodesics(self):
        """Geodesic backtracking (agd/Eikonal/HFM_CUDA/_GetGeodesics.py:9-147)."""
        if not self.hasTips:
            return
        L = _lib.lib()
        step = float(self.GetValue("geodesic_step", default=0.25,
                                   help="Step size, in pixels, for the geodesic ODE solver"))
        eucl_delay = int(self.GetValue("geodesic_PastSeed_delay", default=np.sqrt(self.ndim) / step,
                                       help="Delay, in iterations, for the 'PastSeed' stopping criterion of the "
                                            "geodesic ODE solver"))
        nymin_delay = int(self.GetValue("geodesic_Stationnary_delay", default=8.0 * np.sqrt(self.ndim) / step,
                                        help="Delay, in iterations, for the 'Stationnary' stopping criterion of "
                                             "the geodesic ODE solver"))
        max_len = int(max(40, 20 * np.max(self.shape) / step))
        max_len = self.GetValue("geodesic_max_length", default=max_len, help="Maximum allowed length of geodesics.")
        typical_len = int(max(40, 0.5 * np.max(self.shape) / step))
        typical_len = int(self.GetValue("geodesic_typical_length", default=min(max_len, typical_len),
                                        help="Typical expected length of geodesics (number of points)."))
        pastseed_delay = int(self.GetValue("pastseed_delay", default=0,
                                           help="Number of geodesic backtracking steps before checking "
                                                "the PastSeed criterion (use if seed and tip are close)"))
        causality = float(self.GetValue("geodesic_causalityTolerance", default=4.0,
                                        help="Used in criterion for rejecting points in flow interpolation"))
        eucl_bound = float(self.GetValue("geodesic_targetTolerance", default=6,
                                         help="Tolerance, in pixels, for declaring a seed as reached."))
        if max_len == np.inf or max_len is None:
            max_chunks = 1 << 20
        else:
            max_chunks = int(np.ceil(float(max_len) / typical_len))
        tips = self.tips
        ntips = int(tips.shape[0])
        seed_mask = torch.zeros(self.shape, dtype=torch.uint8, device="cuda")
        seed_mask[tuple(torch.as_tensor(self.seedIndices.T, device="cuda").long())] = 1
        eucl = torch.empty(self.shape, dtype=torch.uint8, device="cuda")
        tmp = torch.empty_like(eucl)
        _lib.check(L.agd_eucl_map(self.ndim, self.c_shape, _lib.ptr(seed_mask), int(np.ceil(eucl_bound)),
                                  int(5 * eucl_bound), _lib.ptr(eucl), _lib.ptr(tmp), self.stream), "eucl")
        start = torch.as_tensor(self.hfmIn.corners[0] + 0.5 * self.hfmIn.gridScales, device="cuda")
        hh = torch.as_tensor(self.h, device="cuda")
        tips_c = ((tips.float() - start) / hh).contiguous()
        cap = max_chunks * (typical_len - 1) + 1
        paths = torch.empty((ntips, cap, self.ndim), dtype=torch.float32, device="cuda")
        lengths = torch.empty(ntips, dtype=torch.int32, device="cuda")
        stops = torch.empty(ntips, dtype=torch.int8, device="cuda")
        inst = self.instance()
        _lib.check(L.agd_geodesics(ctypes.byref(inst), _lib.ptr(self.flow_vector), _lib.ptr(self.flow_weightsum),
                                   _lib.ptr(eucl), _lib.ptr(tips_c), ntips, ctypes.c_float(step),
                                   ctypes.c_float(causality), typical_len, max_chunks, eucl_delay, nymin_delay,
                                   pastseed_delay, _lib.ptr(paths), cap, _lib.ptr(lengths), _lib.ptr(stops), self.stream),
                   "geodesics")
        lens = lengths.cpu().numpy()
        codes = stops.cpu().numpy()
        # all paths to physical coordinates at once; each geodesic is a (ndim, len)
        # view, transposed like the reference's PointFromIndex(geo).T
        maxlen = int(lens.max()) if ntips else 0
        phys = paths[:, :maxlen] * hh + start
        geos = [phys[i, : int(lens[i])].T for i in range(ntips)]
        crit = []
        for i in range(ntips):
            if codes[i] == 0:
                crit.append("Stopping criterion")
            else:
                crit.append(GEODESIC_CODES[int(codes[i])])
        if any(c == "Stopping criterion" for c in crit):
            self.Warn("Geodesic solver failed to converge, or geodesic has too many points"
                      " (in latter case, try setting 'geodesic_max_length':np.inf)")
        self.hfmOut["geodesics"] = geos
        self.hfmOut["geodesic_stopping_criteria"] = crit

    def FinalCheck(self):
        if self.GetValue("exportValues", False, help="Return the solution numerical values"):
            self.hfmOut["values"] = self.values
        self.extractValues = self.GetValue("extractValues", False,
                                           help="Return the solution numerical values separately from other data")
        self.retself = self.GetValue("retself", False, help="Return the class instance that did the work")
        self.hfmOut["stats"] = self.stats
        self.hfmOut["solverGPUTime"] = self.stats["eikonal"].get("time")
        self.hfmOut["keys"]["unused"] = list(set(self.hfmIn.keys()) - set(self.hfmOut["keys"]["used"]))
        if self.verbosity >= 1 and self.hfmOut["keys"]["unused"]:
            print(f"!! Warning !! Unused keys from user : {self.hfmOut['keys']['unused']}")


def _host_scalar(x):
    return float(x.item()) if isinstance(x, torch.Tensor) else float(x)


def _rander_hfm(src, ndim):
    """A Rander metric given as a Metrics.Rander-like object (attributes m of
    shape (d, d, *shape) and w of shape (d, *shape)) or as an HFM array
    (*shape, symdim + d) -> float32 CUDA tensor (*shape, symdim + d), or
    (symdim + d,) for a constant metric.  (The reference's Rander.from_HFM
    infers d from the length alone and fails for d = 2: its users pass the
    object; both forms are taken here.)"""
    sd = ndim * (ndim + 1) // 2
    if hasattr(src, "m") and hasattr(src, "w"):
        m, w = _to_tensor(src.m), _to_tensor(src.w)
        if m.shape[0] != ndim or w.shape[0] != ndim:
            raise ValueError("Metric dimension does not match the model")
        rows = [m[i, j] for i in range(ndim) for j in range(i + 1)] + [w[i] for i in range(ndim)]
        return torch.movedim(torch.stack(torch.broadcast_tensors(*rows)), 0, -1).contiguous()
    arr = _to_tensor(src)
    if arr.shape[-1] != sd + ndim:
        raise ValueError(f"Rander metric array must have {sd + ndim} components in its last axis (HFM layout)")
    return arr.contiguous()


def _costs_hfm(src, ndim):
    """A diagonal metric given as a Metrics.Diagonal-like object (attribute costs,
    shape (d, *shape) or (d,)), an isotropic one (attribute cost), or an HFM
    array (*shape, d) -> float32 CUDA tensor (*shape, d), or (d,) if constant
    (Metrics.Diagonal.from_HFM: the costs per axis, last axis)."""
    if hasattr(src, "costs"):
        c = _to_tensor(src.costs)
        if c.shape[0] != ndim:
            raise ValueError("Metric dimension does not match the model")
        return torch.movedim(c, 0, -1).contiguous()
    if isinstance(src, Metrics.Isotropic) or hasattr(src, "cost"):
        c = _to_tensor(src.cost)
        return c[..., None].expand(tuple(c.shape) + (ndim,)).contiguous()
    arr = _to_tensor(src)
    if arr.shape[-1] != ndim:
        raise ValueError(f"Diagonal metric array must have {ndim} components in its last axis (HFM layout)")
    return arr.contiguous()


def _metric_hfm(src, ndim):
    """A metric given as a Metrics.Riemann-like object (attribute m, shape
    (d,d,*shape) or (d,d)) or as an HFM array (*shape, symdim) -> float32 CUDA
    tensor in HFM layout (*shape, symdim), or (symdim,) for a constant metric."""
    symdim = ndim * (ndim + 1) // 2
    if hasattr(src, "m"):
        m = _to_tensor(src.m)
        if m.shape[0] != ndim or m.shape[1] != ndim:
            raise ValueError("Metric dimension does not match the model")
        rows = [m[i, j] for i in range(ndim) for j in range(i + 1)]
        return torch.movedim(torch.stack(rows), 0, -1).contiguous()
    if isinstance(src, Metrics.Isotropic) or hasattr(src, "cost"):
        c = _to_tensor(src.cost)
        eye = [(1.0 if i == j else 0.0) for i in range(ndim) for j in range(i + 1)]
        e = torch.as_tensor(eye, device="cuda", dtype=torch.float32)
        return (c[..., None] ** 2 * e).contiguous() if c.dim() else (c ** 2 * e).contiguous()
    arr = _to_tensor(src)
    if arr.shape[-1] != symdim:
        raise ValueError(f"Metric array must have {symdim} components in its last axis (HFM layout)")
    return arr.contiguous()
