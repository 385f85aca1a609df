"""dictIn / dictOut: the input and output mappings of the eikonal solver.

Mirrors agd/Eikonal/DictIn.py (class dictIn: 110-525, dictOut: 59-95) for the
GPU modes: 'gpu' holds torch CUDA tensors, 'gpu_transfer' holds numpy arrays
on the host and returns numpy arrays.  The grid helpers (SetRect, Grid, Axes,
PointFromIndex, IndexFromPoint, SetUniformTips, GridNeighbors, gridScales,
corners) follow the reference's definitions.
"""
from collections.abc import MutableMapping

import numpy as np
import torch

_array_float_fields = {
    "origin", "dims", "gridScale", "gridScales", "values",
    "seeds", "tips", "seedValues", "cost", "speed", "costVariation",
}

_singleIn = {"seed": "seeds", "seedValue": "seedValues", "tip": "tips"}
_readonlyIn = {"float_t"}
_singleOut = {"geodesic": "geodesics"}
_modes = ("gpu", "gpu_transfer")


# Fields of at most this many entries keep a host copy taken when they are
# assigned, so that reading them back (domain shape, grid scales, seeds) needs
# no device-to-host copy and no wait for the device.
_SHADOW_MAX = 4096


class _Deferred:
    """A small host-side array of a 'gpu' mode dictIn, copied to the device when
    the key is first read (so that building a dictIn makes no device copy)."""

    __slots__ = ("host",)

    def __init__(self, host):
        self.host = host


def _is_array(x):
    return isinstance(x, (np.ndarray, torch.Tensor))


def _host_copy(x):
    """float32 numpy copy of a small host-side value; None for device tensors
    (reading them would wait for the device) and for large arrays."""
    if isinstance(x, torch.Tensor):
        if x.device.type != "cpu" or x.numel() > _SHADOW_MAX:
            return None
        return x.detach().numpy().astype(np.float32, copy=True)
    try:
        a = np.asarray(x, dtype=np.float32)
    except (TypeError, ValueError):
        return None
    return a.copy() if a.size <= _SHADOW_MAX else None


class dictOut(MutableMapping):
    """Dictionary-like output of the eikonal solver (agd/Eikonal/DictIn.py:59-95)."""

    def __init__(self, store=None):
        self.store = {} if store is None else store

    def __copy__(self):
        return dictOut(self.store.copy())

    def copy(self):
        return self.__copy__()

    def __repr__(self):
        return f"dictOut({self.store})"

    def __setitem__(self, key, value):
        if key in _singleOut:
            key, value = _singleOut[key], [value]
        self.store[key] = value

    def __getitem__(self, key):
        if key in _singleOut:
            values = self.store[_singleOut[key]]
            if len(values) != 1:
                raise ValueError(f"Found {len(values)} values for key {key}")
            return values[0]
        return self.store[key]

    def __delitem__(self, key):
        del self.store[_singleOut.get(key, key)]

    def __iter__(self):
        return iter(self.store)

    def __len__(self):
        return len(self.store)

    def keys(self):
        return self.store.keys()


def CenteredLinspace(a, b, n):
    """linspace shifted by half a step (agd/Eikonal/DictIn.py:97-108)."""
    n_ = int(n)
    assert n == n_
    r, dr = np.linspace(a, b, n_, endpoint=False, retstep=True)
    if np.any(np.isnan(dr)):
        assert n == 1
        dr = b - a
    return r + dr / 2


class dictIn(MutableMapping):
    """Input mapping of the eikonal solver.  Mode 'gpu' (torch CUDA tensors) or
    'gpu_transfer' (numpy arrays in and out); float32 throughout."""

    default_mode = "gpu"

    def __init__(self, store=None):
        if store is None:
            store = {}
        self.store = {"arrayOrdering": "RowMajor"}
        self._shadow = {}
        mode = store.get("mode", dictIn.default_mode)
        if mode not in _modes:
            raise ValueError(f"Unsupported mode {mode!r}: this solver runs on the GPU (modes {_modes})")
        self.store["mode"] = mode
        self._mode = mode
        self._float_t = np.float32
        if "float_t" in store and np.dtype(store["float_t"]) != np.float32:
            raise ValueError("Only float32 data is supported by the GPU solver")
        if store:
            self.update(store)

    # ------------------------------------------------------------ mapping ---
    @property
    def mode(self):
        return self._mode

    @property
    def float_t(self):
        return self._float_t

    def array_float_caster(self, x):
        if self.mode == "gpu":
            if isinstance(x, torch.Tensor):
                return x.to(device="cuda", dtype=torch.float32, non_blocking=x.is_pinned())
            return torch.as_tensor(np.asarray(x, dtype=np.float32), device="cuda")
        if isinstance(x, torch.Tensor):
            x = x.detach().cpu().numpy()
        return np.asarray(x, dtype=np.float32)

    def __copy__(self):
        other = dictIn(self.store.copy())
        other._shadow = {k: v for k, v in self._shadow.items() if other.store.get(k) is v[0]}
        return other

    def copy(self):
        return self.__copy__()

    def __repr__(self):
        return f"dictIn({self.store})"

    def __setitem__(self, key, value):
        if key == "mode":
            if value not in _modes:
                raise ValueError(f"Unsupported mode {value!r}")
            if value != self._mode:
                raise ValueError("Switching between modes with distinct array storage")
        if key in _readonlyIn and self.store.get(key) != value:
            raise ValueError(f"Key {key} is readonly (set at init)")
        if key in _singleIn:
            key, value = _singleIn[key], [value]
        if key in _array_float_fields:
            host = value.host if isinstance(value, _Deferred) else _host_copy(value)
            if isinstance(value, _Deferred):
                pass  # a copied dictIn: the host array stays deferred
            elif host is not None and self.mode == "gpu" and not (isinstance(value, torch.Tensor) and value.is_cuda):
                value = _Deferred(host)  # moved to the device when first read
            else:
                value = self.array_float_caster(value)
            if host is not None:
                self._shadow[key] = (value, host)
            else:
                self._shadow.pop(key, None)
        else:
            self._shadow.pop(key, None)
        self.store[key] = value

    def __getitem__(self, key):
        if key in _singleIn:
            values = self[_singleIn[key]]
            if len(values) != 1:
                raise ValueError(f"Found {len(values)} values for key {key}")
            return values[0]
        value = self.store[key]
        if isinstance(value, _Deferred):
            dev = self.array_float_caster(value.host)
            self.store[key] = dev
            self._shadow[key] = (dev, value.host)
            return dev
        return value

    def raw(self, key):
        """The stored value without moving a deferred host array to the device:
        a device tensor, or a float32 numpy array for small host-side arrays."""
        value = self.store[key]
        return value.host if isinstance(value, _Deferred) else value

    def __delitem__(self, key):
        key = _singleIn.get(key, key)
        del self.store[key]
        self._shadow.pop(key, None)

    def __iter__(self):
        return iter(self.store)

    def __len__(self):
        return len(self.store)

    def keys(self):
        return self.store.keys()

    def host(self, key):
        """numpy copy of a stored field.  Small fields answer from the copy
        taken when they were assigned (an in-place change of the stored device
        tensor after that is not seen); others are read back from the device."""
        value = self.store[key]
        shadow = self._shadow.get(key)
        if shadow is not None and shadow[0] is value:
            return shadow[1]
        return self._np(value)

    def RunHelp(self, mode=None):
        from . import HFM_CUDA
        help(HFM_CUDA.RunGPU)

    def Run(self, join=None, **kwargs):
        """Run the GPU eikonal solver and return a dictOut
        (agd/Eikonal/DictIn.py:248-285, modes 'gpu' and 'gpu_transfer')."""
        if join is not None:
            other = self.copy()
            other.update(join)
            return other.Run(**kwargs)
        if self["arrayOrdering"] != "RowMajor":
            raise ValueError("Unsupported array ordering")
        from . import HFM_CUDA
        out = HFM_CUDA.RunGPU(self, **kwargs)
        if isinstance(out, (list, tuple)):
            res = [dictOut(o) if isinstance(o, dict) else o for o in out]
            return tuple(_to_host(r) for r in res) if self.mode == "gpu_transfer" else tuple(res)
        out = dictOut(out)
        return _to_host(out) if self.mode == "gpu_transfer" else out

    # ------------------------------------------------------- grid helpers ---
    def _np(self, x):
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
        return np.asarray(x)

    @property
    def shape(self):
        dims = self.host("dims")
        return tuple(int(round(float(d))) for d in dims)

    @property
    def size(self):
        return int(np.prod(self.shape))

    @property
    def vdim(self):
        return int(self["model"][-1])

    @property
    def SE(self):
        return False

    @property
    def gridScales(self):
        if "gridScales" in self:
            return self.host("gridScales").astype(np.float32)
        return np.full(self.vdim, float(self.host("gridScale")), np.float32)

    @property
    def corners(self):
        h = self.gridScales
        dims = self.host("dims").astype(np.float32)
        origin = self.host("origin").astype(np.float32) if "origin" in self else np.zeros_like(dims)
        return origin, origin + h * dims

    def Axes(self, dims=None):
        bottom, top = self.corners
        if dims is None:
            dims = self.host("dims")
        return [np.asarray(CenteredLinspace(b, t, d), np.float32) for b, t, d in zip(bottom, top, dims)]

    def Grid(self, dims=None):
        axes = self.Axes(dims)
        return np.array(np.meshgrid(*axes, indexing="ij"))

    def SetUniformTips(self, dims):
        self["tips"] = self.Grid(dims).reshape(self.vdim, -1).T

    def SetRect(self, sides, sampleBoundary=False, gridScale=None, gridScales=None, dimx=None, dims=None):
        """Box domain (agd/Eikonal/DictIn.py:404-440)."""
        domain_count = sum(e in self for e in ("gridScale", "gridScales", "dims", "origin"))
        if domain_count not in (0, 3):
            raise ValueError("Domain already partially set")
        corner0, corner1 = np.asarray(sides, np.float32).T
        dim = len(corner0)
        sb = float(sampleBoundary)
        width = corner1 - corner0
        if gridScale is not None:
            gridScales = [gridScale] * dim
            self["gridScale"] = gridScale
        elif gridScales is not None:
            self["gridScales"] = gridScales
        elif dimx is not None:
            gridScale = width[0] / (dimx - sb)
            gridScales = [gridScale] * dim
            self["gridScale"] = gridScale
        elif dims is not None:
            gridScales = width / (np.asarray(dims, np.float32) - sb)
            self["gridScales"] = gridScales
        else:
            raise ValueError("Missing argument gridScale, gridScales, dimx, or dims")
        h = np.asarray(gridScales, np.float32)
        ratios = (corner1 - corner0) / h + sb
        dims_ = np.round(ratios)
        assert np.min(dims_) > 0
        origin = corner0 + (ratios - dims_ - sb) * h / 2
        self["dims"] = dims_
        self["origin"] = origin

    def PointFromIndex(self, index, to=False):
        """Index -> point, or point -> continuous index with to=True (DictIn.py:442-453)."""
        bottom, _ = self.corners
        scale = self.gridScales
        start = bottom + 0.5 * scale
        index = np.asarray(self._np(index), np.float32)
        assert index.shape[-1] == self.vdim
        return start + scale * index if not to else (index - start) / scale

    def IndexFromPoint(self, point):
        ci = self.PointFromIndex(point, to=True)
        index = np.round(ci)
        return index.astype(int), (ci - index)

    def VectorFromOffset(self, offset, to=False):
        offset = np.asarray(offset, np.float32)
        return offset * self.gridScales if not to else offset / self.gridScales

    def GridNeighbors(self, point, gridRadius):
        point = np.asarray(point, np.float32)
        ci = self.PointFromIndex(point, to=True)
        aX = [np.arange(int(np.floor(c - gridRadius)), int(np.ceil(c + gridRadius) + 1), dtype=np.float32) for c in ci]
        neigh_index = np.stack(np.meshgrid(*aX, indexing="ij"), axis=-1).reshape(-1, len(aX))
        close = np.sum((neigh_index - ci) ** 2, axis=-1) < gridRadius ** 2
        neigh = self.PointFromIndex(neigh_index)
        bottom, top = self.corners
        inRange = np.all(np.logical_and(bottom < neigh, neigh < top), axis=-1)
        return neigh[np.logical_and(close, inRange)]


def _to_host(obj):
    """Device tensors -> numpy, recursively (gpu_transfer mode)."""
    if isinstance(obj, torch.Tensor):
        return obj.detach().cpu().numpy()
    if isinstance(obj, dictOut):
        return dictOut({k: _to_host(v) for k, v in obj.store.items()})
    if isinstance(obj, dict):
        return {k: _to_host(v) for k, v in obj.items()}
    if isinstance(obj, list):
        return [_to_host(v) for v in obj]
    if isinstance(obj, tuple):
        return tuple(_to_host(v) for v in obj)
    return obj
