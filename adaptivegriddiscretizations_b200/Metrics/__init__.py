"""Metrics accepted by the eikonal solver: Riemann, Rander, Isotropic, Diagonal.

The subset of agd/Metrics used by the GPU eikonal path (riemann.py:13-165,
rander.py:10-77, isotropic.py:8-98, diagonal.py, base.py:175-250, misc.py:8-27): tensors are
stored geometry first, m of shape (d, d, *shape); `flatten` packs the lower
triangle [m00, m10, m11, m20, m21, m22]; the HFM layout puts that packing
last, (*shape, symdim).  Arrays may be numpy arrays or torch tensors.
"""
import numpy as np
import torch


def _xp(a):
    return torch if isinstance(a, torch.Tensor) else np


def _asarray(a):
    return a if isinstance(a, torch.Tensor) else np.asarray(a)


def flatten_symmetric_matrix(m):
    d = m.shape[0]
    xp = _xp(m)
    rows = [m[i, : i + 1] for i in range(d)]
    return xp.concatenate(rows, 0) if xp is np else torch.cat(rows, 0)


def expand_symmetric_matrix(arr):
    d = 0
    while (d * (d + 1)) // 2 < len(arr):
        d += 1
    assert len(arr) == d * (d + 1) // 2
    xp = _xp(arr)
    k = 0
    rows = [[None] * d for _ in range(d)]
    for i in range(d):
        for j in range(i + 1):
            rows[i][j] = rows[j][i] = arr[k]
            k += 1
    if xp is np:
        return np.array([[rows[i][j] for j in range(d)] for i in range(d)])
    return torch.stack([torch.stack([rows[i][j] for j in range(d)]) for i in range(d)])


class Base:
    def with_cost(self, cost):
        cost = _asarray(cost)
        xp = _xp(cost)
        costs = xp.broadcast_to(cost, (self.vdim,) + tuple(cost.shape))
        return self.with_costs(costs)

    def with_speed(self, speed):
        return self.with_cost(1.0 / _asarray(speed))

    def with_speeds(self, speeds):
        return self.with_costs(1.0 / _asarray(speeds))

    def to_HFM(self):
        f = self.flatten()
        xp = _xp(f)
        return xp.moveaxis(f, 0, -1) if xp is np else torch.movedim(f, 0, -1)

    @classmethod
    def from_HFM(cls, arr):
        arr = _asarray(arr)
        xp = _xp(arr)
        return cls.expand(xp.moveaxis(arr, -1, 0) if xp is np else torch.movedim(arr, -1, 0))


class Riemann(Base):
    """F(x) = sqrt(<x, m x>), m of shape (d, d, *shape)."""

    def __init__(self, m):
        self.m = _asarray(m)

    @property
    def vdim(self):
        return self.m.shape[0]

    @property
    def shape(self):
        return tuple(self.m.shape[2:])

    def _moved(self):
        xp = _xp(self.m)
        return xp.moveaxis(self.m, (0, 1), (-2, -1)) if xp is np else torch.movedim(self.m, (0, 1), (-2, -1))

    def dual(self):
        mm = self._moved()
        inv = np.linalg.inv(mm) if isinstance(mm, np.ndarray) else torch.linalg.inv(mm)
        xp = _xp(inv)
        return Riemann(xp.moveaxis(inv, (-2, -1), (0, 1)) if xp is np else torch.movedim(inv, (-2, -1), (0, 1)))

    def norm(self, v):
        v = _asarray(v)
        mv = sum(self.m[:, j] * v[j] for j in range(self.vdim))
        s = sum(v[i] * mv[i] for i in range(self.vdim))
        return np.sqrt(s) if _xp(s) is np else torch.sqrt(s)

    def with_costs(self, costs):
        costs = _asarray(costs)
        d = self.vdim
        xp = _xp(self.m)
        out = [[self.m[i, j] * costs[i] * costs[j] for j in range(d)] for i in range(d)]
        if xp is np:
            return Riemann(np.array(out))
        return Riemann(torch.stack([torch.stack(r) for r in out]))

    def flatten(self):
        return flatten_symmetric_matrix(self.m)

    @classmethod
    def expand(cls, arr):
        return cls(expand_symmetric_matrix(arr))

    def model_HFM(self):
        return "Riemann" + str(self.vdim)

    @classmethod
    def needle(cls, u, cost_parallel, cost_orthogonal):
        """Eigenvector u with eigenvalue cost_parallel**2, orthogonal eigenvalue cost_orthogonal**2."""
        u = np.asarray(u, dtype=float)
        nu = np.sqrt(np.sum(u ** 2, axis=0))
        u = np.where(nu > 0, u / np.where(nu > 0, nu, 1), u)
        d = len(u)
        cp, co = np.asarray(cost_parallel), np.asarray(cost_orthogonal)
        eye = np.eye(d).reshape((d, d) + (1,) * (u.ndim - 1))
        uu = u[:, None] * u[None, :]
        return cls((cp ** 2 - co ** 2) * uu + co ** 2 * eye)

    @classmethod
    def from_diagonal(cls, diag):
        diag = np.asarray(diag)
        d = len(diag)
        z = np.zeros_like(diag[0])
        return cls(np.array([[diag[i] if i == j else z for j in range(d)] for i in range(d)]))


class Diagonal(Base):
    """F(x) = sqrt(sum_i (costs_i x_i)^2)."""

    def __init__(self, costs):
        self.costs = _asarray(costs)

    @property
    def vdim(self):
        return len(self.costs)

    def with_costs(self, costs):
        return Diagonal(self.costs * _asarray(costs))

    def dual(self):
        return Diagonal(1.0 / self.costs)

    def flatten(self):
        return self.costs

    @classmethod
    def expand(cls, arr):
        return cls(arr)


class Isotropic(Base):
    """F(x) = cost |x|."""

    def __init__(self, cost, vdim=-1):
        self.cost = _asarray(cost)
        self._vdim = vdim

    @property
    def vdim(self):
        return self._vdim

    def with_cost(self, cost):
        return Isotropic(_asarray(cost) * self.cost, self._vdim)

    def dual(self):
        return Isotropic(1.0 / self.cost, self._vdim)

    def flatten(self):
        return self.cost

    def to_HFM(self):
        return self.cost

    @classmethod
    def from_HFM(cls, arr):
        return cls(arr)


class Rander(Base):
    """F(x) = sqrt(<x, m x>) + <w, x>, with |w|_{m^-1} < 1 (rander.py:10-77).
    m of shape (d, d, *shape), w of shape (d, *shape).  The HFM layout is the
    lower triangle of m followed by w, last axis (*shape, symdim + d)."""

    def __init__(self, m, w):
        self.m, self.w = _asarray(m), _asarray(w)

    @property
    def vdim(self):
        return len(self.m)

    def norm(self, v):
        v = _asarray(v)
        xp = _xp(v)
        quad = (self.m * v[None] * v[:, None]).sum(axis=0).sum(axis=0) if xp is np else \
            (self.m * v[None] * v[:, None]).sum(0).sum(0)
        return quad ** 0.5 + (self.w * v).sum(0)

    def dual(self):
        """The dual of a Rander norm is a Rander norm (rander.py:35-39)."""
        xp = _xp(self.m)
        m = xp.moveaxis(self.m, (0, 1), (-2, -1)) if xp is np else torch.movedim(self.m, (0, 1), (-2, -1))
        w = xp.moveaxis(self.w, 0, -1) if xp is np else torch.movedim(self.w, 0, -1)
        s = (np.linalg.inv if xp is np else torch.linalg.inv)(m - w[..., :, None] * w[..., None, :])
        om = (s @ w[..., :, None])[..., 0]
        mm = (1 + (w * om).sum(-1))[..., None, None] * s
        back = (lambda a, src, dst: np.moveaxis(a, src, dst)) if xp is np else torch.movedim
        return Rander(back(mm, (-2, -1), (0, 1)), back(-om, -1, 0))

    def with_costs(self, costs):
        c = _asarray(costs)
        return Rander(self.m * c[:, None] * c[None, :] if c.ndim == 1 and self.m.ndim == 2 else
                      self.m * (c[:, None] * c[None, :]), self.w * c)

    def flatten(self, inverse_m=False):
        m = self.m
        xp = _xp(m)
        if inverse_m:
            mm = xp.moveaxis(m, (0, 1), (-2, -1)) if xp is np else torch.movedim(m, (0, 1), (-2, -1))
            mi = (np.linalg.inv if xp is np else torch.linalg.inv)(mm)
            m = np.moveaxis(mi, (-2, -1), (0, 1)) if xp is np else torch.movedim(mi, (-2, -1), (0, 1))
        f = flatten_symmetric_matrix(m)
        return np.concatenate([f, self.w], 0) if xp is np else torch.cat([f, self.w], 0)

    @classmethod
    def expand(cls, arr):
        d = 0
        while d * (d + 3) // 2 < len(arr):  # symdim + d components
            d += 1
        assert len(arr) == d * (d + 3) // 2, "a Rander metric has d(d+1)/2 + d components"
        sd = d * (d + 1) // 2
        return cls(expand_symmetric_matrix(arr[:sd]), arr[sd:])
