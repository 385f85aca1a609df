"""Standalone decomposition of symmetric positive definite matrices on the GPU:
D = sum_k lambda_k e_k e_k^T with lambda_k >= 0 and integer offsets e_k.

The reference's `Eikonal.VoronoiDecomposition(arr, mode='gpu')`
(agd/Eikonal/__init__.py:26-90) compiles Kernel_VoronoiDecomposition.h and runs
it on flattened matrices (HFM_CUDA/VoronoiDecomposition.py:15-98); in dimension
2 and 3 that kernel is Selling's algorithm (`decomp_m`, cuda/Geometry2.h:21-48,
Geometry3.h:22-58), in dimension 1 the trivial decomposition.  Here it is the
C ABI entry point `agd_voronoi_decomposition`, with the same layouts: input
(d, d, *shape) or, with `flattened`, the lower triangles (symdim, *shape);
output weights (symdim, *shape) float32 and offsets (d, symdim, *shape).

Modes: 'gpu' (torch CUDA tensors out), 'gpu_transfer' (numpy arrays out); the
default is 'gpu' for CUDA tensors and 'gpu_transfer' otherwise, unless
`VoronoiDecomposition.default_mode` is set.  The reference's 'cpu' mode calls an external binary
(FileVDQ), which is not part of this package.  Dimensions 4 to 6 (Voronoi's
first reduction with a simplex solver in the reference) are not built.

Differentiation: the offsets are piecewise constant in D, and given them the
weights solve the linear system D_flat = A lambda, A[:, k] = flat(e_k e_k^T)
(the reference differentiates its AD inputs the same way).  A tensor input
that requires grad gets weights with that gradient; as in the reference, only
the lower triangle of a full-matrix input receives it.
"""
import numpy as np
import torch

from .. import _lib

_OFFSET_BYTES = {torch.int8: 1, torch.int16: 2, torch.int32: 4, torch.int64: 8}
_NUMPY_INT = {np.dtype(np.int8): torch.int8, np.dtype(np.int16): torch.int16, np.dtype(np.int32): torch.int32,
              np.dtype(np.int64): torch.int64}


def flatten_symmetric_matrix(m):
    """Lower triangles, row major: (d, d, *shape) -> (d(d+1)/2, *shape)
    (agd/Metrics/misc.py:8-15)."""
    d = m.shape[0]
    return torch.cat([m[i, : i + 1] for i in range(d)], dim=0)


def _offset_dtype(offset_t):
    if isinstance(offset_t, torch.dtype):
        t = offset_t
    else:
        t = _NUMPY_INT.get(np.dtype(offset_t))
    if t not in _OFFSET_BYTES:
        raise ValueError(f"offset_t must be a signed integer type of 1, 2, 4 or 8 bytes, not {offset_t}")
    return t


def _decompose(m_flat, ndim, offset_t):
    """Kernel call on (symdim, n) float32 CUDA planes; returns weights, offsets."""
    sd, n = m_flat.shape
    w = torch.empty((sd, n), dtype=torch.float32, device=m_flat.device)
    e = torch.empty((ndim, sd, n), dtype=offset_t, device=m_flat.device)
    L = _lib.lib()
    _lib.check(L.agd_voronoi_decomposition(ndim, _lib.ptr(m_flat), n, _lib.ptr(w), _lib.ptr(e),
                                           _OFFSET_BYTES[offset_t], _lib.stream_ptr()), "voronoi_decomposition")
    return w, e


def _outer_flat(e):
    """flat(e_k e_k^T) for offsets (ndim, symdim, n): returns (n, symdim[c], symdim[k]) float64."""
    ndim = e.shape[0]
    ed = e.to(torch.float64)
    rows = [ed[i] * ed[j] for i in range(ndim) for j in range(i + 1)]  # each (symdim[k], n)
    return torch.stack(rows, 0).permute(2, 0, 1)


class _Weights(torch.autograd.Function):
    """Weights of the decomposition as a differentiable function of D_flat."""

    @staticmethod
    def forward(ctx, m_flat, w, e):
        ctx.save_for_backward(e)
        return w.clone()

    @staticmethod
    def backward(ctx, gw):
        (e,) = ctx.saved_tensors
        A = _outer_flat(e)  # D_flat = A @ lambda, per matrix
        g = torch.linalg.solve(A.transpose(1, 2), gw.T.to(torch.float64).unsqueeze(-1)).squeeze(-1)
        return g.T.to(gw.dtype), None, None


def VoronoiDecomposition(arr, mode=None, steps="Both", offset_t=torch.int32, flattened=False, retry64_tol=2e-5,
                         blockDim=None, traits=None):
    """Weights (symdim, *shape) and offsets (ndim, symdim, *shape) with
    D = sum_k weights[k] offsets[:, k] offsets[:, k]^T, for the d x d matrices
    of `arr` (d, d, *shape), or their lower triangles (symdim, *shape) with
    `flattened`.  `retry64_tol`, `blockDim` and `traits` are accepted for
    compatibility; they matter only in dimensions 4 to 6 in the reference."""
    if mode is None:
        mode = VoronoiDecomposition.default_mode
    if mode is None:
        mode = "gpu" if isinstance(arr, torch.Tensor) and arr.is_cuda else "gpu_transfer"
    if mode == "cpu":
        raise ValueError("VoronoiDecomposition: mode 'cpu' runs the reference's external FileVDQ binary, "
                         "which is not part of this package; use mode 'gpu' or 'gpu_transfer'")
    if mode not in ("gpu", "gpu_transfer"):
        raise ValueError(f"VoronoiDecomposition unsupported mode {mode}")
    if steps != "Both":
        raise ValueError("VoronoiDecomposition: the two-step variant exists in dimensions 4 to 6 only")
    offset_t = _offset_dtype(offset_t)
    host = not isinstance(arr, torch.Tensor)
    t = torch.as_tensor(np.asarray(arr) if host else arr)
    t = t.to(device="cuda", dtype=torch.float32) if t.dtype != torch.float32 or not t.is_cuda else t
    m_flat = t if flattened else flatten_symmetric_matrix(t)
    sd = m_flat.shape[0]
    ndim = {1: 1, 3: 2, 6: 3}.get(sd)
    if ndim is None or (not flattened and t.shape[1] != ndim):
        raise ValueError(f"Voronoi decomposition not implemented in dimension {int(np.sqrt(2 * sd))} "
                         "(dimensions 1 to 3 here)")
    shape = tuple(m_flat.shape[1:])
    flat2 = m_flat.reshape(sd, -1)
    w, e = _decompose(flat2.detach().contiguous(), ndim, offset_t)
    if flat2.requires_grad:
        w = _Weights.apply(flat2, w, e)
    w = w.reshape((sd,) + shape)
    e = e.reshape((ndim, sd) + shape)
    if mode == "gpu_transfer":
        return w.detach().cpu().numpy(), e.cpu().numpy()
    return w, e


VoronoiDecomposition.default_mode = None
