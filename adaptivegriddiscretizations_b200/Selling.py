"""Selling's decomposition of symmetric positive definite matrices of
dimension 1 to 3, D = sum_k lambda_k e_k e_k^T, on the GPU.

The reference's `agd.Selling.Decomposition` sends device (cupy) arrays to the
GPU kernel through `Eikonal.VoronoiDecomposition(m, mode='gpu')`
(agd/Selling.py:45-66) and decomposes host arrays with numpy in float64.  Here
every input is decomposed by that GPU path (`Eikonal.VoronoiDecomposition`, the
C ABI entry point `agd_voronoi_decomposition`), in float32: CUDA tensors give
CUDA tensors, host arrays give numpy arrays.  Shapes as in the reference:
m (d, d, *shape) -> weights (symdim, *shape), offsets (d, symdim, *shape); the
order of the terms is the GPU kernel's (the reference's numpy path lists the
same terms in another order).
"""
import torch

from .Eikonal.Voronoi import VoronoiDecomposition


def Decomposition(m, sb=None):
    """Weights and integer offsets of Selling's decomposition of m (d, d, *shape)."""
    if sb is not None:
        raise NotImplementedError("Selling.Decomposition: a given starting superbase is not supported "
                                  "(the GPU kernel starts from the canonical one, as the reference's does)")
    mode = "gpu" if isinstance(m, torch.Tensor) and m.is_cuda else "gpu_transfer"
    return VoronoiDecomposition(m, mode=mode)
