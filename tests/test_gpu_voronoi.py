"""GPU parity of the standalone decomposition (Eikonal.VoronoiDecomposition,
Selling.Decomposition, agd_voronoi_decomposition).

Offsets bit-exact against the reference's own kernel (decomp_m, golden
fixtures of 3000 tensors in 2D and 3D), weights to the rounding bound of their
cancelling sums, the reference's layouts (weights (symdim, *shape), offsets
(d, symdim, *shape)), reconstruction D = sum_k w_k e_k e_k^T, the integer
types of the offsets, dimension 1, and the gradient of the weights.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _spd(rng, nd, shape, cond=50.0):
    n = int(np.prod(shape))
    q, _ = np.linalg.qr(rng.standard_normal((n, nd, nd)))
    ev = np.exp(rng.uniform(0, np.log(cond), (n, nd)))
    M = q @ (ev[:, :, None] * np.swapaxes(q, 1, 2))
    return np.moveaxis(M, 0, -1).reshape((nd, nd) + shape).astype(np.float32)


def _reconstruct(w, e):
    e = e.to(torch.float64)
    return torch.einsum("k...,ik...,jk...->ij...", w.to(torch.float64), e, e)


@pytest.mark.parametrize("nd", [2, 3])
def test_offsets_bitexact_vs_reference_kernel(nd):
    from adaptivegriddiscretizations_b200 import Eikonal
    f = np.load(os.path.join(GOLDEN, f"selling{nd}.npz"))
    m = torch.as_tensor(np.ascontiguousarray(f["m"].T), device="cuda")  # (symdim, n), flattened
    w, e = Eikonal.VoronoiDecomposition(m, flattened=True)
    assert w.shape == (m.shape[0], m.shape[1]) and e.shape == (nd, m.shape[0], m.shape[1])
    assert e.dtype == torch.int32
    assert np.array_equal(e.cpu().numpy(), np.transpose(f["ref_e"], (2, 1, 0)))
    wr = f["ref_w"].T
    mnorm = np.abs(f["m"]).sum(axis=1)[None] * 2
    b2 = np.maximum((f["ref_e"].astype(np.float64) ** 2).sum(axis=2).max(axis=1)[None], 1)
    assert (np.abs(w.cpu().numpy() - wr) <= 4 * np.finfo(np.float32).eps * b2 * mnorm).all()


@pytest.mark.parametrize("nd", [2, 3])
def test_layout_and_reconstruction(nd):
    from adaptivegriddiscretizations_b200 import Eikonal, Selling
    rng = np.random.default_rng(nd)
    D = _spd(rng, nd, (7, 5))
    Dt = torch.as_tensor(D, device="cuda")
    w, e = Eikonal.VoronoiDecomposition(Dt)
    sd = nd * (nd + 1) // 2
    assert w.shape == (sd, 7, 5) and e.shape == (nd, sd, 7, 5) and w.is_cuda
    assert (w >= -1e-6 * Dt.abs().amax()).all()
    rec = _reconstruct(w, e).cpu().numpy()
    assert np.abs(rec - D).max() <= 1e-5 * np.abs(D).max()
    # host arrays: numpy out, same numbers; Selling.Decomposition is the same op
    wh, eh = Eikonal.VoronoiDecomposition(D, mode="gpu_transfer")
    assert isinstance(wh, np.ndarray) and np.array_equal(wh, w.cpu().numpy()) and np.array_equal(eh, e.cpu().numpy())
    ws, es = Selling.Decomposition(Dt)
    assert torch.equal(ws, w) and torch.equal(es, e)
    ws, es = Selling.Decomposition(D)
    assert isinstance(ws, np.ndarray) and np.array_equal(es, eh)


@pytest.mark.parametrize("offset_t", [torch.int8, torch.int16, torch.int64, np.int32])
def test_offset_types(offset_t):
    from adaptivegriddiscretizations_b200 import Eikonal
    D = torch.as_tensor(_spd(np.random.default_rng(3), 2, (300,), cond=20.0), device="cuda")
    w0, e0 = Eikonal.VoronoiDecomposition(D)
    w, e = Eikonal.VoronoiDecomposition(D, offset_t=offset_t)
    assert torch.equal(w, w0) and torch.equal(e.to(torch.int32), e0)


def test_dimension_one_and_errors():
    from adaptivegriddiscretizations_b200 import Eikonal
    m = torch.rand((1, 1, 10), device="cuda") + 0.5
    w, e = Eikonal.VoronoiDecomposition(m)
    assert torch.equal(w, m[0]) and (e == 1).all() and e.shape == (1, 1, 10)
    with pytest.raises(ValueError):
        Eikonal.VoronoiDecomposition(m, mode="cpu")
    with pytest.raises(ValueError):
        Eikonal.VoronoiDecomposition(torch.eye(4, device="cuda")[:, :, None])


@pytest.mark.parametrize("nd", [2, 3])
def test_weights_gradient(nd):
    """d<g, w>/dD by autograd against central differences along a direction
    that keeps the offsets (the weights are linear in D for fixed offsets); the
    upper triangle of a full-matrix input gets no gradient, as in the reference."""
    from adaptivegriddiscretizations_b200 import Eikonal
    rng = np.random.default_rng(10 + nd)
    D = torch.as_tensor(_spd(rng, nd, (64,), cond=10.0), device="cuda", dtype=torch.float32)
    g = torch.as_tensor(rng.standard_normal((nd * (nd + 1) // 2, 64)), device="cuda", dtype=torch.float32)
    Dv = D.clone().requires_grad_(True)
    w, e = Eikonal.VoronoiDecomposition(Dv)
    (w * g).sum().backward()
    grad = Dv.grad
    iu = torch.triu_indices(nd, nd, 1)
    assert (grad[iu[0], iu[1]] == 0).all()
    S = torch.as_tensor(rng.standard_normal((nd, nd, 64)), device="cuda", dtype=torch.float32)
    S = torch.tril(S.permute(2, 0, 1)).permute(1, 2, 0)  # lower triangle only: the flattened entries
    eps = 1e-3 * D.abs().amax()
    wp, ep = Eikonal.VoronoiDecomposition(D + eps * (S + S.transpose(0, 1) * (1 - torch.eye(nd, device="cuda")[..., None])))
    wm, em = Eikonal.VoronoiDecomposition(D - eps * (S + S.transpose(0, 1) * (1 - torch.eye(nd, device="cuda")[..., None])))
    keep = (ep == e).all(0).all(0) & (em == e).all(0).all(0)
    assert keep.float().mean() > 0.9
    fd = ((wp - wm) * g).sum(0) / (2 * eps)
    ad = (grad * S).sum((0, 1))
    scale = (g.abs().sum(0) * 1.0).clamp(min=1.0)
    assert ((fd - ad).abs()[keep] <= 2e-2 * scale[keep]).all()
