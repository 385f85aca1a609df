"""Differentiable eikonal solve: arrival times as a function of the cost field.

`EikonalValues.apply(cost, hfmIn)` returns the values of the eikonal solve of
hfmIn with its 'cost' replaced by `cost` (a CUDA tensor of the grid shape).
The forward pass solves once and records the causal dependency of the
solution: the upwind flow weights and neighbour indices of every point
(agd_flow), as the reference's SolveAD does before its linear solves
(agd/Eikonal/HFM_CUDA/_PostProcess.py:155-219).  The backward pass reverse-
sweeps that record: it runs the adjoint linear solve of libagd_b200
(agd_reverse) on the saved flow with the incoming gradient as right-hand side,
without solving the eikonal equation again.  The adjoint unknown lam satisfies
dJ/dcost = lam * cost (the forward linearisation of the scheme uses the
right-hand side cost * dcost, _PostProcess.py:181-183), and the reference
reports lam itself as 'costSensitivity'.  Forward mode
(torch.autograd.forward_ad) runs agd_forward on the same saved flow with the
tangent times the cost as right-hand side.
"""
import torch

from .Eikonal.HFM_CUDA import Interface


class EikonalValues(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cost, hfmIn):
        h = hfmIn.copy()
        h["cost"] = cost.detach()
        h["exportValues"] = True
        for key in ("sensitivity", "tips", "costVariation", "seedValueVariation"):
            h.store.pop(key, None)
        itf = Interface(h)
        itf.SetKernelTraits()
        itf.SetGeometry()
        itf.SetArgs()
        itf.Solve()
        itf.reverseAD = True  # the flow pass records the upwind weights and indices
        itf.PostProcess()
        values = itf.values.clone()
        ctx.itf = itf
        ctx.save_for_backward(cost)
        return values

    @staticmethod
    def _seed_positions(itf):
        return tuple(torch.as_tensor(itf.seedIndices.T, device="cuda").long())

    @staticmethod
    def jvp(ctx, dcost, _):
        itf = ctx.itf
        cost = itf.cost.expand(itf.shape) if itf.cost.dim() == 0 else itf.cost
        rhs = dcost.detach().float() * cost
        rhs[EikonalValues._seed_positions(itf)] = 0.0  # seed values do not depend on the cost
        if getattr(itf, "walls", None) is not None:
            rhs[itf.walls.bool()] = 0.0
        if itf.flow_normalization is not None:  # drift models (_PostProcess.py:185)
            rhs = rhs * itf.flow_normalization
        return itf.forward_columns(rhs.contiguous()[..., None])[..., 0]

    @staticmethod
    def backward(ctx, grad):
        (cost,) = ctx.saved_tensors
        itf = ctx.itf
        lam = itf.reverse_columns(grad.detach().float().contiguous()[..., None])[..., 0]
        lam[EikonalValues._seed_positions(itf)] = 0.0
        if itf.flow_normalization is not None:  # drift models (_PostProcess.py:213-214)
            lam = lam / itf.flow_normalization
        return lam * cost, None


def eikonal_values(hfmIn, cost):
    """Values of the solve of hfmIn with the given cost, differentiable in cost."""
    return EikonalValues.apply(cost, hfmIn)
