"""Differentiable eikonal solve: arrival times as a function of the cost field.

`EikonalValues.apply(cost, hfmIn)` returns the values of the eikonal solve of
hfmIn with its 'cost' replaced by `cost` (a CUDA tensor of the grid shape).
The backward pass runs the reverse-mode adjoint of libagd_b200 (agd_reverse)
with the incoming gradient as the 'sensitivity' right-hand side.  The adjoint
unknown lam satisfies dJ/dcost = lam * cost (the forward linearisation of the
scheme uses the right-hand side cost * dcost, agd/Eikonal/HFM_CUDA/_PostProcess.py:181-183),
and the reference reports lam itself as 'costSensitivity'.  Forward mode
(torch.autograd.forward_ad) runs agd_forward with the tangent as 'costVariation'.
"""
import torch

from .Eikonal.HFM_CUDA import Interface


class EikonalValues(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cost, hfmIn):
        h = hfmIn.copy()
        h["cost"] = cost.detach()
        h["exportValues"] = True
        h.store.pop("sensitivity", None)
        h.store.pop("tips", None)
        itf = Interface(h)
        itf.SetKernelTraits()
        itf.SetGeometry()
        itf.SetArgs()
        itf.Solve()
        values = itf.values.clone()
        ctx.hfmIn = h
        ctx.save_for_backward(cost)
        return values

    @staticmethod
    def jvp(ctx, dcost, _):
        h = ctx.hfmIn.copy()
        h["costVariation"] = dcost.detach().float().contiguous()[..., None]
        out = h.Run()
        return out["valueVariation"][..., 0]

    @staticmethod
    def backward(ctx, grad):
        (cost,) = ctx.saved_tensors
        h = ctx.hfmIn.copy()
        h["sensitivity"] = grad.detach().float().contiguous()[..., None]
        out = h.Run()
        lam = out["costSensitivity"][..., 0]
        return lam * cost, None


def eikonal_values(hfmIn, cost):
    """Values of the solve of hfmIn with the given cost, differentiable in cost."""
    return EikonalValues.apply(cost, hfmIn)
