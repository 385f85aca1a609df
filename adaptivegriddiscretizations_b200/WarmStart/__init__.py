"""Learned warm start of the Riemann2 eikonal solver (no counterpart in the
reference, which has no learned component).

`UNet` (unet.py) predicts r = log(T / dref), the log-ratio of the 4x4-block
mean arrival time T to the distance scale dref (distance to the nearest seed
plus two grid steps), from block features of the metric and the seeds; every
layer runs on the tensor cores or in memory-bound kernels of libagd_b200
(include/agd_warmstart.h).  `WarmStart` (warmstart.py) generates training
data with the solver itself, trains the network on the GPU and turns its
predictions into per-tile release epochs and warm-start values for batched
solves, with the cold solve as the check and fallback.
"""
from .unet import UNet  # noqa: F401

__all__ = ["UNet"]
