"""Eikonal solver interface: agd.Eikonal's dictIn/dictOut surface, GPU modes."""
from .DictIn import dictIn, dictOut, CenteredLinspace
from .HFM_CUDA import RunGPU, RunBatch, BatchPlan

__all__ = ["dictIn", "dictOut", "CenteredLinspace", "RunGPU", "RunBatch", "BatchPlan"]
