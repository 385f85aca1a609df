"""Eikonal solver interface: agd.Eikonal's dictIn/dictOut surface, GPU modes."""
from .DictIn import dictIn, dictOut, CenteredLinspace
from .HFM_CUDA import RunGPU, RunBatch, SubmitBatch, BatchJob, BatchPlan
from .BatchSolver import BatchSolver, SolverJob
from .Voronoi import VoronoiDecomposition

__all__ = ["dictIn", "dictOut", "CenteredLinspace", "RunGPU", "RunBatch", "SubmitBatch", "BatchJob", "BatchPlan",
           "BatchSolver", "SolverJob", "VoronoiDecomposition"]
