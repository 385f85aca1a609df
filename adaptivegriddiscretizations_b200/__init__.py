"""B200-native GPU eikonal solver with the surface of agd.Eikonal.dictIn(...).Run().

Models Isotropic2/3, Diagonal2/3 and Riemann2/3; outputs values, flow,
geodesics, forward and reverse sensitivities; a standalone Selling
decomposition (Selling.Decomposition, Eikonal.VoronoiDecomposition).  The work is done by libagd_b200.so (CUDA for sm_100a) through
the C ABI declared in include/agd_b200.h; torch provides device memory and
streams.
"""
from . import Eikonal, Metrics, Selling

__all__ = ["Eikonal", "Metrics", "Selling"]
