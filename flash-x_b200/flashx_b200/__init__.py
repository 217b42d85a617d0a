"""flashx_b200: B200-native drop-in for the Flash-X unsplit-hydro hot path.

The compute path is the C-ABI library libflashx_b200.so (CUDA kernels for
sm_100a behind extern "C" entry points declared in include/flashx_b200.h).
This package is the host-side mirror of the reference's Fortran interface
(Hydro, Hydro_computeDt, Grid_fillGuardCells) plus parameter and
initial-condition helpers.
"""
from .params import HydroParams, Geometry, UNK_VARS, NUNK  # noqa: F401
