"""bowshock_b200: B200-native backend of the reference's axisymmetric finite-volume solver (MUSCL/HLLC residual with
viscous and SST terms, line-implicit block-tridiagonal sweeps), behind a C ABI (include/bowshock_b200.h) that mirrors
the reference's GPU solver interface. The CUDA library is built in-tree by `python -m bowshock_b200.build`."""
from .solver import (BC_CHARACTERISTIC, BC_EXTRAPOLATE, BC_FREESTREAM, BC_PRESSURE_OUTFLOW, BC_SLIPWALL, DT_MIN_DIRECTION,
                     DT_SUM, EXPLICIT, LIM_FIRST_ORDER, LIM_MINMOD, LIM_VAN_ALBADA, LIM_VENKATAKRISHNAN, TURB_LAMINAR,
                     TURB_SST, BowshockError, Config, GpuSolver, ImplicitParams, Viscous, freestream)

__all__ = ["GpuSolver", "Config", "ImplicitParams", "Viscous", "BowshockError", "EXPLICIT", "freestream"]
