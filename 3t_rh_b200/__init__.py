"""rh3t on B200: the 3T_RH semi-discrete operator l() and its SSP-RK3 driver
as FP64 CUDA kernels for sm_100a behind a C ABI (include/rh3t.h), with a host
mirror of the reference's Field / GhostGrid / BCType / rk3_ssp API."""
from .api import (FLUID_INSIDE, FLUID_OUTSIDE, INNER, OUTER, ArcOverride, BCType, CircularArc, Field, GhostGrid,
                  GridInfo, Params, Polygon, RH3TError, Solver, Batch, calc_global_dt, l, rk3_ssp)
from . import cases
from ._lib import lib_path, load

__all__ = ["ArcOverride", "BCType", "CircularArc", "Field", "GhostGrid", "GridInfo", "Params", "Polygon",
           "RH3TError", "Solver", "Batch", "calc_global_dt", "l", "rk3_ssp", "cases", "load", "lib_path", "FLUID_INSIDE",
           "FLUID_OUTSIDE", "OUTER", "INNER"]
