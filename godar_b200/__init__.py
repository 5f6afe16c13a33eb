"""godar_b200: a B200 (sm_100a) implementation of GODAR's per-time-step DEM
loop (the reference's `stepper`, model/src/stepper.f90) behind a C ABI
(include/godar_gpu.h).

- params      namelist/derived parameters (ctypes mirror of godar_params)
- lib         Stepper (one field) and Batch (many fields) over libgodar_gpu.so
- generators  seeded synthetic floe fields of the benchmark configurations
- serve       continuous-batching request loop with HBM-budget admission
- build       in-tree build of the CUDA library (sm_100a)
"""
from .params import (GodarParams, default_params, make_params, derive, read_namelist,
                     PREC_FP64, PREC_MIXED, BC_PERIODIC_X, BC_PERIODIC_Y, BC_OPEN_LEFT,
                     BC_OPEN_RIGHT, BC_OPEN_BOTTOM, BC_OPEN_TOP)

__all__ = ["GodarParams", "default_params", "make_params", "derive", "read_namelist",
           "PREC_FP64", "PREC_MIXED", "BC_PERIODIC_X", "BC_PERIODIC_Y", "BC_OPEN_LEFT",
           "BC_OPEN_RIGHT", "BC_OPEN_BOTTOM", "BC_OPEN_TOP"]
