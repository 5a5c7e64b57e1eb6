"""B200-native DSMC engine: a drop-in for the SolvikaAS/DSMC_erlend time step.

The physics runs in hand-written sm_100a kernels behind the C ABI of
include/dsmc.h (lib/libdsmc_b200.so); this package loads that library.
"""
from .abi import (FP32, FP64, WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Counters, Derived, Params,
                  default_params, large_case, reference_case, warm_start_case)
from .engine import Engine, setup, write_field

__all__ = [
    "Engine", "Params", "Derived", "Counters", "setup", "write_field", "default_params",
    "reference_case", "large_case", "warm_start_case", "FP32", "FP64", "WALL_CLL",
    "WALL_DIFFUSE", "WALL_SPECULAR",
]
