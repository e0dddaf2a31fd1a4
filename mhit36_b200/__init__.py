"""mhit36_b200: the MHIT36 timestep (NS + ACDI phase field) on one B200.

The compute is libmhit.so (hand-written sm_100a CUDA kernels behind the C ABI
of include/mhit.h); this package is its host-side mirror of the reference's
surface: input.inp parameters (config), raw .dat field files and the seeded
initial fields (fields), the timestep object (solver) and the main.f90 time
loop (driver).
"""
from .config import InputParams, read_input, write_input  # noqa: F401
from .capi import MhitError, load_library  # noqa: F401
from .solver import Solver  # noqa: F401

__all__ = ["InputParams", "read_input", "write_input", "MhitError", "load_library", "Solver"]
