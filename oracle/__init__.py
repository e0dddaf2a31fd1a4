"""CPU oracle for the MHIT36 timestep -- TEST INFRASTRUCTURE ONLY.

The oracle is a C++/OpenMP restatement of the reference step
(aroccon/MHIT36 multi/main.f90:329-977) in FP64 on the reference's halo'd
(nx, ny+2, nz+2) layout, built from ``oracle/mhit_oracle.cpp`` by
``oracle/Makefile`` into ``oracle/_build/libmhit_oracle.so``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference legs may import this package, and only as the checker / the timed
CPU stand-in for the reference.  The product library (``mhit36_b200``) never
imports, links or calls it.
"""
from .oracle import Oracle, OracleParams, build_oracle, dissipation, drop_count, fft1d, lib_path  # noqa: F401
