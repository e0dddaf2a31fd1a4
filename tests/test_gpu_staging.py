"""Plane staging of the stencil kernels on the GPU.

The phase and momentum kernels stage each z plane of their inputs in
shared-memory rings.  Tiles whose staged boxes lie inside the grid load a
plane with tensor-map box loads (cp.async.bulk.tensor) completed on a
shared-memory barrier; tiles at the periodic edges copy the same boxes
element-wise with cp.async and wrap, into the same cells.  Every grid from
96^3 up has both kinds of tile, so the step parity tests against the oracle
(tests/test_gpu_parity.py, tests/test_gpu_bench_workload.py) cover both; at
32^3 and 64^3 every tile is an edge tile.

This file tests the bounded barrier wait: with nothing arriving it gives up
after the given number of cycles and reports MHIT_ERR_TIMEOUT, the kernel
returns, and the CUDA context stays usable (a 96^3 step afterwards matches
the oracle).  The served ensemble's batched kernels copy element-wise on every tile;
tests/test_gpu_ensemble.py checks them bitwise against the solo handle at
grids with interior tiles.
"""
import ctypes

import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _params():
    from mhit36_b200.config import InputParams
    return InputParams(dt=1e-3, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1)


def test_bounded_wait_gives_up_and_context_survives():
    from mhit36_b200 import Solver, capi, fields
    from oracle import Oracle
    lib = capi.load_library()
    st = ctypes.c_int(-1)
    rc = lib.mhit_check_bounded_wait(0, 2_000_000, ctypes.byref(st))  # ~1 ms of SM cycles
    assert rc == capi.MHIT_OK, lib.mhit_strerror(rc)
    assert st.value == capi.MHIT_ERR_TIMEOUT
    rc = lib.mhit_check_bounded_wait(1, 2_000_000, ctypes.byref(st))
    assert rc == capi.MHIT_OK and st.value == capi.MHIT_OK
    assert lib.mhit_check_bounded_wait(0, 0, ctypes.byref(st)) == capi.MHIT_ERR_INVALID
    n, p = 96, _params()
    case = fields.seeded_case(n, ndrops=3, rmin=0.5, rmax=0.8)
    with Solver(n, p) as s:
        s.set_fields(*case)
        d = s.step(3)
        got = s.get_fields()
    assert d["status"] == capi.MHIT_OK
    o = Oracle(n, dt=p.dt, mu=p.mu, rho=p.rho, sigma=p.sigma, epsr=p.epsr, lin_force=p.lin_force, phase_field=1,
               tanh_identity=p.tanh_identity, phi_floor=p.phi_floor)
    o.set_fields(*case)
    rc, _ = o.step(3)
    assert rc == 0
    for a, b in zip(got, o.get_fields()):
        assert rel_err(a, b) <= 1e-12
    o.close()
