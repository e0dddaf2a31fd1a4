"""The benchmarked configuration against the oracle.

bench.py's own workload -- 512^3 NS+ACDI, 64 seeded drops of radius
0.2-0.35, the seeded random-phase velocity, dt = 2e-4, linear forcing 0.1 --
run for 3 steps through the C ABI and through the oracle (the step of
multi/main.f90:329-977).  From 512^3 up the stencil kernels march 64-plane z
chunks, the column passes run the radix 8*8*8 plan and the x inverse fused
into the projection runs its 16-plane configuration; no smaller test reaches
those kernel configurations.  Bar: max|gpu - oracle| / max|oracle| <= 1e-12
per field, and the same for Umax and CFL.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_bench_workload_512_3_steps():
    import bench
    from mhit36_b200 import Solver
    from oracle import Oracle
    n, steps = 512, 3
    p, case, recipe = bench.workload(n, True, 2e-4)
    assert recipe == (64, 0.2, 0.35)
    with Solver(n, p, phase_field=True) as s:
        s.set_fields(*case)
        d = s.step(steps)
        got = s.get_fields()
        pgot = s.get_pressure()
    assert d["status"] == 0 and d["step"] == steps
    o = Oracle(n, dt=p.dt, mu=p.mu, rho=p.rho, f1=p.f1, f2=p.f2, f3=p.f3, k0=p.k0, sigma=p.sigma, epsr=p.epsr,
               lin_force=p.lin_force, k2_mode=p.k2_mode, grid_mode=p.grid_mode, tanh_identity=p.tanh_identity,
               phi_floor=p.phi_floor, phase_field=1)
    o.set_fields(*case)
    del case
    rc, od = o.step(steps)
    assert rc == 0
    ref = o.get_fields()
    pref = o.get_pressure()
    o.close()
    errs = {name: rel_err(a, b) for name, a, b in zip(("u", "v", "w", "phi"), got, ref)}
    errs["p"] = rel_err(pgot, pref)
    errs["umax"] = abs(d["umax"] - od["umax"]) / abs(od["umax"])
    errs["cfl"] = abs(d["cfl"] - od["cfl"]) / abs(od["cfl"])
    print("512^3 bench workload, 3 steps, relative errors:", errs)
    assert all(errs[k] <= TOL for k in ("u", "v", "w", "phi", "umax", "cfl")), errs
    assert errs["p"] <= 1e-11, errs
    assert np.isfinite(got[3]).all()
