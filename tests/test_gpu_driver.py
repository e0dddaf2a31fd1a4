"""The reference's time loop and restart, on the GPU, against the oracle.

* A drop-in restart from files in the reference's format: raw u, v, w, phi
  .dat files and no exact-resume sidecar.  The reference then starts with an
  Euler step and gumax = 1 (multi/main.f90:241-246, 290-292, 323-325;
  multi/readwrite.f90:218-317); the oracle, started from the same files, does
  the same.
* mhit36_b200.driver.run, the mirror of program main (multi/main.f90:3-987):
  input.inp, the input/*.dat start (inflow = inphi = 1), the initial dump, the
  loop with a dump every `dump` steps, and a restart from output/.
"""
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _params(**kw):
    from mhit36_b200.config import InputParams
    base = dict(dt=1e-3, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1)
    base.update(kw)
    return InputParams(**base)


def _oracle(n, p):
    from oracle import Oracle
    return Oracle(n, dt=p.dt, mu=p.mu, rho=p.rho, f1=p.f1, f2=p.f2, f3=p.f3, k0=p.k0, radius=p.radius,
                  sigma=p.sigma, epsr=p.epsr, lin_force=p.lin_force, k2_mode=p.k2_mode, grid_mode=p.grid_mode,
                  tanh_identity=p.tanh_identity, phi_floor=p.phi_floor, phase_field=1)


def _read(d, t, n):
    from mhit36_b200 import fields
    return tuple(fields.read_field(os.path.join(d, f"{name}_{t:08d}.dat"), n) for name in ("u", "v", "w", "phi"))


def _check(got, ref):
    errs = {name: rel_err(a, b) for name, a, b in zip(("u", "v", "w", "phi"), got, ref)}
    assert all(e <= TOL for e in errs.values()), errs


@pytest.mark.parametrize("n", [32, 64])
def test_reference_restart_without_sidecar(tmp_path, n):
    from mhit36_b200 import Solver, fields
    p = _params()
    case = fields.seeded_case(n, ndrops=2, rmin=0.6, rmax=0.8)
    with Solver(n, p) as a:
        a.set_fields(*case)
        a.step(3)
        a.save(str(tmp_path), 3)
    os.remove(os.path.join(str(tmp_path), "state_00000003.bin"))
    with Solver(n, p) as b:
        b.load(str(tmp_path), 3)
        d0 = b.diag()
        assert d0["step"] == 0 and d0["umax"] == 1.0  # gumax = 1 (multi/main.f90:325)
        d = b.step(4)
        got = b.get_fields()
    o = _oracle(n, p)
    o.set_fields(*_read(str(tmp_path), 3, n))
    rc, od = o.step(4)
    assert rc == 0
    _check(got, o.get_fields())
    assert abs(d["umax"] - od["umax"]) <= TOL * abs(od["umax"])
    # the first step after a reference restart is Euler: it differs from the
    # exact resume, which continues AB2
    with Solver(n, p) as c:
        c.set_fields(*case)
        c.step(7)
        cont = c.get_fields()
    assert rel_err(got[0], cont[0]) > 1e-9


def test_driver_loop_dumps_and_restarts(tmp_path):
    from mhit36_b200 import driver, fields
    from mhit36_b200.config import write_input
    n = 32
    run = str(tmp_path)
    os.makedirs(os.path.join(run, "input"))
    case = fields.seeded_case(n, ndrops=2, rmin=0.6, rmax=0.8)
    for name, a in zip(("u", "v", "w", "phi"), case):
        fields.write_field(os.path.join(run, "input", f"{name}.dat"), a)
    p = _params(restart=0, tstart=0, tfin=6, dump=3, inflow=1, inphi=1)
    write_input(os.path.join(run, "input.inp"), p)
    lines = []
    hist = driver.run(n, run, log=lines.append)
    assert len(hist) == 6 and all(h["rc"] == 0 for h in hist)
    assert any(ln.startswith("CFL (max among tasks)") for ln in lines)
    out = os.path.join(run, "output")
    for a, b in zip(_read(out, 0, n), case):  # initial dump (multi/main.f90:296-305)
        assert np.array_equal(a, b)
    o = _oracle(n, p)
    o.set_fields(*case)
    for t in (3, 6):
        o.step(3)
        _check(_read(out, t, n), o.get_fields())
    o.close()
    # restart from t = 3: with the exact-resume sidecar the run continues AB2
    # and reproduces the uninterrupted dump bit for bit
    ref6 = _read(out, 6, n)
    p2 = _params(restart=1, tstart=3, tfin=6, dump=3, inflow=1, inphi=1)
    write_input(os.path.join(run, "input.inp"), p2)
    driver.run(n, run, verbose=False)
    for a, b in zip(_read(out, 6, n), ref6):
        assert np.array_equal(a, b)
    # without the sidecar it restarts as the reference does (Euler, gumax = 1)
    os.remove(os.path.join(out, "state_00000003.bin"))
    driver.run(n, run, verbose=False)
    o = _oracle(n, p2)
    o.set_fields(*_read(out, 3, n))
    o.step(3)
    _check(_read(out, 6, n), o.get_fields())
