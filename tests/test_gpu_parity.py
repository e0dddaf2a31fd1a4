"""GPU parity of the CUDA step (through the C ABI) against the CPU oracle.

Bar (plain FP64 form): max|gpu - oracle| / max|oracle| <= 1e-12 per field
after 10 steps on the same seeded inputs.  The two differ only in rounding:
the FFT algorithm (own shared-memory radix-8/4/2/3 Stockham real-to-complex
vs the oracle's full complex transform), FMA contraction, and reduction order.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _params(**kw):
    from mhit36_b200.config import InputParams
    base = dict(dt=1e-3, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1)
    base.update(kw)
    return InputParams(**base)


def _oracle_kw(p):
    return dict(dt=p.dt, mu=p.mu, rho=p.rho, f1=p.f1, f2=p.f2, f3=p.f3, k0=p.k0, radius=p.radius,
                sigma=p.sigma, epsr=p.epsr, lin_force=p.lin_force, k2_mode=p.k2_mode, grid_mode=p.grid_mode,
                tanh_identity=p.tanh_identity, phi_floor=p.phi_floor)


def _case(n, pf, ndrops=None, rmin=None, rmax=None, grid_mode=0):
    from mhit36_b200 import fields
    return fields.seeded_case(n, phase_field=pf, ndrops=ndrops, rmin=rmin, rmax=rmax, grid_mode=grid_mode)


def run_pair(n, steps, pf, p, case=None, oracle_p=None):
    from oracle import Oracle
    from mhit36_b200 import Solver
    u, v, w, phi = case if case is not None else _case(n, pf, grid_mode=p.grid_mode)
    o = Oracle(n, phase_field=int(pf), **_oracle_kw(oracle_p or p))
    o.set_fields(u, v, w, phi)
    rc, od = o.step(steps)
    assert rc == 0
    ref = o.get_fields()
    with Solver(n, p, phase_field=pf) as s:
        s.set_fields(u, v, w, phi)
        d = s.step(steps)
        got = s.get_fields()
        pres = s.get_pressure()
    return ref, got, od, d, o.get_pressure(), pres


def _check(ref, got, pf, tol=TOL):
    errs = {}
    for name, a, b in zip("uvw", got[:3], ref[:3]):
        errs[name] = rel_err(a, b)
    if pf:
        errs["phi"] = rel_err(got[3], ref[3])
    assert all(e <= tol for e in errs.values()), errs
    return errs


@pytest.mark.parametrize("n", [32, 64])
def test_ns_only_10_steps(n):
    p = _params()
    ref, got, od, d, pref, pgot = run_pair(n, 10, False, p)
    _check(ref, got, False)
    assert rel_err(pgot, pref) <= 1e-11
    assert abs(d["umax"] - od["umax"]) <= 1e-12 * abs(od["umax"])
    assert abs(d["cfl"] - od["cfl"]) <= 1e-12 * abs(od["cfl"])
    assert d["step"] == 10 and d["status"] == 0


def test_ns_acdi_64_10_steps():
    p = _params()
    ref, got, od, d, _, _ = run_pair(64, 10, True, p, case=_case(64, True, ndrops=4, rmin=0.4, rmax=0.6))
    _check(ref, got, True)
    assert abs(d["umax"] - od["umax"]) <= 1e-12 * abs(od["umax"])


def test_ns_acdi_128_10_steps():
    """The 128^3 NS+ACDI configuration: 8 seeded drops of radius 0.4-0.6."""
    p = _params()
    ref, got, od, d, _, _ = run_pair(128, 10, True, p)
    _check(ref, got, True)


@pytest.mark.parametrize("n", [64, 128])
def test_default_fast_path_vs_exact_reference_formula(n):
    """The default ACDI evaluation (tanh(psi/2eps) as (2phi-1)/(1+2enum), phi
    floored at 0 inside the log) against the oracle running the reference's
    exact formulas (FP64 tanh, min(phi,1) only; multi/main.f90:388-389, 463-465)."""
    p = _params()
    exact = _params(tanh_identity=0, phi_floor=0)
    case = _case(n, True, ndrops=4, rmin=0.4, rmax=0.6) if n == 64 else None
    ref, got, _, _, _, _ = run_pair(n, 10, True, p, case=case, oracle_p=exact)
    _check(ref, got, True)


@pytest.mark.parametrize("opt", ["abc", "k2fd", "consistent", "exact_tanh", "no_lin"])
def test_options_32(opt):
    kw = {"abc": dict(f1=0.3, f2=0.2, f3=0.1, k0=2.0), "k2fd": dict(k2_mode=1),
          "consistent": dict(grid_mode=1), "exact_tanh": dict(tanh_identity=0, phi_floor=0),
          "no_lin": dict(lin_force=0.0)}[opt]
    p = _params(**kw)
    case = _case(32, True, ndrops=2, rmin=0.6, rmax=0.8, grid_mode=p.grid_mode)
    ref, got, _, _, _, _ = run_pair(32, 10, True, p, case=case)
    _check(ref, got, True)


def test_poisson_manufactured():
    """p = sin(x)cos(2y)sin(3z) on the consistent grid: lap p = -14 p."""
    from mhit36_b200 import Solver
    for n in (32, 64, 96):
        with Solver(n, _params(grid_mode=1), phase_field=False) as s:
            x = np.arange(n) * (2 * np.pi / n)
            p = np.sin(x)[:, None, None] * np.cos(2 * x)[None, :, None] * np.sin(3 * x)[None, None, :]
            got = s.poisson(-14.0 * p)
            assert np.max(np.abs(got - p)) < 1e-13, n


def test_poisson_vs_oracle_random_rhs():
    from oracle import Oracle
    from mhit36_b200 import Solver
    rng = np.random.default_rng(7)
    for n in (32, 64, 96, 192, 384):
        rhs = rng.standard_normal((n, n, n))
        o = Oracle(n, phase_field=0)
        ref = o.poisson(rhs)
        with Solver(n, _params(), phase_field=False) as s:
            got = s.poisson(rhs)
        assert rel_err(got, ref) < 1e-13, n


def test_taylor_green_val_series():
    """Against the reference's val/cudec_128_ab.txt (t = 0.2, 0.4)."""
    from oracle import dissipation
    from mhit36_b200 import Solver, fields
    from mhit36_b200.config import InputParams
    val = json.load(open(os.path.join(GOLDEN, "val_taylor_green.json")))["series"]["cudec_128_ab"]
    n = 128
    u, v, w = fields.taylor_green(n)
    p = InputParams(dt=2e-4, mu=6.25e-4, rho=1.0)
    with Solver(n, p, phase_field=False) as s:
        s.set_fields(u, v, w)
        for sample in (1, 2):
            s.step(1000)
            uu, vv, ww, _ = s.get_fields()
            e = dissipation(uu, vv, ww, 6.25e-4, pi_f32=True)
            assert abs(e / val[sample][1] - 1) < 1e-11, (sample, e, val[sample][1])


def test_save_load_exact_resume(tmp_path):
    from mhit36_b200 import Solver
    n = 32
    p = _params()
    u, v, w, phi = _case(n, True, ndrops=2, rmin=0.6, rmax=0.8)
    with Solver(n, p) as a:
        a.set_fields(u, v, w, phi)
        a.step(3)
        a.save(str(tmp_path), 3)
        a.step(4)
        ref = a.get_fields()
    with Solver(n, p) as b:
        b.load(str(tmp_path), 3)
        assert b.diag()["step"] == 3
        b.step(4)
        got = b.get_fields()
    for x, y in zip(ref, got):
        assert np.array_equal(x, y)
    # the saved fields are the reference's raw format
    from mhit36_b200 import fields
    raw = fields.read_field(os.path.join(str(tmp_path), "u_00000003.dat"), n)
    assert raw.shape == (n, n, n)


def test_determinism_bitwise():
    from mhit36_b200 import Solver
    n = 64
    case = _case(n, True, ndrops=4, rmin=0.4, rmax=0.6)
    outs = []
    for _ in range(2):
        with Solver(n, _params()) as s:
            s.set_fields(*case)
            s.step(5)
            outs.append(s.get_fields())
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


def test_cfl_guard_stops_and_freezes():
    from mhit36_b200 import Solver, MhitError
    from mhit36_b200.capi import MHIT_ERR_CFL
    n = 32
    p = _params(cfl_limit=1e-6)
    u, v, w, _ = _case(n, False)
    with Solver(n, p, phase_field=False) as s:
        s.set_fields(u, v, w)
        d = s.step(5, raise_on_error=False)
        assert d["rc"] == MHIT_ERR_CFL and d["step"] == 1
        after1 = s.get_fields()
        d2 = s.step(2, raise_on_error=False)
        assert d2["rc"] == MHIT_ERR_CFL and d2["step"] == 1
        for x, y in zip(after1[:3], s.get_fields()[:3]):
            assert np.array_equal(x, y)
        with pytest.raises(MhitError):
            s.step(1)


def test_nonfinite_detected():
    from mhit36_b200 import Solver
    from mhit36_b200.capi import MHIT_ERR_NONFINITE
    n = 32
    u, v, w, _ = _case(n, False)
    u = u.copy()
    u[3, 4, 5] = np.nan
    with Solver(n, _params(), phase_field=False) as s:
        s.set_fields(u, v, w)
        d = s.step(3, raise_on_error=False)
        assert d["rc"] == MHIT_ERR_NONFINITE and d["step"] == 1


def test_phi_volume_conserved_and_bounded():
    from mhit36_b200 import Solver
    n = 64
    case = _case(n, True, ndrops=4, rmin=0.4, rmax=0.6)
    with Solver(n, _params()) as s:
        s.set_fields(*case)
        s.step(50)
        phi = s.get_fields()[3]
    assert abs(phi.sum() / case[3].sum() - 1) < 1e-11
    assert phi.min() > -0.05 and phi.max() < 1.05


def test_ns_acdi_256_10_steps_every_tile_shape():
    """256^3 NS+ACDI (8 drops) for 10 steps against the oracle: exercises the
    8x8x4 radix plan and the x inverse fused into the projection, whose
    pressure is recomputed from the last step's spectrum on request.  The GPU
    runs the default tiles and every (z chunk, momentum tile height) the
    ensemble's autotuner may pick, each against the same oracle run."""
    from oracle import Oracle
    from mhit36_b200 import Solver
    n, steps = 256, 10
    p = _params(dt=5e-4)  # inside the explicit ACDI diffusion limit Umax*dt/dx < 1/6
    case = _case(n, True)
    o = Oracle(n, phase_field=1, **_oracle_kw(p))
    o.set_fields(*case)
    rc, od = o.step(steps)
    assert rc == 0
    ref = o.get_fields()
    pref = o.get_pressure()
    o.close()
    for kz, mty in [(0, 0), (64, 8), (32, 16), (16, 8), (16, 16), (8, 8), (8, 16)]:
        with Solver(n, p, phase_field=True) as s:
            s.set_tiles(kz, mty)
            s.set_fields(*case)
            d = s.step(steps)
            got = s.get_fields()
            pgot = s.get_pressure()
        errs = _check(ref, got, True)
        assert rel_err(pgot, pref) <= 1e-11, (kz, mty)
        assert abs(d["umax"] - od["umax"]) <= 1e-12 * abs(od["umax"]), (kz, mty, errs)
        assert abs(d["cfl"] - od["cfl"]) <= 1e-12 * abs(od["cfl"]), (kz, mty)


@pytest.mark.parametrize("n", [256, 384, 512, 768])
def test_poisson_manufactured_large(n):
    """sin(x)cos(2y)sin(3z) at 256^3, 384^3, 512^3 and 768^3 (radix plans
    8x8x4, 4x4x4x2x3 with 12 elements per thread, 8x8x8, 4x4x4x4x3)."""
    from mhit36_b200 import Solver
    with Solver(n, _params(grid_mode=1), phase_field=False) as s:
        x = np.arange(n) * (2 * np.pi / n)
        p = np.sin(x)[:, None, None] * np.cos(2 * x)[None, :, None] * np.sin(3 * x)[None, None, :]
        got = s.poisson(-14.0 * p)
    assert np.max(np.abs(got - p)) < 1e-12


@pytest.mark.parametrize("n,pf,steps", [(96, True, 5), (192, False, 3)])
def test_mixed_radix_sizes_vs_oracle(n, pf, steps):
    """Sizes whose FFT plans use radix 3 (96 = 8*4*3, 192 = 8*8*3)."""
    p = _params()
    case = _case(n, True, ndrops=4, rmin=0.4, rmax=0.6) if pf else None
    ref, got, _, _, _, _ = run_pair(n, steps, pf, p, case=case)
    _check(ref, got, pf)


@pytest.mark.parametrize("n", [32, 64, 96, 128, 192])
def test_fp32_refinement_converges_at_every_size(n):
    """max|div u| of the FP32 form's FP64 projection <= 1e-10 at each built size
    up to 192^3 (each size has its own FFT chunking and x-pass configuration)."""
    from mhit36_b200 import Solver, fields
    p = _params(k2_mode=1)
    u, v, w = fields.random_velocity(n, 11)
    c, r = fields.place_drops(n, 12, 2, 0.4, 0.6)
    with Solver(n, p, precision="fp32", phase_field=True) as s:
        s.set_fields(u, v, w, fields.drop_field(n, c, r))
        d = s.step(4)
    assert d["max_div"] <= 1e-10, d["max_div"]
