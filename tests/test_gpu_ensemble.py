"""GPU tests of the served ensemble (continuous batching of independent
simulations).  Each request's result must be the same alone and in any mix:
the batched kernels run exactly the single-simulation arithmetic per slot,
so the bar here is bitwise equality with the plain Solver."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(**kw):
    from mhit36_b200.config import InputParams
    base = dict(dt=1e-3, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1)
    base.update(kw)
    return InputParams(**base)


def _case(n, pf, seed):
    from mhit36_b200 import fields
    u, v, w = fields.random_velocity(n, seed)
    phi = None
    if pf:
        c, r = fields.place_drops(n, seed + 1, 2, 0.5, 0.7)
        phi = fields.drop_field(n, c, r)
    return u, v, w, phi


def _solo(n, p, case, steps, precision="fp64"):
    from mhit36_b200 import Solver
    with Solver(n, p, precision=precision, phase_field=case[3] is not None) as s:
        s.set_fields(*case)
        s.step(steps, raise_on_error=False)
        return s.get_fields()


def _same(a, b):
    for x, y in zip(a, b):
        if x is None:
            assert y is None
            continue
        assert np.array_equal(x, y), float(np.max(np.abs(x - y)))


REQS = [(32, True, 7, 6e-3), (64, False, 5, 3e-3), (32, True, 9, 1e-2), (32, False, 4, 5e-3), (64, True, 3, 8e-3)]


def test_mix_matches_solo_solver_bitwise():
    from mhit36_b200.ensemble import Ensemble
    cases = [_case(n, pf, 100 + i) for i, (n, pf, _, _) in enumerate(REQS)]
    with Ensemble(slots_per_class=4) as ens:
        ids = [ens.submit(n, _params(mu=mu), *cases[i], nsteps=st) for i, (n, pf, st, mu) in enumerate(REQS)]
        ens.run()
        for i, (n, pf, st, mu) in enumerate(REQS):
            q = ens.query(ids[i])
            assert q["state"] == "done" and q["diag"]["step"] == st
            _same(ens.result(ids[i]), _solo(n, _params(mu=mu), cases[i], st))


def test_continuous_admission_with_few_slots():
    """More requests than slots: later ones are admitted as earlier ones
    retire, while the class keeps running."""
    from mhit36_b200.ensemble import Ensemble
    case = _case(32, True, 7)
    with Ensemble(slots_per_class=2) as ens:
        ids = [ens.submit(32, _params(), *case, nsteps=3 + i) for i in range(5)]
        ens.progress()
        states = [ens.query(i)["state"] for i in ids]
        assert states.count("running") == 2 and states.count("queued") == 3
        # a request arriving while others run joins without a re-capture
        late = ens.submit(32, _params(), *case, nsteps=2)
        ens.run()
        infos = [ens.query(i) for i in ids + [late]]
        assert all(q["state"] == "done" for q in infos)
        ref = _solo(32, _params(), case, 2)
        _same(ens.result(late), ref)
        admits = [q["t_admit"] for q in infos[:5]]
        assert admits[2] >= min(admits[:2])


def test_fused_projection_class_matches_solver_bitwise():
    """From 256^3 the FP64 step fuses the x inverse into the projection, in
    the batched class graph as in the plain Solver; two requests of one
    class (one with ACDI) must still match their solo runs bit for bit."""
    from mhit36_b200.ensemble import Ensemble
    cases = [_case(256, True, 21), _case(256, False, 22)]
    with Ensemble(slots_per_class=2) as ens:
        a = ens.submit(256, _params(dt=2e-4), *cases[0], nsteps=3)
        b = ens.submit(256, _params(dt=2e-4, mu=3e-3), *cases[1], nsteps=2)
        ens.run()
        assert ens.query(a)["state"] == "done" and ens.query(b)["state"] == "done"
        _same(ens.result(a), _solo(256, _params(dt=2e-4), cases[0], 3))
        _same(ens.result(b), _solo(256, _params(dt=2e-4, mu=3e-3), cases[1], 2))


def test_fp32_form_in_ensemble_matches_solver():
    from mhit36_b200.ensemble import Ensemble
    p = _params(k2_mode=1)
    cases = [_case(32, True, 11), _case(64, False, 12)]
    with Ensemble() as ens:
        a = ens.submit(32, p, *cases[0], nsteps=6, precision="fp32")
        b = ens.submit(64, p, *cases[1], nsteps=4, precision="fp32")
        ens.run()
        q = ens.query(a)
        assert q["diag"]["max_div"] <= 1e-10
        _same(ens.result(a), _solo(32, p, cases[0], 6, "fp32"))
        _same(ens.result(b), _solo(64, p, cases[1], 4, "fp32"))


def test_hbm_budget_admission():
    """A budget that fits one 64^3 slot serialises the requests, which still all finish."""
    from mhit36_b200.ensemble import Ensemble
    case = _case(64, False, 3)
    budget = int(1.5 * 64 ** 3 * 8 * 11.5)
    with Ensemble(budget_bytes=budget) as ens:
        ids = [ens.submit(64, _params(), *case, nsteps=2) for _ in range(3)]
        ens.progress()
        assert [ens.query(i)["state"] for i in ids].count("running") == 1
        ens.run()
        assert all(ens.query(i)["state"] == "done" for i in ids)
        assert ens.stats()["bytes_used"] <= budget


def test_failed_request_is_isolated():
    from mhit36_b200.ensemble import Ensemble
    from mhit36_b200.capi import MHIT_ERR_NONFINITE
    good = _case(32, False, 5)
    bad = tuple(x.copy() if x is not None else None for x in good)
    bad[0][1, 2, 3] = np.nan
    with Ensemble() as ens:
        a = ens.submit(32, _params(), *bad, nsteps=4)
        b = ens.submit(32, _params(), *good, nsteps=4)
        ens.run()
        qa, qb = ens.query(a), ens.query(b)
        assert qa["state"] == "failed" and qa["status"] == MHIT_ERR_NONFINITE
        assert qb["state"] == "done"
        _same(ens.result(b), _solo(32, _params(), good, 4))


def test_cancel():
    from mhit36_b200.ensemble import Ensemble
    case = _case(32, False, 9)
    with Ensemble(slots_per_class=1) as ens:
        a = ens.submit(32, _params(), *case, nsteps=50)
        b = ens.submit(32, _params(), *case, nsteps=50)
        ens.progress()
        ens.cancel(b)  # queued
        ens.cancel(a)  # running
        assert ens.query(a)["state"] == "cancelled" and ens.query(b)["state"] == "cancelled"
        c = ens.submit(32, _params(), *case, nsteps=3)
        ens.run()
        _same(ens.result(c), _solo(32, _params(), case, 3))


def test_fp32_fused_projection_class_matches_solver_bitwise():
    """From 256^3 the FP32 refinement form fuses the correction solve's x
    inverse into the projection, batched as in the plain Solver."""
    from mhit36_b200.ensemble import Ensemble
    p = _params(dt=2e-4, k2_mode=1)
    case = _case(256, True, 31)
    with Ensemble(slots_per_class=2) as ens:
        a = ens.submit(256, p, *case, nsteps=3, precision="fp32")
        ens.run()
        assert ens.query(a)["state"] == "done"
        _same(ens.result(a), _solo(256, p, case, 3, "fp32"))
