"""GPU post-processing against the oracle: drop count and sizes
(post/DropCountSize) and the FP64 diagnostics after real steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _params(**kw):
    from mhit36_b200.config import InputParams
    base = dict(dt=1e-3, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1)
    base.update(kw)
    return InputParams(**base)


@pytest.mark.parametrize("n,steps", [(128, 0), (128, 20), (64, 5)])
def test_drop_count_matches_oracle(n, steps):
    from oracle import drop_count
    from mhit36_b200 import Solver, fields
    u, v, w, phi = fields.seeded_case(n) if n == 128 else fields.seeded_case(n, ndrops=5, rmin=0.4, rmax=0.6)
    with Solver(n, _params()) as s:
        s.set_fields(u, v, w, phi)
        if steps:
            s.step(steps)
        cells, deq = s.drops()
        cur = s.get_fields()[3]
    ref_cells, ref_deq = drop_count(cur, 2 * np.pi / (n - 1))
    assert np.array_equal(cells, ref_cells)
    assert np.allclose(deq, ref_deq, rtol=1e-15, atol=0)
    if n == 128 and steps == 0:
        assert len(cells) == 8  # the 128^3 recipe's 8 drops


def test_drop_count_periodic_and_corner_cases():
    from oracle import drop_count
    from mhit36_b200 import Solver
    n = 32
    phi = np.zeros((n, n, n))
    phi[30:32, 5:8, 5:8] = 1.0
    phi[0:2, 5:8, 5:8] = 1.0            # joins the previous across x = 0
    phi[10, 10, 31] = phi[11, 11, 0] = 1  # corner contact across z
    phi[20:23, 20:23, 20:23] = 0.6
    z = np.zeros((n, n, n))
    with Solver(n, _params()) as s:
        s.set_fields(z, z, z, phi)
        cells, _ = s.drops()
    ref, _ = drop_count(phi, 2 * np.pi / (n - 1))
    assert list(cells) == list(ref) and len(cells) == 3
