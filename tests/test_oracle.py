"""CPU tests of the oracle itself, pinned to the reference's own data.

The reference has no unit tests; its validation is the Taylor-Green
dissipation series in val/ (README:95-101), which tests/golden holds.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_err


def test_fft_matches_numpy(oracle_mod):
    rng = np.random.default_rng(0)
    for n in (8, 12, 16, 32, 48, 64, 96, 128, 192, 256, 384, 512, 768, 1024):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        ref = np.fft.fft(x)
        assert rel_err(oracle_mod.fft1d(x, -1), ref) < 1e-14
        assert rel_err(oracle_mod.fft1d(x, +1), np.fft.ifft(x) * n) < 1e-14


def test_poisson_manufactured_consistent_grid(oracle_mod):
    # p = sin(x)cos(2y)sin(3z): lap p = -14 p (commented hook, multi/main.f90:739-741)
    n = 32
    o = oracle_mod.Oracle(n, grid_mode=1, phase_field=0)
    x = np.arange(n) * (2 * np.pi / n)
    p = np.sin(x)[:, None, None] * np.cos(2 * x)[None, :, None] * np.sin(3 * x)[None, None, :]
    got = o.poisson(-14.0 * p)
    assert np.max(np.abs(got - p)) < 1e-13


def test_poisson_zero_mean_and_spectral_symbol(oracle_mod):
    n = 16
    o = oracle_mod.Oracle(n, phase_field=0)
    rng = np.random.default_rng(1)
    rhs = rng.standard_normal((n, n, n))
    got = o.poisson(rhs)
    # divide by -k^2 with k^2 spectral and the (0,0,0) mode zeroed
    k = np.fft.fftfreq(n, 1.0 / n)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    F = np.fft.fftn(rhs)
    k2[0, 0, 0] = 1.0
    F = -F / k2
    F[0, 0, 0] = 0.0
    ref = np.real(np.fft.ifftn(F))
    assert rel_err(got, ref) < 1e-13
    assert abs(got.mean()) < 1e-14


def test_val_t0_dissipation(oracle_mod):
    from mhit36_b200 import fields
    val = json.load(open(os.path.join(GOLDEN, "val_taylor_green.json")))
    for n in (128, 256):
        u, v, w = fields.taylor_green(n)
        e = oracle_mod.dissipation(u, v, w, 6.25e-4, pi_f32=True)
        ref = val["series"][f"cudec_{n}_ab"][0][1]
        assert abs(e / ref - 1) < 2e-12, (n, e, ref)
        # without the float32 pi of post/compute_diss/module.f90:5 it is off by ~5.6e-8
        e64 = oracle_mod.dissipation(u, v, w, 6.25e-4, pi_f32=False)
        assert abs(e64 / ref - 1) > 1e-8


def test_recorded_oracle_dynamics_match_val():
    """The oracle's Taylor-Green run (make_golden.py --oracle) against val/."""
    val = json.load(open(os.path.join(GOLDEN, "val_taylor_green.json")))["series"]
    rec = json.load(open(os.path.join(GOLDEN, "oracle_taylor_green_128.json")))["samples"]
    ab = dict((round(t, 6), e) for t, e in val["cudec_128_ab"])
    eu = dict((round(t, 6), e) for t, e in val["cudec_128_eulero"])
    for t, e in rec[1:]:
        assert abs(e / ab[round(t, 6)] - 1) < 1e-12
        assert abs(e / eu[round(t, 6)] - 1) > 1e-7  # Euler-only history is distinguishable


def test_oracle_short_run_invariants(oracle_mod):
    """Mean removal, signed Umax and conservation of the phi volume."""
    from mhit36_b200 import fields
    n = 32
    u, v, w, phi = fields.seeded_case(n, ndrops=2, rmin=0.6, rmax=0.8)
    o = oracle_mod.Oracle(n, dt=1e-3, mu=6e-3, lin_force=0.1, phase_field=1)
    o.set_fields(u, v, w, phi)
    vol0 = phi.sum()
    rc, d = o.step(5)
    assert rc == 0
    uu, vv, ww, pp = o.get_fields()
    for f in (uu, vv, ww):
        assert abs(f.mean()) < 1e-15
    assert d["umax"] == max(uu.max(), vv.max(), ww.max())
    assert abs(pp.sum() / vol0 - 1) < 1e-12
    assert pp.min() > -1e-3 and pp.max() < 1 + 1e-3


def test_oracle_cfl_stop(oracle_mod):
    from mhit36_b200 import fields
    n = 16
    u, v, w = fields.taylor_green(n)
    o = oracle_mod.Oracle(n, dt=1e-3, phase_field=0)
    o.set_fields(u, v, w)
    rc, d = o.step(3, cfl_limit=1e-6)
    assert rc == 1 and d["step"] == 1


def test_oracle_drop_count_rules(oracle_mod):
    """post/DropCountSize rules: threshold 0.5, 26-connectivity, periodic wrap, scan order."""
    n = 16
    phi = np.zeros((n, n, n))
    phi[2:5, 2:5, 2:5] = 1.0              # 27 cells, first in scan order
    phi[10, 10, 10] = phi[11, 11, 11] = 1  # corner contact only: one drop (26-connected)
    phi[15, 7, 7] = phi[0, 7, 7] = 0.5     # across the x boundary, exactly at the threshold
    phi[7, 0, 3] = 0.4999                  # below the threshold
    dx = 2 * np.pi / (n - 1)
    cells, deq = oracle_mod.drop_count(phi, dx)
    assert list(cells) == [27, 2, 2]
    assert np.allclose(deq, dx * (6 / np.pi * cells) ** (1 / 3), rtol=0, atol=1e-15)
