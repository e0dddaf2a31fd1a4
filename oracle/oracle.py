"""ctypes binding of the CPU oracle (test infrastructure only).

See ``oracle/mhit_oracle.cpp`` for the restated reference stages and the
file:line citations into aroccon/MHIT36.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(_HERE, "_build", "libmhit_oracle.so")


class OracleParams(ctypes.Structure):
    """input.inp lines 7-16 (multi/readinput.f90:19-31) plus extensions."""

    _fields_ = [
        ("dt", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("rho", ctypes.c_double),
        ("f1", ctypes.c_double),
        ("f2", ctypes.c_double),
        ("f3", ctypes.c_double),
        ("k0", ctypes.c_double),
        ("radius", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("epsr", ctypes.c_double),
        ("lin_force", ctypes.c_double),
        ("k2_mode", ctypes.c_int),
        ("grid_mode", ctypes.c_int),
        ("phase_field", ctypes.c_int),
        ("tanh_identity", ctypes.c_int),
        ("phi_floor", ctypes.c_int),
    ]


class OracleDiag(ctypes.Structure):
    _fields_ = [
        ("umax", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("umean", ctypes.c_double),
        ("vmean", ctypes.c_double),
        ("wmean", ctypes.c_double),
        ("step", ctypes.c_int),
    ]


def build_oracle(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O3 -fopenmp)."""
    src = os.path.join(_HERE, "mhit_oracle.cpp")
    if force or not os.path.exists(lib_path) or os.path.getmtime(lib_path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return lib_path


_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(lib_path):
            build_oracle()
        lib = ctypes.CDLL(lib_path)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.oracle_create.restype = ctypes.c_void_p
        lib.oracle_create.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int]
        lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_set_threads.argtypes = [ctypes.c_int]
        lib.oracle_set_threads.restype = ctypes.c_int
        lib.oracle_set_fields.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        lib.oracle_get_fields.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        lib.oracle_get_pressure.argtypes = [ctypes.c_void_p, dp]
        lib.oracle_get_state.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp]
        lib.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(OracleDiag)]
        lib.oracle_step.restype = ctypes.c_int
        lib.oracle_poisson.argtypes = [ctypes.c_void_p, dp, dp]
        lib.oracle_fft1d.argtypes = [ctypes.c_int, dp, ctypes.c_int]
        lib.oracle_dissipation.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_int]
        lib.oracle_dissipation.restype = ctypes.c_double
        lib.oracle_drop_count.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_void_p, dp, ctypes.c_double]
        lib.oracle_drop_count.restype = ctypes.c_int
        _lib = lib
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _raw(a, n):
    """Accept an (n,n,n) array indexed [i,j,k] (x fastest in memory) or flat."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 3:
        a = np.asfortranarray(a).ravel(order="F")
    assert a.size == n ** 3
    return np.ascontiguousarray(a)


class Oracle:
    """One oracle simulation of size n^3.  Arrays are indexed a[i, j, k]."""

    def __init__(self, n: int, dt=1e-3, mu=6e-3, rho=1.0, f1=0.0, f2=0.0, f3=0.0, k0=2.0,
                 radius=0.5, sigma=0.5, epsr=1.0, lin_force=0.0, k2_mode=0, grid_mode=0,
                 phase_field=1, tanh_identity=0, phi_floor=0, threads: int = 0):
        self.lib = _load()
        if threads:
            self.lib.oracle_set_threads(threads)
        self.n = n
        self.params = OracleParams(dt, mu, rho, f1, f2, f3, k0, radius, sigma, epsr, lin_force,
                                   k2_mode, grid_mode, phase_field, tanh_identity, phi_floor)
        self.h = self.lib.oracle_create(ctypes.byref(self.params), n)
        if not self.h:
            raise ValueError(f"oracle_create failed for n={n}")

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, u, v, w, phi=None):
        n = self.n
        self._keep = [_raw(u, n), _raw(v, n), _raw(w, n), None if phi is None else _raw(phi, n)]
        self.lib.oracle_set_fields(self.h, *[_ptr(a) for a in self._keep])

    def _out(self):
        return np.empty(self.n ** 3, dtype=np.float64)

    @staticmethod
    def _shape(a, n):
        return a.reshape((n, n, n), order="F")

    def get_fields(self):
        n = self.n
        u, v, w, phi = self._out(), self._out(), self._out(), self._out()
        self.lib.oracle_get_fields(self.h, _ptr(u), _ptr(v), _ptr(w), _ptr(phi))
        return tuple(self._shape(a, n) for a in (u, v, w, phi))

    def get_pressure(self):
        p = self._out()
        self.lib.oracle_get_pressure(self.h, _ptr(p))
        return self._shape(p, self.n)

    def get_state(self):
        outs = [self._out() for _ in range(6)]
        self.lib.oracle_get_state(self.h, *[_ptr(a) for a in outs])
        return tuple(self._shape(a, self.n) for a in outs)

    def step(self, nsteps: int = 1, cfl_limit: float = 7.0):
        d = OracleDiag()
        rc = self.lib.oracle_step(self.h, nsteps, cfl_limit, ctypes.byref(d))
        return rc, {"umax": d.umax, "cfl": d.cfl, "umean": d.umean, "vmean": d.vmean,
                    "wmean": d.wmean, "step": d.step}

    def poisson(self, rhs):
        r = _raw(rhs, self.n)
        p = self._out()
        self.lib.oracle_poisson(self.h, _ptr(r), _ptr(p))
        return self._shape(p, self.n)


def fft1d(x: np.ndarray, sign: int = -1) -> np.ndarray:
    lib = _load()
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib.oracle_fft1d(a.size, a.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), sign)
    return a


def dissipation(u, v, w, nu: float, pi_f32: bool = True) -> float:
    """post/compute_diss/main.f90:72-117 on raw fields indexed [i,j,k]."""
    lib = _load()
    n = u.shape[0]
    a = [_raw(x, n) for x in (u, v, w)]
    return lib.oracle_dissipation(n, *[_ptr(x) for x in a], nu, 1 if pi_f32 else 0)


def drop_count(phi, dx: float):
    """post/DropCountSize on a raw field indexed [i,j,k]: (cells, deq) in discovery order."""
    lib = _load()
    n = phi.shape[0]
    a = _raw(phi, n)
    cap = 1 << 16
    cells = np.empty(cap, dtype=np.int64)
    deq = np.empty(cap)
    cnt = lib.oracle_drop_count(n, _ptr(a), cap, cells.ctypes.data, _ptr(deq), dx)
    return cells[:min(cnt, cap)], deq[:min(cnt, cap)]
