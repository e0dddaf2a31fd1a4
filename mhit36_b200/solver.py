"""Host-side mirror of the reference's timestep surface.

``Solver`` owns one libmhit handle: the module arrays of
multi/module.f90:39-58 resident on the GPU, advanced by ``step`` (the loop
body of multi/main.f90:334-946).  Arrays cross the boundary as numpy float64
arrays indexed a[i, j, k] (x fastest in memory, the Fortran order of the
reference), or as raw device pointers.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import capi
from .capi import MhitDiag, MhitError, MhitParams, MhitStats, load_library
from .config import InputParams


def make_params(p: InputParams) -> MhitParams:
    lib = load_library()
    m = MhitParams()
    lib.mhit_default_params(ctypes.byref(m))
    for name in ("restart", "tstart", "tfin", "dump", "inflow", "inphi"):
        setattr(m, name, int(getattr(p, name)))
    for name in ("dt", "mu", "rho", "f1", "f2", "f3", "k0", "radius", "sigma", "epsr", "lin_force", "cfl_limit"):
        setattr(m, name, float(getattr(p, name)))
    m.k2_mode = int(p.k2_mode)
    m.grid_mode = int(p.grid_mode)
    m.tanh_identity = int(p.tanh_identity)
    m.phi_floor = int(p.phi_floor)
    return m


def _to_raw(a, n: int) -> np.ndarray:
    """numpy [i,j,k] (or flat, x fastest) -> contiguous float64 in file order."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 3:
        if a.shape != (n, n, n):
            raise ValueError(f"expected shape {(n, n, n)}, got {a.shape}")
        return np.ascontiguousarray(a.T)  # (k,j,i) C order == Fortran (i,j,k)
    if a.size != n ** 3:
        raise ValueError("wrong size")
    return np.ascontiguousarray(a.reshape(-1))


def _from_raw(flat: np.ndarray, n: int) -> np.ndarray:
    return flat.reshape((n, n, n)).T  # view indexed [i,j,k]


class Solver:
    """One MHIT36 simulation of n^3 cells on the current CUDA device."""

    def __init__(self, n: int, params: InputParams | None = None, precision: str = "fp64",
                 phase_field: bool = True):
        self.lib = load_library()
        self.n = n
        self.params = params if params is not None else InputParams()
        self.phase_field = bool(phase_field)
        self.precision = {"fp64": capi.MHIT_FP64, "fp32": capi.MHIT_FP32_REFINE,
                          "fp32_refine": capi.MHIT_FP32_REFINE}[precision]
        self._mp = make_params(self.params)
        h = ctypes.c_void_p()
        rc = self.lib.mhit_create(ctypes.byref(self._mp), n, n, n, self.precision, int(self.phase_field),
                                  ctypes.byref(h))
        if rc:
            raise MhitError(rc, f"mhit_create(n={n})")
        self.h = h

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.mhit_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, where: str):
        if rc:
            detail = self.lib.mhit_last_error(self.h).decode() if self.h else ""
            raise MhitError(rc, where, detail)

    # -- state
    def set_fields(self, u, v, w, phi=None):
        n = self.n
        arrs = [_to_raw(u, n), _to_raw(v, n), _to_raw(w, n)]
        arrs.append(_to_raw(phi, n) if (phi is not None and self.phase_field) else None)
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        self._check(self.lib.mhit_set_fields(self.h, *ptrs, capi.MHIT_LAYOUT_RAW), "mhit_set_fields")

    def set_fields_ptr(self, u, v, w, phi, layout: int = capi.MHIT_LAYOUT_RAW):
        """Host pointers (ints) to float64 arrays in file order."""
        self._check(self.lib.mhit_set_fields(self.h, u, v, w, phi, layout), "mhit_set_fields")

    def get_fields(self):
        n = self.n
        out = [np.empty(n ** 3) for _ in range(4)]
        phi_ptr = out[3].ctypes.data if self.phase_field else None
        self._check(self.lib.mhit_get_fields(self.h, out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data,
                                             phi_ptr, capi.MHIT_LAYOUT_RAW), "mhit_get_fields")
        res = [_from_raw(a, n) for a in out[:3]]
        res.append(_from_raw(out[3], n) if self.phase_field else None)
        return tuple(res)

    def get_fields_ptr(self, u, v, w, phi, layout: int = capi.MHIT_LAYOUT_RAW):
        self._check(self.lib.mhit_get_fields(self.h, u, v, w, phi, layout), "mhit_get_fields")

    def get_pressure(self):
        out = np.empty(self.n ** 3)
        self._check(self.lib.mhit_get_pressure(self.h, out.ctypes.data, capi.MHIT_LAYOUT_RAW), "mhit_get_pressure")
        return _from_raw(out, self.n)

    # -- time stepping
    def step(self, nsteps: int = 1, raise_on_error: bool = True) -> dict:
        d = MhitDiag()
        rc = self.lib.mhit_step(self.h, nsteps, ctypes.byref(d))
        if rc and raise_on_error:
            self._check(rc, "mhit_step")
        out = d.as_dict()
        out["rc"] = rc
        return out

    def step_async(self, nsteps: int = 1):
        self._check(self.lib.mhit_step_async(self.h, nsteps), "mhit_step_async")

    def diag(self) -> dict:
        d = MhitDiag()
        self._check(self.lib.mhit_get_diag(self.h, ctypes.byref(d)), "mhit_get_diag")
        return d.as_dict()

    def stats(self, pi_f32: bool = True) -> dict:
        """FP64 KE, dissipation (post/compute_diss convention), max|div u|, phi sum/bounds."""
        st = MhitStats()
        self._check(self.lib.mhit_diagnostics(self.h, int(pi_f32), ctypes.byref(st)), "mhit_diagnostics")
        return st.as_dict()

    def drops(self):
        """Drop count and sizes of the current phi (post/DropCountSize convention):
        returns (cells, deq), numpy arrays in the reference's discovery order."""
        nd = ctypes.c_int()
        self._check(self.lib.mhit_drop_count(self.h, 0, ctypes.byref(nd), None, None), "mhit_drop_count")
        cells = np.empty(max(nd.value, 1), dtype=np.int64)
        deq = np.empty(max(nd.value, 1))
        self._check(self.lib.mhit_drop_count(self.h, nd.value, ctypes.byref(nd), cells.ctypes.data, deq.ctypes.data),
                    "mhit_drop_count")
        return cells[:nd.value], deq[:nd.value]

    # -- files
    def save(self, outdir: str, t: int):
        os.makedirs(outdir, exist_ok=True)
        self._check(self.lib.mhit_save(self.h, outdir.encode(), t), "mhit_save")

    def load(self, outdir: str, t: int):
        self._check(self.lib.mhit_load(self.h, outdir.encode(), t), "mhit_load")

    # -- Poisson
    def poisson(self, rhs) -> np.ndarray:
        r = _to_raw(rhs, self.n)
        p = np.empty(self.n ** 3)
        self._check(self.lib.mhit_poisson(self.h, r.ctypes.data, p.ctypes.data), "mhit_poisson")
        return _from_raw(p, self.n)

    def poisson_device(self, rhs_ptr: int, p_ptr: int):
        self._check(self.lib.mhit_poisson_device(self.h, rhs_ptr, p_ptr), "mhit_poisson_device")

    # -- introspection
    def device_state(self):
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        self._check(self.lib.mhit_device_state(self.h, *[ctypes.byref(p) for p in ptrs]), "mhit_device_state")
        return tuple(p.value for p in ptrs)

    def sync_state(self):
        self._check(self.lib.mhit_sync_state(self.h), "mhit_sync_state")

    def memory_bytes(self) -> int:
        b = ctypes.c_size_t()
        self._check(self.lib.mhit_memory_bytes(self.h, ctypes.byref(b)), "mhit_memory_bytes")
        return b.value

    def launches_per_step(self) -> int:
        v = ctypes.c_int()
        self._check(self.lib.mhit_launches_per_step(self.h, ctypes.byref(v)), "mhit_launches_per_step")
        return v.value

    def profile_step(self, reps: int = 3) -> dict:
        """Mean ms per kernel over `reps` individually launched steps."""
        ms = (ctypes.c_double * 16)()
        ns = ctypes.c_int()
        rc = self.lib.mhit_profile_step(self.h, reps, ms, ctypes.byref(ns))
        self._check(rc, "mhit_profile_step")
        out = {}
        for k in range(ns.value):
            out[self.lib.mhit_stage_name(self.h, k).decode()] = ms[k]
        return out

    def set_tiles(self, kz: int = 0, mty: int = 0):
        """Stencil z chunk and momentum tile height (0 = defaults); results do not depend on them."""
        self._check(self.lib.mhit_set_tiles(self.h, kz, mty), "mhit_set_tiles")

    def stream(self) -> int:
        return self.lib.mhit_stream(self.h)
