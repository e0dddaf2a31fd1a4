"""Served ensemble of independent MHIT36 simulations (mhit_ens_* in include/mhit.h).

Requests of uneven grid sizes are queued, admitted as slots and HBM free up,
kept resident and advanced together by per-class CUDA graphs of batched
kernels (one graph per grid size / precision / phase-field class).  The
driver calls ``progress()`` in a loop, with ``wait()`` between calls; each
progress call admits what fits and keeps a few milliseconds of batched steps
queued on every busy class.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi
from .capi import MhitEnsInfo, MhitEnsStats, MhitError, load_library
from .config import InputParams
from .solver import _from_raw, _to_raw, make_params

STATE_NAMES = {capi.RQ_QUEUED: "queued", capi.RQ_RUNNING: "running", capi.RQ_DONE: "done",
               capi.RQ_FAILED: "failed", capi.RQ_CANCELLED: "cancelled"}


class Ensemble:
    def __init__(self, budget_bytes: int = 0, slots_per_class: int = 8):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.mhit_ens_create(budget_bytes, slots_per_class, ctypes.byref(h))
        if rc:
            raise MhitError(rc, "mhit_ens_create")
        self.h = h
        self._n = {}
        self._borrowed = {}  # borrowed input arrays, kept alive until release()

    def _check(self, rc, where):
        if rc:
            raise MhitError(rc, where, self.lib.mhit_ens_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhit_ens_destroy(self.h)
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

    def submit(self, n: int, params: InputParams, u, v, w, phi=None, nsteps: int = 100, precision: str = "fp64",
               keep: bool = True, borrow: bool = False) -> int:
        """Queue a request.  borrow=True hands the (raw-layout) input arrays to
        the ensemble without a copy; they are held here until release()."""
        prec = {"fp64": capi.MHIT_FP64, "fp32": capi.MHIT_FP32_REFINE, "fp32_refine": capi.MHIT_FP32_REFINE}[precision]
        mp = make_params(params)
        arrs = [_to_raw(u, n), _to_raw(v, n), _to_raw(w, n), _to_raw(phi, n) if phi is not None else None]
        ptrs = [a.ctypes.data if a is not None else None for a in arrs]
        flags = (capi.MHIT_ENS_KEEP_RESULT if keep else 0) | (capi.MHIT_ENS_BORROW_INPUT if borrow else 0)
        rid = ctypes.c_int64()
        self._check(self.lib.mhit_ens_submit(self.h, ctypes.byref(mp), n, prec, int(phi is not None), nsteps,
                                             *ptrs, flags, ctypes.byref(rid)), "mhit_ens_submit")
        self._n[rid.value] = (n, phi is not None)
        if borrow:
            self._borrowed[rid.value] = arrs
        return rid.value

    def progress(self) -> int:
        pending = ctypes.c_int()
        self._check(self.lib.mhit_ens_progress(self.h, ctypes.byref(pending)), "mhit_ens_progress")
        return pending.value

    def wait(self, timeout: float) -> bool:
        """Sleep until progress() has something to do (True) or `timeout` s pass (False)."""
        ready = ctypes.c_int()
        self._check(self.lib.mhit_ens_wait(self.h, float(timeout), ctypes.byref(ready)), "mhit_ens_wait")
        return bool(ready.value)

    def query(self, rid: int) -> dict:
        info = MhitEnsInfo()
        self._check(self.lib.mhit_ens_query(self.h, rid, ctypes.byref(info)), "mhit_ens_query")
        return {"state": STATE_NAMES[info.state], "status": info.status, "n": info.n,
                "steps_issued": info.steps_issued, "t_submit": info.t_submit, "t_admit": info.t_admit,
                "t_done": info.t_done, "diag": info.diag.as_dict(), "kz": info.kz, "mty": info.mty}

    def result(self, rid: int):
        n, pf = self._n[rid]
        out = [np.empty(n ** 3) for _ in range(4)]
        self._check(self.lib.mhit_ens_result(self.h, rid, out[0].ctypes.data, out[1].ctypes.data,
                                             out[2].ctypes.data, out[3].ctypes.data if pf else None),
                    "mhit_ens_result")
        res = [_from_raw(a, n) for a in out[:3]]
        res.append(_from_raw(out[3], n) if pf else None)
        return tuple(res)

    def release(self, rid: int):
        self._check(self.lib.mhit_ens_release(self.h, rid), "mhit_ens_release")
        self._borrowed.pop(rid, None)

    def cancel(self, rid: int):
        self._check(self.lib.mhit_ens_cancel(self.h, rid), "mhit_ens_cancel")

    def stats(self) -> dict:
        st = MhitEnsStats()
        self._check(self.lib.mhit_ens_stats(self.h, ctypes.byref(st)), "mhit_ens_stats")
        return {k: getattr(st, k) for k, _ in st._fields_}

    def run(self, max_rounds: int = 10 ** 9) -> None:
        """Progress until nothing is queued or running, sleeping between
        rounds until there is something to do."""
        for _ in range(max_rounds):
            if self.progress() == 0:
                return
            self.wait(0.01)
        raise RuntimeError("ensemble did not drain")
