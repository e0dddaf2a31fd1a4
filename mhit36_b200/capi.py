"""ctypes binding of libmhit.so (the C ABI declared in include/mhit.h).

This is the Python side of the drop-in boundary.  There is no CPU path: if the
library is not built, importing the binding raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmhit.so")

MHIT_OK = 0
MHIT_ERR_INVALID = 1
MHIT_ERR_CUDA = 2
MHIT_ERR_NOMEM = 3
MHIT_ERR_CFL = 4
MHIT_ERR_NONFINITE = 5
MHIT_ERR_IO = 6
MHIT_ERR_UNSUPPORTED = 7
MHIT_ERR_STATE = 8
MHIT_ERR_SCRATCH_LIMIT = 9
MHIT_ERR_TIMEOUT = 10
MHIT_NOALLOC_MAX_N = 128

MHIT_LAYOUT_RAW = 0
MHIT_LAYOUT_PIX_HALO = 1
MHIT_FP64 = 0
MHIT_FP32_REFINE = 1


class MhitParams(ctypes.Structure):
    """struct mhit_params: input.inp lines 1-16 then the extensions."""

    _fields_ = [
        ("restart", ctypes.c_int32), ("tstart", ctypes.c_int32), ("tfin", ctypes.c_int32), ("dump", ctypes.c_int32),
        ("inflow", ctypes.c_int32), ("inphi", ctypes.c_int32),
        ("dt", ctypes.c_double), ("mu", ctypes.c_double), ("rho", ctypes.c_double),
        ("f1", ctypes.c_double), ("f2", ctypes.c_double), ("f3", ctypes.c_double), ("k0", ctypes.c_double),
        ("radius", ctypes.c_double), ("sigma", ctypes.c_double), ("epsr", ctypes.c_double),
        ("lin_force", ctypes.c_double),
        ("k2_mode", ctypes.c_int32), ("grid_mode", ctypes.c_int32),
        ("cfl_limit", ctypes.c_double),
        ("tanh_identity", ctypes.c_int32),
        ("phi_floor", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 6),
    ]


class MhitDiag(ctypes.Structure):
    _fields_ = [
        ("umax", ctypes.c_double), ("cfl", ctypes.c_double),
        ("umean", ctypes.c_double), ("vmean", ctypes.c_double), ("wmean", ctypes.c_double),
        ("gamma", ctypes.c_double), ("max_div", ctypes.c_double),
        ("step", ctypes.c_int64), ("status", ctypes.c_int32), ("reserved", ctypes.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class MhitStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in
                ("ke", "dissipation", "max_div", "phi_sum", "phi_min", "phi_max", "umean", "reserved")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class MhitEnsInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32), ("n", ctypes.c_int32),
                ("steps_issued", ctypes.c_int32), ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double), ("diag", MhitDiag), ("kz", ctypes.c_int32), ("mty", ctypes.c_int32)]


class MhitEnsStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int64), ("graph_launches", ctypes.c_int64), ("bytes_used", ctypes.c_size_t),
                ("bytes_budget", ctypes.c_size_t), ("classes", ctypes.c_int32), ("slots", ctypes.c_int32)]


RQ_QUEUED, RQ_RUNNING, RQ_DONE, RQ_FAILED, RQ_CANCELLED = range(5)
MHIT_ENS_KEEP_RESULT, MHIT_ENS_BORROW_INPUT = 1, 2

# Every symbol include/mhit.h declares (checked by the CPU tests).
HEADER_SYMBOLS = [
    "mhit_default_params", "mhit_create", "mhit_set_fields", "mhit_get_fields", "mhit_get_pressure",
    "mhit_step", "mhit_get_diag", "mhit_save", "mhit_load", "mhit_poisson", "mhit_poisson_device",
    "mhit_device_state", "mhit_sync_state", "mhit_memory_bytes", "mhit_launches_per_step",
    "mhit_destroy", "mhit_strerror", "mhit_size_supported", "mhit_profile_step", "mhit_stage_name",
    "mhit_step_async", "mhit_stream", "mhit_last_error", "mhit_diagnostics", "mhit_poisson_noalloc",
    "mhit_ens_create", "mhit_ens_submit", "mhit_ens_progress", "mhit_ens_wait", "mhit_ens_query", "mhit_ens_result",
    "mhit_ens_release", "mhit_ens_cancel", "mhit_ens_stats", "mhit_ens_last_error", "mhit_ens_destroy",
    "mhit_set_tiles", "mhit_drop_count", "mhit_check_bounded_wait",
]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libmhit.so and declare its signatures.  Raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built (python -m mhit36_b200.build); there is no CPU fallback")
    lib = ctypes.CDLL(path)
    H = ctypes.c_void_p
    dp = ctypes.c_void_p  # pointers passed as integers (numpy .ctypes.data / torch data_ptr)
    P = ctypes.POINTER
    sig = {
        "mhit_default_params": (None, [P(MhitParams)]),
        "mhit_create": (ctypes.c_int, [P(MhitParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, P(H)]),
        "mhit_set_fields": (ctypes.c_int, [H, dp, dp, dp, dp, ctypes.c_int]),
        "mhit_get_fields": (ctypes.c_int, [H, dp, dp, dp, dp, ctypes.c_int]),
        "mhit_get_pressure": (ctypes.c_int, [H, dp, ctypes.c_int]),
        "mhit_step": (ctypes.c_int, [H, ctypes.c_int, P(MhitDiag)]),
        "mhit_step_async": (ctypes.c_int, [H, ctypes.c_int]),
        "mhit_get_diag": (ctypes.c_int, [H, P(MhitDiag)]),
        "mhit_save": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_int]),
        "mhit_load": (ctypes.c_int, [H, ctypes.c_char_p, ctypes.c_int]),
        "mhit_poisson": (ctypes.c_int, [H, dp, dp]),
        "mhit_poisson_device": (ctypes.c_int, [H, dp, dp]),
        "mhit_device_state": (ctypes.c_int, [H, P(ctypes.c_void_p), P(ctypes.c_void_p), P(ctypes.c_void_p),
                                             P(ctypes.c_void_p)]),
        "mhit_sync_state": (ctypes.c_int, [H]),
        "mhit_memory_bytes": (ctypes.c_int, [H, P(ctypes.c_size_t)]),
        "mhit_launches_per_step": (ctypes.c_int, [H, P(ctypes.c_int)]),
        "mhit_destroy": (ctypes.c_int, [H]),
        "mhit_strerror": (ctypes.c_char_p, [ctypes.c_int]),
        "mhit_size_supported": (ctypes.c_int, [ctypes.c_int]),
        "mhit_check_bounded_wait": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, P(ctypes.c_int)]),
        "mhit_last_error": (ctypes.c_char_p, [H]),
        "mhit_stream": (ctypes.c_void_p, [H]),
        "mhit_profile_step": (ctypes.c_int, [H, ctypes.c_int, P(ctypes.c_double), P(ctypes.c_int)]),
        "mhit_stage_name": (ctypes.c_char_p, [H, ctypes.c_int]),
        "mhit_diagnostics": (ctypes.c_int, [H, ctypes.c_int, P(MhitStats)]),
        "mhit_poisson_noalloc": (ctypes.c_int, [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
        "mhit_ens_create": (ctypes.c_int, [ctypes.c_size_t, ctypes.c_int, P(H)]),
        "mhit_ens_submit": (ctypes.c_int, [H, P(MhitParams), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           dp, dp, dp, dp, ctypes.c_int, P(ctypes.c_int64)]),
        "mhit_ens_progress": (ctypes.c_int, [H, P(ctypes.c_int)]),
        "mhit_ens_wait": (ctypes.c_int, [H, ctypes.c_double, P(ctypes.c_int)]),
        "mhit_ens_query": (ctypes.c_int, [H, ctypes.c_int64, P(MhitEnsInfo)]),
        "mhit_ens_result": (ctypes.c_int, [H, ctypes.c_int64, dp, dp, dp, dp]),
        "mhit_ens_release": (ctypes.c_int, [H, ctypes.c_int64]),
        "mhit_ens_cancel": (ctypes.c_int, [H, ctypes.c_int64]),
        "mhit_ens_stats": (ctypes.c_int, [H, P(MhitEnsStats)]),
        "mhit_ens_last_error": (ctypes.c_char_p, [H]),
        "mhit_ens_destroy": (ctypes.c_int, [H]),
        "mhit_set_tiles": (ctypes.c_int, [H, ctypes.c_int, ctypes.c_int]),
        "mhit_drop_count": (ctypes.c_int, [H, ctypes.c_int, P(ctypes.c_int), dp, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MhitError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        lib = load_library()
        msg = f"{where}: {lib.mhit_strerror(status).decode()} (status {status})"
        if detail:
            msg += f" [{detail}]"
        super().__init__(msg)
        self.status = status
