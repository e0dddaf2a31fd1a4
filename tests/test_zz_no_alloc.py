"""GPU test of mhit_poisson_noalloc, the Poisson solve for callers that cannot
let the library allocate device memory (their device memory belongs to their
own allocator, or they cannot absorb cudaFree's device-wide synchronisation).

It is called through the C ABI and checked against the handle-based
mhit_poisson_device on the same device inputs, on two calls in a row (the
scratch keeps the previous call's contents).  The sizes run largest first,
each with a different k2 / grid mode, so every solve after the first starts
from a spectrum array left behind by a solve of another size and row pitch.
This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the Poisson tolerance of tests/test_gpu_parity.py

# largest first; 96 exercises the mixed-radix (radix-3) register transform
CASES = [(128, 1, 1), (96, 0, 1), (64, 0, 0), (32, 1, 0)]


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


def _reference(n, k2_mode, grid_mode, rhs):
    import torch
    from mhit36_b200 import Solver
    from mhit36_b200.config import InputParams
    ref = [torch.empty_like(r) for r in rhs]
    with Solver(n, InputParams(k2_mode=k2_mode, grid_mode=grid_mode), phase_field=False) as s:
        for r, o in zip(rhs, ref):
            s.poisson_device(r.data_ptr(), o.data_ptr())
        torch.cuda.synchronize()
    return ref


def test_noalloc_matches_handle_solve_twice():
    import torch
    from mhit36_b200 import capi
    lib = capi.load_library()
    for n, k2_mode, grid_mode in CASES:
        gen = torch.Generator(device="cuda").manual_seed(n)
        rhs = [torch.randn(n ** 3, dtype=torch.float64, device="cuda", generator=gen) for _ in range(2)]
        ref = _reference(n, k2_mode, grid_mode, rhs)
        for r, o in zip(rhs, ref):  # two calls in a row share the scratch
            got = torch.full_like(r, float("nan"))
            rc = lib.mhit_poisson_noalloc(r.data_ptr(), got.data_ptr(), n, k2_mode, grid_mode, None)
            assert rc == capi.MHIT_OK, lib.mhit_strerror(rc)
            torch.cuda.synchronize()
            assert _rel(got, o) <= TOL, (n, k2_mode, grid_mode)


def test_noalloc_on_caller_stream():
    """The documented use: the caller's own non-blocking stream."""
    import torch
    from mhit36_b200 import capi
    lib = capi.load_library()
    n, k2_mode, grid_mode = 96, 1, 0
    gen = torch.Generator(device="cuda").manual_seed(3)
    rhs = [torch.randn(n ** 3, dtype=torch.float64, device="cuda", generator=gen) for _ in range(2)]
    ref = _reference(n, k2_mode, grid_mode, rhs)
    stream = torch.cuda.Stream()
    outs = [torch.full_like(r, float("nan")) for r in rhs]
    torch.cuda.synchronize()
    for r, o, want in zip(rhs, outs, ref):
        rc = lib.mhit_poisson_noalloc(r.data_ptr(), o.data_ptr(), n, k2_mode, grid_mode, stream.cuda_stream)
        assert rc == capi.MHIT_OK, lib.mhit_strerror(rc)
        stream.synchronize()
        assert _rel(o, want) <= TOL


def test_noalloc_rejects_sizes_beyond_scratch():
    import torch
    from mhit36_b200 import capi
    lib = capi.load_library()
    n = 2 * capi.MHIT_NOALLOC_MAX_N
    rhs = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.mhit_poisson_noalloc(rhs.data_ptr(), rhs.data_ptr(), n, 0, 0, None)
    assert rc == capi.MHIT_ERR_SCRATCH_LIMIT
    assert b"scratch" in lib.mhit_strerror(rc)
