"""1024^3 Navier-Stokes on one B200, in both forms.

The mixed-precision configuration at 1024^3 (NS only, FP32 state with the
FP64-residual refinement, about 52 GB resident) against the FP64 form of the
same discrete problem (FD-modified k^2 in both, about 95 GB), run one after
the other.  Bars as at the smaller sizes: max |div u| of the FP64 projection
<= 1e-10 after every step, kinetic energy and dissipation within 1e-4 of the
FP64 form; the velocity error and the step times are stated.  This is also
the only test that runs the 1024 kernel configurations (radix-8 column
passes over two-column chunks, 2-line-pair x passes, the fused projection
with 2 line pairs per CTA).

The seeded initial field is fields.random_velocity's spectral band; its
inverse FFT runs on the GPU here (torch), only to make the input quickly.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _velocity_raw_gpu(n, seed):
    """fields.random_velocity(n, seed) made on the GPU, returned in the C
    ABI's raw layout (x fastest) as host float64 arrays."""
    import torch
    from mhit36_b200 import fields
    ix, iz, F = fields.velocity_band(n, seed)
    dev = torch.device("cuda")
    tix, tiz = torch.as_tensor(ix, device=dev), torch.as_tensor(iz, device=dev)
    comps = []
    for c in range(3):
        G = torch.zeros((n, n, n // 2 + 1), dtype=torch.complex128, device=dev)
        G[tix[:, None, None], tix[None, :, None], tiz[None, None, :]] = torch.from_numpy(F[c]).to(dev)
        f = torch.fft.irfftn(G, s=(n, n, n), dim=(0, 1, 2))
        del G
        f -= f.mean()
        comps.append(f)
    cur = float(torch.sqrt(sum(torch.mean(f * f) for f in comps) / 3.0))
    raw = []
    for f in comps:
        f *= 1.0 / cur
        raw.append(f.permute(2, 1, 0).contiguous().cpu().numpy().reshape(-1))  # [k][j][i]: x fastest
    del comps, f
    torch.cuda.empty_cache()
    return raw


def _run(n, p, precision, raw, steps, timed_steps):
    import torch
    from mhit36_b200 import Solver
    with Solver(n, p, precision=precision, phase_field=False) as s:
        s.set_fields_ptr(raw[0].ctypes.data, raw[1].ctypes.data, raw[2].ctypes.data, None)
        worst = -1.0
        for _ in range(steps):
            d = s.step(1)
            worst = max(worst, d["max_div"])
        st = s.stats()
        out = [np.empty(n ** 3) for _ in range(3)]
        s.get_fields_ptr(out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data, None)
        stream = torch.cuda.ExternalStream(s.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step_async(timed_steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / timed_steps
        assert s.diag()["status"] == 0
    return worst, st, out, ms


def test_ns_1024_fp32_refine_vs_fp64():
    from mhit36_b200.config import InputParams
    n, steps = 1024, 10
    t0 = time.perf_counter()
    raw = _velocity_raw_gpu(n, n)
    gen_s = time.perf_counter() - t0
    p = InputParams(dt=2e-4, mu=6e-3, rho=1.0, lin_force=0.1, k2_mode=1)
    div32, st32, f32, ms32 = _run(n, p, "fp32", raw, steps, 5)
    div64, st64, f64, ms64 = _run(n, p, "fp64", raw, steps, 5)
    errs = {name: float(np.max(np.abs(a - b)) / np.max(np.abs(b))) for name, a, b in zip("uvw", f32, f64)}
    errs["ke"] = abs(st32["ke"] / st64["ke"] - 1)
    errs["dissipation"] = abs(st32["dissipation"] / st64["dissipation"] - 1)
    print(f"1024^3 NS, {steps} steps: FP32 refine {ms32:.2f} ms/step, FP64 {ms64:.2f} ms/step "
          f"({n ** 3 / ms32 / 1e3:.0f} and {n ** 3 / ms64 / 1e3:.0f} Mpts*steps/s), worst max|div| {div32:.3e}, "
          f"errors vs FP64 {errs}, input generation {gen_s:.1f} s")
    assert div64 == -1.0
    assert 0 < div32 <= 1e-10
    assert errs["ke"] <= 1e-4 and errs["dissipation"] <= 1e-4
    assert all(errs[c] < 1e-4 for c in "uvw"), errs
