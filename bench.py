"""Benchmark of the MHIT36 timestep on B200: Mpts*steps/s at 512^3 NS+ACDI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 512] [--precision fp64] [--ns-only]

One JSON line on rank 0.  `value` is N^3 * steps / s with the state resident
in HBM (device-timed with CUDA events on the solver's stream, max over ranks,
summed over replicas).  `e2e` is the same metric through the public API with
host buffers: the upload of the state from pinned host memory, K steps each
returning its diagnostics to the host, and the download of the state.

On one GPU the line also carries the library's two other forms:
`fp32_refine` (the FP32 + FP64-residual refinement form on the same workload:
its step time, speed-up over the FP64 form and per-kernel roofline, and its
errors against the FP64 form of the same discrete problem after the same
steps) and `serving` (a seeded stream of --serve-requests requests served by
the ensemble in both forms and one at a time with the plain form).

Multi-GPU: the step does not shard (one simulation per GPU), so N ranks run N
independent replicas of the workload ("replicas only", weak scaling); there is
no collective on the data path.

--impl reference times the CPU oracle (the C++ restatement of the
reference's step, on all host threads) on the same workload (512^3 NS+ACDI,
about 5 s per step on 16 cores); the reference's own Fortran/OpenACC/cuDecomp
build needs nvfortran and cuDecomp, which this image does not have.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mpts*steps/s at 512^3 NS+ACDI (FP64 plain form)"
UNIT = "Mpts*steps/s"
# Compulsory HBM traffic per grid point per step under a schedule in which
# each stage reads its inputs once and writes its outputs once, the half
# spectrum counts as one field pass and the inverse x transform feeds the
# projection without storing p: FP64 NS+ACDI 35 field passes (280 B), NS-only
# 29 (232 B).  The FP32 refinement form: 50 four-byte passes with ACDI
# (200 B), 44 without (176 B) -- the same passes plus the residual and the
# second solve.
ALGO_BYTES_STEP = {"fp64": {True: 280, False: 232}, "fp32": {True: 200, False: 176}}

# DRAM bytes (read + write) per grid point per launch, from ncu captures of
# the FP64 kernels at 256^3 (dram__bytes_read.sum + dram__bytes_write.sum of
# a launch / 256^3; summaries in profiles/momentum_fp64_256_full.md,
# profiles/phase_fp64_256_full.md and, for the Poisson kernels,
# profiles/kernels_fp64_256_full.md).  A stencil or column pass touches every
# point the same way at any size, so traffic scales with the points
# processed; a full 512^3 capture is too large to take under ncu.
DRAM_BYTES_PER_POINT_FP64 = {"momentum": 103.45, "phase": 40.25, "project": 54.13, "xfwd": 30.80,
                             "yfwd": 13.59, "zsolve": 13.64, "yinv": 13.59, "xinv": 13.82, "xinvproj": 55.30}


def kernel_bytes_per_point(n: int, pf: bool, precision: str = "fp64") -> dict:
    """Algorithmic HBM bytes per grid point for each kernel of the form."""
    e = 8.0 if precision == "fp64" else 4.0   # bytes per stored real
    spec = 2 * e * (n // 2 + 1) / n           # half spectrum, complex
    kb = {
        "phase": 5 * e,                           # read u,v,w,phi; write phi
        "momentum": (13 if pf else 12) * e,       # read u,v,w,rhs_o(3)[,phi]; write ustar(3), rhs_o(3)
        "xfwd": 3 * e + spec,                     # read ustar(3); write half spectrum
        "yfwd": 2 * spec,
        "zsolve": 2 * spec,
        "yinv": 2 * spec,
        "xinv": spec + e,                         # read spectrum; write p (p0)
        "project": 7 * e,                         # read p, ustar(3); write u,v,w
        "xinvproj": spec + 6 * e,                 # fused: read spectrum, ustar(3); write u,v,w
        "finalize": 0.0,
    }
    if precision != "fp64":
        # second solve, of the FP64 residual r - L(p0): read ustar(3) and p0,
        # write the half spectrum; the same column passes; write dp.  The
        # projection also reads dp.
        kb.update({"xres": 4 * e + spec, "yfwd2": 2 * spec, "zsolve2": 2 * spec, "yinv2": 2 * spec,
                   "xinv2": spec + e, "project": 8 * e,
                   # fused: read the correction spectrum, p0, ustar(3); write u,v,w
                   "xinvproj": spec + 7 * e})
    return kb


def metric_name(n: int, pf: bool, precision: str = "fp64") -> str:
    """The headline metric for the 512^3 NS+ACDI FP64 workload, else the same
    metric named for the configuration actually run."""
    if precision == "fp64" and n == 512 and pf:
        return METRIC
    return f"Mpts*steps/s at {n}^3 NS{'+ACDI' if pf else ''} ({precision} form)"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--ns-only", action="store_true")
    # The explicit ACDI diffusion gamma*eps*lap(phi) (gamma = Umax, eps = dx) is
    # stable only for Umax*dt/dx < 1/6; at 512^3 with Umax ~ 4 that needs
    # dt < 5e-4.  The default is the reference's own input.inp dt (2e-4);
    # throughput does not depend on dt.
    ap.add_argument("--dt", type=float, default=2e-4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32 refinement form's sub-record")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-ensemble sub-record")
    ap.add_argument("--serve-requests", type=int, default=32)
    return ap.parse_args(argv)


def workload_params(n, dt, precision="fp64"):
    from mhit36_b200 import fields
    from mhit36_b200.config import InputParams
    # the FP32 refinement form solves with the FD-modified k^2 (the symbol of
    # the 7-point Laplacian its FP64 residual uses)
    p = InputParams(dt=dt, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1,
                    k2_mode=1 if precision == "fp32" else 0)
    if n >= 512:
        recipe = (64, 0.2, 0.35)
    else:
        recipe = fields.DROP_RECIPES.get(n, (8, 0.4, 0.6))
    return p, None, recipe


def workload(n, pf, dt, precision="fp64"):
    from mhit36_b200 import fields
    p, _, recipe = workload_params(n, dt, precision)
    u, v, w = fields.random_velocity(n, n)
    phi = None
    if pf:
        c, r = fields.place_drops(n, n + 1, *recipe)
        phi = fields.drop_field(n, c, r)
    return p, (u, v, w, phi), recipe


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    nvidia-smi takes a moment to start, so start() returns only once the
    sampler has written its first row; the rows written after that (during
    the timed region, plus the first one after it if the region was shorter
    than the sampling period) are the ones reported."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    PERIOD_MS = 100

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None
        self.n0 = 0

    def _rows(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        return rows

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while not self._rows() and time.time() - t0 < 10.0 and self.proc.poll() is None:
            time.sleep(0.02)
        self.n0 = len(self._rows())

    def stop(self):
        if self.proc is None:
            return None
        t0 = time.time()
        while len(self._rows()) <= self.n0 and time.time() - t0 < 3 * self.PERIOD_MS / 1000 and \
                self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = self._rows()[self.n0:]
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_oracle_rate(n, pf, dt, case, threads=0, max_seconds=20.0, min_steps=1, max_steps=5):
    """Time the oracle on host cores; returns (Mpts*steps/s, steps, threads)."""
    from oracle import Oracle
    from oracle.oracle import build_oracle
    build_oracle()
    p = case[0]
    o = Oracle(n, dt=p.dt, mu=p.mu, rho=p.rho, sigma=p.sigma, epsr=p.epsr, lin_force=p.lin_force,
               phase_field=int(pf), threads=threads)
    u, v, w, phi = case[1]
    o.set_fields(u, v, w, phi)
    nthreads = o.lib.oracle_set_threads(0)
    steps = 0
    t0 = time.perf_counter()
    while steps < max_steps:
        o.step(1)
        steps += 1
        if steps >= min_steps and time.perf_counter() - t0 > max_seconds:
            break
    el = time.perf_counter() - t0
    o.close()
    return n ** 3 * steps / el / 1e6, steps, nthreads, el


def run_reference(args, rank, world):
    """--impl reference: the CPU oracle on all host threads, rank 0 only, on
    the same workload as the GPU arm (512^3 NS+ACDI by default)."""
    if rank != 0:
        return
    pf = not args.ns_only
    n = args.n
    case = workload(n, pf, args.dt)
    from oracle import Oracle
    from oracle.oracle import build_oracle
    build_oracle()
    p = case[0]
    o = Oracle(n, dt=p.dt, mu=p.mu, rho=p.rho, sigma=p.sigma, epsr=p.epsr, lin_force=p.lin_force,
               phase_field=int(pf))
    o.set_fields(*case[1])
    threads = o.lib.oracle_set_threads(0)
    for _ in range(args.warmup):
        o.step(1)
    t0 = time.perf_counter()
    rc, _ = o.step(args.steps)
    el = time.perf_counter() - t0
    value = n ** 3 * args.steps / el / 1e6
    recipe = case[2]
    sample = (f"{n}^3 NS{'+ACDI' if pf else ''} FP64 oracle step, {recipe[0] if pf else 0} drops "
              f"r in [{recipe[1]},{recipe[2]}], {args.steps} steps")
    line = {"impl": "reference", "metric": metric_name(n, pf), "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded random-phase velocity, seeded drops)",
            "config": {"workload": sample, "n": n, "phase_field": pf},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Fortran (nvfortran+OpenACC+cuDecomp) cannot be built in this image; "
                    "timed: the C++ oracle restating multi/main.f90:329-977", "status": rc}
    print(json.dumps(line), flush=True)


def max_over_ranks(x: float, world: int, device="cuda") -> float:
    """The slowest rank's time: all-reduce MAX over the process group (every
    rank takes part; world == 1 returns x)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_rate(world: int, npts: int, steps: int, seconds: float) -> float:
    """Whole-job Mpts*steps/s of `world` independent replicas, each doing
    `steps` steps of `npts` points, timed by the slowest rank."""
    return world * npts * steps / seconds / 1e6


def timed_steps(s, steps, warmup):
    """ms per step of `steps` graph replays on the solver's stream (CUDA events)."""
    import torch
    stream = torch.cuda.ExternalStream(s.stream())
    s.step(warmup)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step_async(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def fp32_refine_leg(n, pf, case, args, ms64, peak):
    """The FP32 + FP64-residual refinement form on the same workload: its own
    step time, per-kernel roofline and speed-up over the FP64 form, then its
    errors against the FP64 form of the same discrete problem (FD-modified
    k^2 in both) after the same number of steps."""
    from mhit36_b200 import Solver
    p, _, _ = workload_params(n, args.dt, "fp32")
    npts = n ** 3
    with Solver(n, p, precision="fp32", phase_field=pf) as s:
        s.set_fields(*case)
        ms = timed_steps(s, args.steps, args.warmup)
        prof = s.profile_step(3)
        d = s.step(0)  # diagnostics of the last step, max |div u| of its FP64 projection
        st32 = s.stats()
        f32 = s.get_fields()
    total = args.warmup + args.steps + 3
    with Solver(n, p, precision="fp64", phase_field=pf) as s:
        s.set_fields(*case)
        s.step(total)
        st64 = s.stats()
        f64 = s.get_fields()
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))  # noqa: E731
    errs = {name: rel(a, b) for name, a, b in zip(("u", "v", "w", "phi"), f32, f64) if b is not None}
    kb = kernel_bytes_per_point(n, pf, "fp32")
    step_bytes = ALGO_BYTES_STEP["fp32"][pf] * npts
    return {"ms_per_step": ms, "value": npts / (ms / 1e3) / 1e6, "unit": UNIT,
            "speedup_vs_fp64": ms64 / ms, "dtype": "f32 (FP64 residual, projection, reductions)",
            "per_kernel_ms": {k: round(v, 4) for k, v in prof.items()},
            "per_kernel_gbs": {k: round(kb[k] * npts / (v / 1e3) / 1e9, 1) for k, v in prof.items() if kb.get(k)},
            "step": {"algo_bytes_per_point": ALGO_BYTES_STEP["fp32"][pf],
                     "achieved": step_bytes / (ms / 1e3) / 1e9, "frac": step_bytes / (ms / 1e3) / 1e9 / peak},
            "errors_vs_fp64": {"after_steps": total, "max_div_fp64_projection": d["max_div"],
                               "ke_rel": abs(st32["ke"] / st64["ke"] - 1),
                               "dissipation_rel": abs(st32["dissipation"] / st64["dissipation"] - 1),
                               **{f"{k}_rel_to_max": v for k, v in errs.items()}},
            "k2_mode": "FD-modified (both forms, for the error comparison)", "status": d["status"]}


def serving_leg(nreq):
    """A bounded seeded stream through the served ensemble, both forms,
    against the same requests one at a time with the plain FP64 form."""
    from mhit36_b200.serve_bench import run_stream
    out = {}
    for line in run_stream(requests=nreq, forms=("fp64", "fp32")):
        out[line["form"]] = {k: line[k] for k in ("steps_per_s", "p50_latency_s", "p99_latency_s",
                                                   "vs_sequential_plain", "failed", "bitwise_same_as_alone",
                                                   "device_only_plain_steps_per_s")}
        out["sequential_plain"] = line["sequential_plain"]
        out["requests"] = line["requests"]
        out["total_steps"] = line["total_steps"]
        out["sizes"] = line["sizes"]
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    import torch.distributed as dist
    from mhit36_b200 import Solver

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    pf = not args.ns_only
    n = args.n
    p, case, recipe = workload(n, pf, args.dt, args.precision)
    s = Solver(n, p, precision=args.precision, phase_field=pf)
    s.set_fields(*case)
    stream = torch.cuda.ExternalStream(s.stream())

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (graph capture happens here)
    s.step(args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step_async(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    diag = s.diag()
    ms = max_over_ranks(ms, world)
    value = replicas_rate(world, n ** 3, args.steps, ms / 1e3)
    launches = s.launches_per_step() * args.steps

    # per-kernel durations (individually launched, CUDA events on the stream)
    prof = s.profile_step(3)
    kb = kernel_bytes_per_point(n, pf, args.precision)
    dominant = max(prof, key=lambda k: prof[k])
    peak, peak_kind = peaks()
    npts = n ** 3
    dom_bytes = kb[dominant] * npts
    achieved = dom_bytes / (prof[dominant] / 1e3) / 1e9
    step_ms = ms / args.steps
    step_bytes = ALGO_BYTES_STEP[args.precision][pf] * npts
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": (DRAM_BYTES_PER_POINT_FP64[dominant] * npts
                            if args.precision == "fp64" and pf and dominant in DRAM_BYTES_PER_POINT_FP64 else None),
                "traffic_source": "ncu dram__bytes_read+write at 256^3, scaled by points",
                "algo_bytes_per_launch": dom_bytes,
                "per_kernel_ms": {k: round(v, 4) for k, v in prof.items()},
                "per_kernel_gbs": {k: round(kb[k] * npts / (v / 1e3) / 1e9, 1) for k, v in prof.items() if kb[k]},
                "step": {"algo_bytes_per_point": ALGO_BYTES_STEP[args.precision][pf],
                         "achieved": step_bytes / (step_ms / 1e3) / 1e9,
                         "frac": step_bytes / (step_ms / 1e3) / 1e9 / peak}}

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        hb = [torch.empty(npts, dtype=torch.float64, pin_memory=True) for _ in range(4 if pf else 3)]
        for b, src in zip(hb, case):
            b.numpy()[:] = np.ascontiguousarray(src.T).reshape(-1)
        ptr = [b.data_ptr() for b in hb] + ([None] if not pf else [])
        barrier()
        torch.cuda.synchronize()
        # CUDA events on the solver's stream bracket the whole job: the uploads
        # and downloads run on that stream, and every host pause between its
        # operations shows as stream idle time inside the span
        f0, fa, fb, f1 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        f0.record(stream)
        s.set_fields_ptr(*ptr)
        fa.record(stream)
        for _ in range(args.steps):
            s.step(1)  # returns the step's diagnostics to the host
        fb.record(stream)
        s.get_fields_ptr(*ptr)
        f1.record(stream)
        f1.synchronize()
        torch.cuda.synchronize()
        el = max_over_ranks(f0.elapsed_time(f1) / 1e3, world)
        nf = len(hb)
        # where the time goes: the upload, the steps (each one waits for its
        # diagnostics on the host, so the gap to the device-timed step is the
        # cost of that synchronisation), the download
        steps_ms = fa.elapsed_time(fb) / args.steps
        e2e = {"value": replicas_rate(world, npts, args.steps, el), "unit": UNIT,
               "h2d_bytes_per_step": nf * npts * 8 / args.steps,
               "d2h_bytes_per_step": nf * npts * 8 / args.steps + 88,
               "ms_per_step": el / args.steps * 1e3,
               "upload_ms": round(f0.elapsed_time(fa), 3), "download_ms": round(fb.elapsed_time(f1), 3),
               "step_with_diag_readback_ms": round(steps_ms, 4),
               "diag_sync_overhead_ms": round(steps_ms - step_ms, 4)}

    mem_bytes = s.memory_bytes()
    s.close()
    # the library's two other forms, on one GPU only: the FP32
    # refinement form on the same workload, and a bounded served stream
    fp32 = serving = None
    if world == 1 and args.precision == "fp64" and not args.no_fp32:
        fp32 = fp32_refine_leg(n, pf, case, args, step_ms, peak)
    if world == 1 and not args.no_serve and args.serve_requests > 0:
        serving = serving_leg(args.serve_requests)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, st, thr, el = cpu_oracle_rate(n, pf, args.dt, (p, case), max_seconds=20.0)
        cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{n}^3 NS{'+ACDI' if pf else ''} FP64, {st} oracle step(s), {el:.1f} s"}

    if rank == 0:
        line = {
            "metric": metric_name(n, pf, args.precision),
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
            "data": "synthetic (seeded random-phase velocity E(k)~k^4exp(-2(k/4)^2), seeded drops)",
            "config": {"workload": f"{n}^3 NS{'+ACDI' if pf else ''} plain {args.precision} form, "
                                   f"{recipe[0] if pf else 0} drops r in [{recipe[1]},{recipe[2]}]",
                       "n": n, "phase_field": pf, "precision": args.precision, "dt": args.dt, "mu": 6e-3,
                       "lin_force": 0.1, "parallelism": f"replicas x{world}",
                       "l2": "state larger than L2 (resident fields ~{:.0f} GB)".format(mem_bytes / 1e9)},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "status": diag["status"], "umax": diag["umax"], "cfl": diag["cfl"],
            "fp32_refine": fp32, "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
