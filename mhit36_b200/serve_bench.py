"""Served-ensemble benchmark: a seeded Poisson-arrival stream of independent
HIT / drop simulations of uneven grid sizes, served (a) one at a time with the
plain form and (b) by the ensemble (continuous batching), in the FP64 and the
FP32-refinement forms.

    python -m mhit36_b200.serve_bench [--requests 256] [--forms fp64,fp32] [--slots 8] [--load 4]

Stream (seeded numpy PCG64): N uniform over {64,96,128,192,256}; nu uniform in
[3e-3, 1e-2]; ACDI on for exactly half of the requests, with 2-16 drops of
radius 0.3-0.5; 50-500 steps; dt = 2e-4 (inside the explicit ACDI limit
Umax*dt/dx < 1/6 at every size); Poisson arrivals whose rate is `--load`
times the rate the one-at-a-time plain form can serve (the default 4 keeps
both servers saturated, so aggregate steps/s measures capacity).  Velocity
fields are seeded per grid size; drops per request.  Inputs are generated
before timing in the C ABI's raw layout (x fastest, as the reference's input
files hold them), so neither arm times a numpy transpose.

One JSON line per form: aggregate steps/s = total steps / (last completion -
first arrival); p50/p99 request latency = completion - arrival.  The
one-at-a-time baseline is measured per request (create, upload, steps,
download, destroy) and its queueing under the same arrivals is replayed
exactly (FIFO, one request at a time).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from mhit36_b200 import Solver, fields  # noqa: E402
from mhit36_b200.config import InputParams  # noqa: E402
from mhit36_b200.ensemble import Ensemble  # noqa: E402


def make_stream(nreq, seed, sizes):
    rng = np.random.Generator(np.random.PCG64(seed))
    pf = np.array([True] * (nreq // 2) + [False] * (nreq - nreq // 2))
    rng.shuffle(pf)
    reqs = []
    for i in range(nreq):
        n = int(sizes[rng.integers(len(sizes))])
        reqs.append({"i": i, "n": n, "nu": float(rng.uniform(3e-3, 1e-2)), "pf": bool(pf[i]),
                     "ndrops": int(rng.integers(2, 17)), "steps": int(rng.integers(50, 501)),
                     "seed": int(rng.integers(1 << 30))})
    gaps = rng.exponential(1.0, size=nreq)  # scaled to the target rate later
    return reqs, gaps


def raw(a):
    """[i,j,k] array -> the C ABI's raw layout (x fastest), as input files hold it."""
    return None if a is None else np.ascontiguousarray(np.asarray(a).T).reshape(-1)


def build_inputs(reqs):
    vel = {}
    for r in reqs:
        n = r["n"]
        if n not in vel:
            vel[n] = tuple(raw(a) for a in fields.random_velocity(n, n))
        phi = None
        if r["pf"]:
            c, rad = fields.place_drops(n, r["seed"], r["ndrops"], 0.3, 0.5)
            phi = raw(fields.drop_field(n, c, rad))
        r["fields"] = (*vel[n], phi)


def params(r, precision):
    return InputParams(dt=2e-4, mu=r["nu"], rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1,
                       k2_mode=1 if precision == "fp32" else 0)


def sequential(reqs):
    """Each request alone with the plain FP64 form: service times (s)."""
    out = []
    for r in reqs:
        t0 = time.perf_counter()
        with Solver(r["n"], params(r, "fp64"), precision="fp64", phase_field=r["pf"]) as s:
            s.set_fields(*r["fields"])
            s.step(r["steps"])
            res = s.get_fields()
        out.append(time.perf_counter() - t0)
        r["seq_result"] = res if r["n"] <= 64 else None
    return out


def replay_fifo(arrivals, service):
    done, lat, t = [], [], 0.0
    for a, sv in zip(arrivals, service):
        start = max(a, t)
        t = start + sv
        done.append(t)
        lat.append(t - a)
    return np.array(done), np.array(lat)


def serve(reqs, arrivals, precision, slots):
    order = np.argsort(arrivals)
    with Ensemble(slots_per_class=slots) as ens:
        t0 = time.perf_counter()
        nxt, ids = 0, {}
        while True:
            now = time.perf_counter() - t0
            while nxt < len(order) and arrivals[order[nxt]] <= now:
                r = reqs[order[nxt]]
                ids[r["i"]] = ens.submit(r["n"], params(r, precision), *r["fields"], nsteps=r["steps"],
                                         precision=precision, keep=True, borrow=True)
                nxt += 1
            pending = ens.progress()
            to_next = arrivals[order[nxt]] - (time.perf_counter() - t0) if nxt < len(order) else None
            if pending == 0:
                if nxt >= len(order):
                    break
                time.sleep(max(0.0, to_next))
            else:  # sleep until the ensemble has work for a round, or the next arrival
                ens.wait(0.01 if to_next is None else max(0.0, min(0.01, to_next)))
        lat, done, subm, fails, same = [], [], [], 0, []
        for r in reqs:
            q = ens.query(ids[r["i"]])
            if q["state"] != "done":
                fails += 1
            done.append(q["t_done"])
            subm.append(q["t_submit"])
            lat.append(q["t_done"] - q["t_submit"])
            if precision == "fp64" and r.get("seq_result") is not None:
                got = ens.result(ids[r["i"]])
                same.append(all((a is None and b is None) or np.array_equal(a, b)
                                for a, b in zip(got, r["seq_result"])))
            ens.release(ids[r["i"]])
        st = ens.stats()
    first = float(np.min(subm))
    return np.array(done), np.array(lat), fails, same, st, first


def run_stream(requests=256, forms=("fp64", "fp32"), sizes=(64, 96, 128, 192, 256), slots=8, load=4.0,
               seed=2024, log=None):
    """Serve one seeded stream one request at a time (plain FP64) and through
    the ensemble in each form; returns one result dict per form."""
    reqs, gaps = make_stream(requests, seed, list(sizes))
    t = time.perf_counter()
    build_inputs(reqs)
    gen_s = time.perf_counter() - t
    step_s = {}  # plain FP64 device time per step of each (n, ACDI) class
    # warm the library: module loading of every kernel the stream uses is a
    # one-time process cost, not part of a request (tile autotuning is, and
    # the timed ensembles below start with fresh classes)
    for n in sizes:
        case = fields.random_velocity(n, 1)
        phi = fields.drop_field(n, *fields.place_drops(n, 1, 2, 0.3, 0.5))
        for pf in (False, True):
            with Solver(n, params(reqs[0], "fp64"), phase_field=pf) as s:
                s.set_fields(*case, phi if pf else None)
                s.step(2)
                t = time.perf_counter()
                s.step(20)  # returns after the device finished (diagnostics read back)
                step_s[(n, pf)] = (time.perf_counter() - t) / 20
    with Ensemble(slots_per_class=slots) as ens:
        for n in sizes:
            case = [raw(x) for x in fields.random_velocity(n, 1)]
            phi = raw(fields.drop_field(n, *fields.place_drops(n, 1, 2, 0.3, 0.5)))
            for form in forms:
                for pf in (False, True):
                    ens.submit(n, params(reqs[0], form), *case, phi if pf else None, nsteps=2, precision=form)
        ens.run()
    service = np.array(sequential(reqs))
    total_steps = sum(r["steps"] for r in reqs)
    # what the stream costs the device alone, one request after another: the
    # bound a server reaches by hiding all host work without batching gains
    device_s = sum(r["steps"] * step_s[(r["n"], r["pf"])] for r in reqs)
    rate = load * len(reqs) / service.sum()  # requests per second offered
    arrivals = np.cumsum(gaps) / rate
    arrivals -= arrivals[0]
    sdone, slat = replay_fifo(arrivals, service)
    seq = {"steps_per_s": total_steps / (sdone.max() - arrivals.min()),
           "busy_steps_per_s": total_steps / service.sum(),
           "p50_s": float(np.percentile(slat, 50)), "p99_s": float(np.percentile(slat, 99))}
    out = []
    for form in forms:
        done, lat, fails, same, st, first = serve(reqs, arrivals, form, slots)
        agg = total_steps / (np.max(done) - first)
        line = {"metric": "served ensemble: aggregate steps/s and request latency", "form": form,
                "requests": len(reqs), "total_steps": total_steps, "offered_load_vs_sequential": load,
                "steps_per_s": agg, "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)), "failed": fails,
                "vs_sequential_plain": agg / seq["steps_per_s"], "sequential_plain": seq,
                "bitwise_same_as_alone": (sum(same), len(same)) if same else None,
                "ensemble": {"slots_per_class": slots, "classes": st["classes"], "rounds": st["rounds"],
                             "graph_launches": st["graph_launches"]},
                "sizes": list(sizes), "input_generation_s": gen_s,
                "device_only_plain_steps_per_s": total_steps / device_s}
        if log:
            log(line)
        out.append(line)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--forms", default="fp64,fp32")
    ap.add_argument("--sizes", default="64,96,128,192,256")
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--load", type=float, default=4.0)
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args()
    run_stream(a.requests, a.forms.split(","), [int(x) for x in a.sizes.split(",")], a.slots, a.load, a.seed,
               log=lambda line: print(json.dumps(line), flush=True))


if __name__ == "__main__":
    main()
