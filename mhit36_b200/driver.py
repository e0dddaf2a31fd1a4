"""The reference's main program (multi/main.f90:3-987) over libmhit.

    python -m mhit36_b200.driver --n 128 [--dir RUN] [--precision fp64] [--ns-only]

Runs in directory RUN exactly as the reference runs in multi/: reads
``input.inp`` (multi/readinput.f90), initialises the fields (Taylor-Green or
``input/*.dat``; one centred drop or ``input/phi.dat``; or the restart files
``output/*_<tstart>.dat``; multi/main.f90:218-293), writes the initial fields
(multi/main.f90:296-305), then loops t = tstart+1..tfin: one step, the CFL
print and guard (multi/main.f90:942-946), and ``output/*_<t>.dat`` every
``dump`` steps (multi/main.f90:960-971).  The grid size is an argument because
the reference fixes it at compile time (multi/module.f90:2).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

from . import fields
from .capi import MHIT_ERR_CFL, MhitError
from .config import read_input
from .solver import Solver


def initial_fields(n: int, p, workdir: str, phase_field: bool):
    indir = os.path.join(workdir, "input")
    if p.inflow == 0:
        u, v, w = fields.taylor_green(n, p.grid_mode)
    else:
        u = fields.read_field(os.path.join(indir, "u.dat"), n)
        v = fields.read_field(os.path.join(indir, "v.dat"), n)
        w = fields.read_field(os.path.join(indir, "w.dat"), n)
    phi = None
    if phase_field:
        if p.inphi == 0:
            phi = fields.centred_drop(n, p.radius, p.epsr, p.grid_mode)
        else:
            phi = fields.read_field(os.path.join(indir, "phi.dat"), n)
    return u, v, w, phi


def run(n: int, workdir: str = ".", precision: str = "fp64", phase_field: bool = True, verbose: bool = True,
        log=print):
    p = read_input(os.path.join(workdir, "input.inp"))
    outdir = os.path.join(workdir, "output")
    os.makedirs(outdir, exist_ok=True)
    s = Solver(n, p, precision=precision, phase_field=phase_field)
    try:
        if p.restart == 0:
            if verbose:
                log("Initialize velocity field (fresh start)")
            s.set_fields(*initial_fields(n, p, workdir, phase_field))
            if verbose:
                log("Save initial fields")
            s.save(outdir, p.tstart)
        else:
            if verbose:
                log(f"Initialize velocity field (from output folder), iteration: {p.tstart}")
            s.load(outdir, p.tstart)
        history = []
        for t in range(p.tstart + 1, p.tfin + 1):
            t0 = time.perf_counter()
            if verbose:
                log(f"Time step {t} of {p.tfin}")
            d = s.step(1, raise_on_error=False)
            history.append(d)
            if verbose:
                log(f"CFL (max among tasks) {d['cfl']:.15e}")
                log(f" Time elapsed = {1000 * (time.perf_counter() - t0):6.1f} ms")
            if d["rc"] == MHIT_ERR_CFL:
                log("CFL limit exceeded: stop")
                break
            if d["rc"]:
                raise MhitError(d["rc"], f"step {t}")
            if t % p.dump == 0:
                if verbose:
                    log("Saving output files")
                s.save(outdir, t)
        return history
    finally:
        s.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, required=True)
    ap.add_argument("--dir", default=".")
    ap.add_argument("--precision", default="fp64")
    ap.add_argument("--ns-only", action="store_true")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    run(a.n, a.dir, a.precision, not a.ns_only, verbose=not a.quiet)
    return 0


if __name__ == "__main__":
    sys.exit(main())
