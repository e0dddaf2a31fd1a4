"""A small seeded NS+ACDI case for profiling one kernel of the step.

    python -m mhit36_b200.profile_case N FORM STEPS     (FORM: fp64 or fp32)

Builds the seeded velocity and drop field at N^3 (64 drops of radius
0.2-0.35 from 512^3 up, else 8 of radius 0.4-0.6), creates a Solver of that
form (the FP32 refinement form with the FD-modified k^2), and advances STEPS
steps through the C ABI.  Under ncu, select one kernel with -k and skip the
first step's launches with -s.
"""
from __future__ import annotations

import sys

from . import fields
from .config import InputParams
from .solver import Solver


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    n, form, steps = int(argv[0]), argv[1], int(argv[2])
    p = InputParams(dt=2e-4, mu=6e-3, rho=1.0, sigma=0.5, epsr=1.0, lin_force=0.1,
                    k2_mode=1 if form == "fp32" else 0)
    big = n >= 512
    case = fields.seeded_case(n, ndrops=64 if big else 8, rmin=0.2 if big else 0.4, rmax=0.35 if big else 0.6)
    with Solver(n, p, precision=form, phase_field=True) as s:
        s.set_fields(*case)
        d = s.step(steps)
    print(f"{n}^3 {form}: {steps} steps, status {d['status']}, umax {d['umax']:.6f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
