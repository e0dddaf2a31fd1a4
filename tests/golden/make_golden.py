"""Generate the committed golden fixtures under tests/golden/.

1. val_taylor_green.json -- the reference's own validation series
   (aroccon/MHIT36 val/cudec_*_{ab,eulero}.txt, val/single_*_ab.txt): viscous
   dissipation of the Taylor-Green vortex (nu = 6.25e-4, dt = 2e-4, rho = 1,
   no forcing, phase field off; val/comparison_diss.m:5,10) every 0.2 time
   units, i.e. every 1000 steps.  Read from the reference checkout given by
   --reference (or the MHIT36_REFERENCE environment variable) and copied
   verbatim as numbers.

2. (with --oracle) oracle_taylor_green_128.json -- the CPU oracle's own
   dissipation on the same case at t = 0, 0.2, 0.4 (1000 and 2000 steps at
   128^3), recording how closely the oracle reproduces the reference's series.
   Takes a few minutes on 8 cores.

    python tests/golden/make_golden.py --reference DIR [--oracle]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

SERIES = ["cudec_128_ab", "cudec_128_eulero", "cudec_256_ab", "cudec_256_eulero", "cudec_512_ab",
          "cudec_512_eulero", "cudec_1024_ab", "single_128_ab", "single_256_ab", "single_512_ab"]


def extract_val(refdir: str) -> dict:
    out = {"source": "aroccon/MHIT36 val/*.txt", "case": {"flow": "Taylor-Green", "nu": 6.25e-4, "dt": 2e-4,
                                                           "rho": 1.0, "steps_per_sample": 1000},
           "series": {}}
    for name in SERIES:
        path = os.path.join(refdir, "val", name + ".txt")
        rows = []
        with open(path) as f:
            for line in f:
                tok = line.replace(",", " ").split()
                if len(tok) >= 2:
                    rows.append([float(tok[0]), float(tok[1])])
        out["series"][name] = rows
    return out


def oracle_check(steps=(1000, 2000)) -> dict:
    sys.path.insert(0, ROOT)
    from oracle import Oracle, dissipation
    from mhit36_b200 import fields
    n = 128
    u, v, w = fields.taylor_green(n)
    o = Oracle(n, dt=2e-4, mu=6.25e-4, rho=1.0, phase_field=0)
    o.set_fields(u, v, w)
    res = {"n": n, "samples": [[0.0, dissipation(u, v, w, 6.25e-4)]]}
    done = 0
    for s in steps:
        o.step(s - done)
        done = s
        uu, vv, ww, _ = o.get_fields()
        res["samples"].append([s * 2e-4, dissipation(uu, vv, ww, 6.25e-4)])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MHIT36_REFERENCE"),
                    help="checkout of aroccon/MHIT36 (or set MHIT36_REFERENCE)")
    ap.add_argument("--oracle", action="store_true")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give the reference checkout with --reference DIR or MHIT36_REFERENCE")
    val = extract_val(a.reference)
    with open(os.path.join(HERE, "val_taylor_green.json"), "w") as f:
        json.dump(val, f, indent=1)
    if a.oracle:
        res = oracle_check()
        with open(os.path.join(HERE, "oracle_taylor_green_128.json"), "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
