"""``input.inp`` parameters, mirroring the reference's readinput.

The reference reads 16 positional lines (multi/readinput.f90:13-31) and
derives dx, dxi, ddxi, rhoi, eps, epsi, enum from them
(multi/readinput.f90:34-43).  This module reads the same file.  An optional
17th line carries the linear-forcing coefficient A (rhs += A*u), which the
reference does not have; a 16-line file therefore reads exactly as the
reference reads it, with A = 0.
"""
from __future__ import annotations

import dataclasses
import math
import re

_FIELDS = [
    ("restart", int), ("tstart", int), ("tfin", int), ("dump", int),
    ("inflow", int), ("inphi", int),
    ("dt", float), ("mu", float), ("rho", float),
    ("f1", float), ("f2", float), ("f3", float), ("k0", float),
    ("radius", float), ("sigma", float), ("epsr", float),
]

_COMMENTS = [
    "fresh start=0 restart =1", "iteration to start from", "Final time step",
    "Saving frequency", "inflow condition (0=Taylor green, 1=read from fields)",
    "phase-field initial condition (0=circular drop, 1=read from fields)",
    "dt for the simulation", "mu (viscosity)", "density",
    "A forcing parameter (ABC forcing)", "B forcing parameter (ABC forcing)",
    "C forcing parameter (ABC forcing)", "Forced wavenumber (ABC forcing)",
    "Initial drop radius for phase-field", "Surface tension", "Ratio eps/dx",
]


@dataclasses.dataclass
class InputParams:
    """The 16 reference parameters plus this implementation's switches."""

    restart: int = 0
    tstart: int = 0
    tfin: int = 100
    dump: int = 1000
    inflow: int = 1
    inphi: int = 1
    dt: float = 1e-3
    mu: float = 6e-3
    rho: float = 1.0
    f1: float = 0.0
    f2: float = 0.0
    f3: float = 0.0
    k0: float = 2.0
    radius: float = 0.5
    sigma: float = 0.5
    epsr: float = 1.0
    # extensions (not in the reference)
    lin_force: float = 0.0   # optional input.inp line 17
    k2_mode: int = 0         # 0 spectral k^2 (reference), 1 FD-modified
    grid_mode: int = 0       # 0 dx = 2pi/(N-1) (reference), 1 dx = 2pi/N
    cfl_limit: float = 7.0   # multi/main.f90:945
    tanh_identity: int = 1   # 1: tanh(psi/2eps) as (2phi-1)/(1+2enum), its exact value; 0: FP64 tanh
    phi_floor: int = 1       # 1: psi from max(min(phi,1),0); 0: min(phi,1) as the reference

    # derived constants, multi/readinput.f90:34-43
    def derived(self, n: int) -> dict:
        twopi = 8.0 * math.atan(1.0)
        dx = twopi / n if self.grid_mode == 1 else twopi / (n - 1)
        import numpy as np
        return {
            "lx": twopi, "dx": dx, "dxi": 1.0 / dx, "ddxi": 1.0 / dx / dx,
            "rhoi": 1.0 / self.rho, "eps": self.epsr * dx, "epsi": 1.0 / (self.epsr * dx),
            "enum": float(np.float32(1.0e-16)),
        }


_NUM = re.compile(r"^\s*([-+0-9.eEdD]+)")


def _parse_value(line: str, typ):
    m = _NUM.match(line)
    if not m:
        raise ValueError(f"input.inp: cannot read a number from {line!r}")
    tok = m.group(1).replace("d", "e").replace("D", "e")
    return int(float(tok)) if typ is int else float(tok)


def read_input(path: str = "input.inp") -> InputParams:
    """Read ``input.inp`` as multi/readinput.f90:13-31 does (list-directed,
    one value per line, trailing text ignored), plus the optional line 17."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if ln.strip()]
    if len(lines) < len(_FIELDS):
        raise ValueError(f"input.inp: expected at least 16 lines, found {len(lines)}")
    vals = {name: _parse_value(lines[i], typ) for i, (name, typ) in enumerate(_FIELDS)}
    p = InputParams(**vals)
    if len(lines) > 16:
        p.lin_force = _parse_value(lines[16], float)
    return p


def write_input(path: str, p: InputParams) -> None:
    """Write a 16-line reference-compatible file (+ line 17 when A != 0)."""
    out = []
    for (name, typ), com in zip(_FIELDS, _COMMENTS):
        val = getattr(p, name)
        s = str(int(val)) if typ is int else repr(float(val))
        out.append(f"{s:<12}! {com}")
    if p.lin_force != 0.0:
        out.append(f"{repr(float(p.lin_force)):<12}! linear forcing A (extension, rhs += A*u)")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
