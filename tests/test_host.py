"""CPU tests of the host side: input.inp, field files, seeded inputs, and the
C ABI library's exports (no compute call needs a GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

INPUT_INP_REF_STYLE = """0           ! fresh start=0 restart =1
0           ! iteration to start from (fresh start 0 otherwise different)
20000       ! Final time step
1000        ! Saving frequency
0           ! inflow condition (0=Taylor green, 1=read from fields)
0           ! phase-field initial condition (0=circular drop, 1=read from fields)
0.0002      ! dt for the simulation
0.006       ! mu (viscosity)
1.000       ! density
0.0         ! A forcing parameter (ABC forcing)
0.0         ! B forcing parameter (ABC forcing)
0.0         ! C forcing parameter (ABC forcing)
2.0         ! Forced wavenumber (ABC forcing)
0.5         ! Initial drop radius for phase-field
1.0d0       ! Surface tension
1.0         ! Ratio eps/dx
"""


def test_read_input_reference_format(tmp_path):
    from mhit36_b200.config import read_input
    p = tmp_path / "input.inp"
    p.write_text(INPUT_INP_REF_STYLE)
    prm = read_input(str(p))
    assert (prm.restart, prm.tstart, prm.tfin, prm.dump, prm.inflow, prm.inphi) == (0, 0, 20000, 1000, 0, 0)
    assert (prm.dt, prm.mu, prm.rho) == (0.0002, 0.006, 1.0)
    assert (prm.f1, prm.f2, prm.f3, prm.k0) == (0.0, 0.0, 0.0, 2.0)
    assert (prm.radius, prm.sigma, prm.epsr) == (0.5, 1.0, 1.0)  # "1.0d0" is a Fortran double literal
    assert prm.lin_force == 0.0
    # optional 17th line: linear forcing
    p.write_text(INPUT_INP_REF_STYLE + "0.1   ! linear forcing A\n")
    assert read_input(str(p)).lin_force == 0.1


def test_input_roundtrip_and_derived(tmp_path):
    from mhit36_b200.config import InputParams, read_input, write_input
    prm = InputParams(tfin=200, dt=1e-3, mu=6e-3, sigma=0.5, lin_force=0.1, inflow=1, inphi=1)
    write_input(str(tmp_path / "input.inp"), prm)
    back = read_input(str(tmp_path / "input.inp"))
    for k in ("tfin", "dt", "mu", "sigma", "lin_force", "inflow", "inphi", "rho", "epsr"):
        assert getattr(back, k) == getattr(prm, k)
    d = prm.derived(128)
    assert d["dx"] == 8.0 * np.arctan(1.0) / 127  # multi/readinput.f90:37
    assert d["enum"] == float(np.float32(1e-16))


def test_field_file_roundtrip(tmp_path):
    from mhit36_b200 import fields
    n = 8
    a = np.random.default_rng(0).standard_normal((n, n, n))
    path = str(tmp_path / "u.dat")
    fields.write_field(path, a)
    raw = np.fromfile(path, dtype="<f8")
    assert raw.size == n ** 3
    assert raw[1] == a[1, 0, 0] and raw[n] == a[0, 1, 0] and raw[n * n] == a[0, 0, 1]  # x fastest
    assert np.array_equal(fields.read_field(path, n), a)
    with pytest.raises(ValueError):
        fields.read_field(path, n + 1)
    assert fields.output_name("out", 5, 12) == os.path.join("out", "phi_00000012.dat")


def test_random_velocity_properties():
    from mhit36_b200 import fields
    n = 32
    u, v, w = fields.random_velocity(n, seed=n)
    for f in (u, v, w):
        assert abs(f.mean()) < 1e-14
    rms = np.sqrt((np.mean(u ** 2) + np.mean(v ** 2) + np.mean(w ** 2)) / 3)
    assert abs(rms - 1.0) < 1e-12
    # solenoidal in index space once the half-cell stagger is undone
    k = np.fft.fftfreq(n, 1.0 / n)
    U = np.fft.fftn(u) * np.exp(1j * np.pi * k / n)[:, None, None]
    V = np.fft.fftn(v) * np.exp(1j * np.pi * k / n)[None, :, None]
    W = np.fft.fftn(w) * np.exp(1j * np.pi * k / n)[None, None, :]
    div = k[:, None, None] * U + k[None, :, None] * V + k[None, None, :] * W
    assert np.max(np.abs(div)) / np.max(np.abs(U)) < 1e-10
    # seeded: same seed, same field
    u2, _, _ = fields.random_velocity(n, seed=n)
    assert np.array_equal(u, u2)


def test_drop_field_recipe():
    from mhit36_b200 import fields
    n = 64
    c, r = fields.place_drops(n, seed=n + 1, ndrops=4, rmin=0.4, rmax=0.6)
    dx = fields.grid_dx(n)
    period = n * dx
    for a in range(4):
        for b in range(a):
            d = c[a] - c[b]
            d -= period * np.round(d / period)
            assert np.linalg.norm(d) > r[a] + r[b] + 4 * dx
    phi = fields.drop_field(n, c, r)
    assert phi.min() >= 0 and phi.max() <= 1
    vol = phi.sum() * dx ** 3
    # 0.5(1 - tanh((d-r)/2eps)) = 1/(1+exp((d-r)/eps)): volume (4pi/3)(r^3 + pi^2 eps^2 r)
    eps = dx
    ref = 4 / 3 * np.pi * (r ** 3 + np.pi ** 2 * eps ** 2 * r).sum()
    assert abs(vol / ref - 1) < 0.02


def test_centred_drop_matches_reference_formula():
    from mhit36_b200 import fields
    n = 16
    phi = fields.centred_drop(n, 0.5)
    dx = 2 * np.pi / (n - 1)
    x = np.arange(n) * dx
    i, j, k = 3, 7, 11
    pos = (x[i] - np.pi) ** 2 + (x[j] - np.pi) ** 2 + (x[k] - np.pi) ** 2
    assert phi[i, j, k] == 0.5 * (1 - np.tanh((np.sqrt(pos) - 0.5) / 2 / dx))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "mhit.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mhit_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    from mhit36_b200 import capi
    lib = capi.load_library()
    names = _header_functions()
    assert set(capi.HEADER_SYMBOLS) <= set(names)
    for name in names:
        assert hasattr(lib, name), name
    # pure host calls, no GPU needed
    assert lib.mhit_strerror(capi.MHIT_ERR_CFL).decode() == "CFL above the limit"
    assert lib.mhit_size_supported(512) == 1
    assert lib.mhit_size_supported(500) == 0
    p = capi.MhitParams()
    lib.mhit_default_params(ctypes.byref(p))
    assert (p.dt, p.mu, p.tfin, p.cfl_limit) == (0.0002, 0.006, 20000, 7.0)  # multi/input.inp


def test_params_struct_layout_matches_header():
    """The ctypes mirror and the C struct agree on size (checked with gcc)."""
    import subprocess
    import tempfile
    from mhit36_b200 import capi
    src = '#include "mhit.h"\n#include <stdio.h>\nint main(){printf("%zu %zu\\n", sizeof(mhit_params), sizeof(mhit_diag));return 0;}\n'
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        a, b = map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split())
    assert a == ctypes.sizeof(capi.MhitParams)
    assert b == ctypes.sizeof(capi.MhitDiag)


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from mhit36_b200 import Solver, MhitError
    from mhit36_b200.ensemble import Ensemble
    with pytest.raises(MhitError):
        Solver(32, phase_field=False)
    with pytest.raises(MhitError):  # no silent CPU fallback for the served ensemble either
        Ensemble()


def test_vtk_export_format(tmp_path):
    from mhit36_b200 import vtk
    n = 8
    rng = np.random.default_rng(3)
    u = rng.standard_normal((n, n, n))
    phi = rng.random((n, n, n))
    path = vtk.write_vtk(vtk.vtk_name(str(tmp_path), 42), {"u": u, "phi": phi})
    assert path.endswith("OUTPAR_00000042.vtk")
    raw = open(path, "rb").read()
    assert raw.startswith(b"# vtk DataFile Version 3.0\nPhase field\nBINARY\nDATASET RECTILINEAR_GRID\n")
    assert b"DIMENSIONS        8       8       8\n" in raw  # Fortran i8 fields
    assert b"POINT_DATA              512\n" in raw          # i16
    back = vtk.read_vtk(path)
    assert back["dims"] == [n, n, n]
    assert np.array_equal(back["u"], u.astype(np.float32))
    assert np.array_equal(back["phi"], phi.astype(np.float32))
    assert abs(float(back["coords"][0][-1]) - 2 * np.pi) < 1e-6  # x(n) = 2 pi on the reference grid


def test_clock_sampler_reports_rows_of_the_timed_region(tmp_path, monkeypatch):
    """bench.py's clock record, against a stand-in nvidia-smi that prints one
    CSV row per period (the real one only exists on the GPU box)."""
    import sys
    import time
    sys.path.insert(0, ROOT)
    import bench
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\nsleep 0.3\nwhile true; do\n"
                    "  echo '0, 1965, 1965, 700.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active'\n"
                    "  sleep 0.05\ndone\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    s = bench.ClockSampler(0)
    t0 = time.time()
    s.start()
    assert time.time() - t0 >= 0.25  # waited for the sampler's first row
    time.sleep(0.2)
    rec = s.stop()
    assert rec["samples"] >= 1 and rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap"]


def test_integration_c_examples_compile_and_link(tmp_path):
    """The C snippets of INTEGRATION.md compile against include/mhit.h and
    every function they call resolves in libmhit.so (linked, not run)."""
    import subprocess
    from mhit36_b200 import capi
    if not os.path.exists(capi.LIB_PATH):
        pytest.skip("libmhit.so not built")
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\n(.*?)```", text, re.S)
    assert len(blocks) >= 2
    body = "\n".join(b.replace('#include "mhit.h"', "") for b in blocks)
    src = ('#include "mhit.h"\n#include <stdint.h>\n'
           "int example(double* u, double* v, double* w, double* phi) {\n" + body + "\nreturn rc;\n}\n"
           "int main(void) { return 0; }\n")
    c = tmp_path / "example.c"
    c.write_text(src)
    lib_dir = os.path.dirname(capi.LIB_PATH)
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-Wno-unused-variable", "-I",
                        os.path.join(ROOT, "include"), str(c), "-o", str(tmp_path / "example"), "-L", lib_dir,
                        "-lmhit", "-Wl,--unresolved-symbols=ignore-in-shared-libs"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_integration_python_examples_parse_and_name_real_api():
    """The Python snippets of INTEGRATION.md parse, and the package names
    they import exist."""
    import ast
    import importlib
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```python\n(.*?)```", text, re.S)
    assert blocks
    for src in blocks:
        tree = ast.parse(src)
        for node in ast.walk(tree):
            if isinstance(node, ast.ImportFrom) and node.module and node.module.startswith("mhit36_b200"):
                mod = importlib.import_module(node.module)
                for alias in node.names:
                    assert hasattr(mod, alias.name) or importlib.util.find_spec(
                        f"{node.module}.{alias.name}") is not None, (node.module, alias.name)


def test_serve_stream_follows_its_recipe():
    """The served-ensemble stream: N over {64,96,128,192,256}, nu in
    [3e-3, 1e-2], ACDI on for exactly half, 2-16 drops, 50-500 steps,
    seeded (the same seed gives the same stream)."""
    from mhit36_b200 import serve_bench
    sizes = [64, 96, 128, 192, 256]
    reqs, gaps = serve_bench.make_stream(256, 2024, sizes)
    again, gaps2 = serve_bench.make_stream(256, 2024, sizes)
    assert reqs == again and np.array_equal(gaps, gaps2)
    assert {r["n"] for r in reqs} == set(sizes)
    assert sum(r["pf"] for r in reqs) == 128
    assert all(3e-3 <= r["nu"] <= 1e-2 and 2 <= r["ndrops"] <= 16 and 50 <= r["steps"] <= 500 for r in reqs)
    assert len(gaps) == 256 and np.all(gaps > 0)
    # the same replay of FIFO queueing the benchmark uses for the one-at-a-time arm
    done, lat = serve_bench.replay_fifo(np.array([0.0, 0.5, 0.6]), np.array([1.0, 1.0, 1.0]))
    assert np.allclose(done, [1.0, 2.0, 3.0]) and np.allclose(lat, [1.0, 1.5, 2.4])
