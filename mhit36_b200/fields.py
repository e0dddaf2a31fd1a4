"""Field files in the reference's raw format, and the seeded initial fields.

File format (multi/readwrite.f90:1-96 writefield, :107-207 readfield,
:218-317 readfield_restart): one raw little-endian float64 array of
nx*ny*nz values per field, Fortran order (x fastest), no header and no halo
cells.  Output names are ``output/{u,v,w,p,phi}_%08d.dat``
(multi/readwrite.f90:41); inputs are ``input/{u,v,w,phi}.dat``
(multi/readwrite.f90:146).

Arrays in this package are numpy arrays indexed ``a[i, j, k]`` (x, y, z).  A
C-contiguous array ``a.T`` (shape (nz, ny, nx)) has the same bytes as the
file, so the conversion is a transpose.

The seeded generator writes the inputs that both this implementation and the
oracle start from (through ``inflow=1``/``inphi=1``).  The reference itself has
only a Taylor-Green field and one centred drop (multi/main.f90:220-233,
266-278); random-phase turbulence and N seeded drops are this project's.
"""
from __future__ import annotations

import math
import os

import numpy as np

FIELD_NAMES = {1: "u", 2: "v", 3: "w", 4: "p", 5: "phi"}


def write_field(path: str, a: np.ndarray) -> None:
    a = np.asarray(a, dtype="<f8")
    np.asfortranarray(a).ravel(order="F").tofile(path)


def read_field(path: str, n: int) -> np.ndarray:
    flat = np.fromfile(path, dtype="<f8")
    if flat.size != n ** 3:
        raise ValueError(f"{path}: expected {n**3} float64 values, found {flat.size}")
    return flat.reshape((n, n, n), order="F")


def output_name(outdir: str, fieldn: int, t: int) -> str:
    return os.path.join(outdir, f"{FIELD_NAMES[fieldn]}_{t:08d}.dat")


def grid_dx(n: int, grid_mode: int = 0) -> float:
    twopi = 8.0 * math.atan(1.0)
    return twopi / n if grid_mode == 1 else twopi / (n - 1)


def taylor_green(n: int, grid_mode: int = 0):
    """Taylor-Green velocity of multi/main.f90:222-232 on x(i)=(i-1)dx.

    The global interior index g = 1..N maps to x(g); the reference's
    ``jg = piX%lo(2)+j-1`` with halo'd j is taken to mean that."""
    dx = grid_dx(n, grid_mode)
    x = np.arange(n) * dx
    sx, cx = np.sin(x), np.cos(x)
    u = sx[:, None, None] * cx[None, :, None] * cx[None, None, :]
    v = -cx[:, None, None] * sx[None, :, None] * cx[None, None, :]
    w = np.zeros((n, n, n))
    return u, v, w


def velocity_band(n: int, seed: int, kp: float = 4.0):
    """The seeded spectral band of random_velocity: (ix, iz, F) with F[c] the
    complex amplitudes of component c on the half-spectrum index grid
    np.ix_(ix, ix, iz) of an (n, n, n//2+1) array (axes x, y, z)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kmax = min(n // 2 - 1, int(round(8 * kp)))
    kk = np.arange(-kmax, kmax + 1, dtype=np.float64)
    kz = np.arange(0, kmax + 1, dtype=np.float64)
    KX = kk[:, None, None]
    KY = kk[None, :, None]
    KZ = kz[None, None, :]
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    Kmag = np.sqrt(K2)
    theta = rng.uniform(0.0, 2.0 * np.pi, size=(3,) + K2.shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        E = Kmag ** 4 * np.exp(-2.0 * (Kmag / kp) ** 2)
        amp = np.sqrt(E / (4.0 * np.pi * K2))
    amp[K2 == 0] = 0.0
    amp[Kmag > kmax] = 0.0
    F = amp[None] * np.exp(1j * theta)
    with np.errstate(divide="ignore", invalid="ignore"):
        kdotF = (KX * F[0] + KY * F[1] + KZ * F[2]) / K2
    kdotF[K2 == 0] = 0.0
    F[0] -= KX * kdotF
    F[1] -= KY * kdotF
    F[2] -= KZ * kdotF
    F[0] *= np.exp(-1j * np.pi * KX / n)
    F[1] *= np.exp(-1j * np.pi * KY / n)
    F[2] *= np.exp(-1j * np.pi * KZ / n)
    ix = (np.arange(-kmax, kmax + 1) % n)
    iz = np.arange(0, kmax + 1)
    return ix, iz, F


def random_velocity(n: int, seed: int, rms: float = 1.0, kp: float = 4.0):
    """Random-phase solenoidal velocity with E(k) ~ k^4 exp(-2 (k/kp)^2).

    Built in index space (period n cells) on the band |k_i| <= kmax =
    min(n/2 - 1, 8 kp) (E(8 kp) / E(kp) ~ 1e-53, so nothing is lost): uniform
    random phases from seeded numpy PCG64, shell amplitude
    sqrt(E(k) / (4 pi k^2)), projection onto k-perpendicular, the u/v/w
    components sampled at their staggered faces (half a cell back along
    x/y/z), then the mean removed and one common factor applied so that the
    per-component rms averages to `rms` (a common factor keeps the field
    solenoidal).
    """
    try:
        from scipy import fft as sfft
        irfftn = lambda G: sfft.irfftn(G, s=(n, n, n), axes=(0, 1, 2), workers=-1)  # noqa: E731
    except ImportError:  # pragma: no cover
        irfftn = lambda G: np.fft.irfftn(G, s=(n, n, n), axes=(0, 1, 2))  # noqa: E731
    ix, iz, F = velocity_band(n, seed, kp)
    out = []
    for c in range(3):
        G = np.zeros((n, n, n // 2 + 1), dtype=np.complex128)
        G[np.ix_(ix, ix, iz)] = F[c]
        f = irfftn(G)
        del G
        f -= f.mean()
        out.append(f)
    cur = math.sqrt(sum(float(np.mean(f * f)) for f in out) / 3.0)
    for f in out:
        f *= rms / cur
    return out[0], out[1], out[2]


def _min_image(d: np.ndarray, period: float) -> np.ndarray:
    return d - period * np.round(d / period)


def place_drops(n: int, seed: int, ndrops: int, rmin: float, rmax: float,
                epsr: float = 1.0, grid_mode: int = 0, max_tries: int = 100000):
    """Seeded non-overlapping drop centres/radii (periodic minimum image,
    separation > r1 + r2 + 4 eps)."""
    dx = grid_dx(n, grid_mode)
    eps = epsr * dx
    period = n * dx
    rng = np.random.Generator(np.random.PCG64(seed))
    centres, radii = [], []
    tries = 0
    while len(centres) < ndrops:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place non-overlapping drops")
        c = rng.uniform(0.0, period, size=3)
        r = rng.uniform(rmin, rmax)
        ok = True
        for c2, r2 in zip(centres, radii):
            d = np.linalg.norm(_min_image(c - c2, period))
            if d <= r + r2 + 4.0 * eps:
                ok = False
                break
        if ok:
            centres.append(c)
            radii.append(r)
    return np.array(centres), np.array(radii)


def drop_field(n: int, centres, radii, epsr: float = 1.0, grid_mode: int = 0) -> np.ndarray:
    """phi = max over drops of 0.5*(1 - tanh((d - r)/2/eps)), the profile of
    multi/main.f90:273-274 with the periodic minimum-image distance d.
    Evaluated in a box of half-width r + 40 eps around each drop; beyond it
    the profile is exactly 0.0 in float64."""
    dx = grid_dx(n, grid_mode)
    eps = epsr * dx
    period = n * dx
    phi = np.zeros((n, n, n))
    for c, r in zip(centres, radii):
        half = int(math.ceil((r + 40.0 * eps) / dx)) + 1
        idx = []
        for ax in range(3):
            ic = int(round(c[ax] / dx))
            rng_ = np.arange(ic - half, ic + half + 1)
            if rng_.size >= n:
                rng_ = np.arange(n)
            idx.append(np.unique(np.mod(rng_, n)))
        ii, jj, kk = idx
        dxs = _min_image(ii * dx - c[0], period)
        dys = _min_image(jj * dx - c[1], period)
        dzs = _min_image(kk * dx - c[2], period)
        pos = dxs[:, None, None] ** 2 + dys[None, :, None] ** 2 + dzs[None, None, :] ** 2
        val = 0.5 * (1.0 - np.tanh((np.sqrt(pos) - r) / 2 / eps))
        sub = phi[np.ix_(ii, jj, kk)]
        phi[np.ix_(ii, jj, kk)] = np.maximum(sub, val)
    return phi


def centred_drop(n: int, radius: float, epsr: float = 1.0, grid_mode: int = 0) -> np.ndarray:
    """The reference's single centred drop (multi/main.f90:266-278)."""
    dx = grid_dx(n, grid_mode)
    eps = epsr * dx
    lx = 8.0 * math.atan(1.0)
    x = np.arange(n) * dx
    pos = (x[:, None, None] - lx / 2) ** 2 + (x[None, :, None] - lx / 2) ** 2 + (x[None, None, :] - lx / 2) ** 2
    return 0.5 * (1.0 - np.tanh((np.sqrt(pos) - radius) / 2 / eps))


# Workload recipes (sizes and drop counts of the benchmark configurations).
DROP_RECIPES = {
    128: (8, 0.4, 0.6),
    256: (8, 0.4, 0.6),
    512: (64, 0.2, 0.35),
}


def seeded_case(n: int, phase_field: bool = True, ndrops=None, rmin=None, rmax=None,
                epsr: float = 1.0, grid_mode: int = 0, seed=None):
    """Velocity seeded with N (or `seed`), drops seeded with N+1."""
    s = n if seed is None else seed
    u, v, w = random_velocity(n, s)
    phi = None
    if phase_field:
        d, lo, hi = DROP_RECIPES.get(n, (max(2, n // 16), 0.4, 0.6))
        ndrops = d if ndrops is None else ndrops
        rmin = lo if rmin is None else rmin
        rmax = hi if rmax is None else rmax
        c, r = place_drops(n, s + 1, ndrops, rmin, rmax, epsr, grid_mode)
        phi = drop_field(n, c, r, epsr, grid_mode)
    return u, v, w, phi


def write_inputs(indir: str, u, v, w, phi=None) -> None:
    os.makedirs(indir, exist_ok=True)
    write_field(os.path.join(indir, "u.dat"), u)
    write_field(os.path.join(indir, "v.dat"), v)
    write_field(os.path.join(indir, "w.dat"), w)
    if phi is not None:
        write_field(os.path.join(indir, "phi.dat"), phi)
