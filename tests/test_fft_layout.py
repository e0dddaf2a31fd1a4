"""CPU model of the register-resident FFT (reg_fft_stages in
mhit36_b200/csrc/fft.cuh) and of the shared-memory slots its callers give it.

Each thread of a line holds E elements v[m] = x[t + (N/E)*m] (E = 8 for
power-of-two N, 12 for N = 3*2^k); a stage with radix R (R divides E) and
span NS runs butterfly b on j = t + (N/E)*b with inputs v[b + (E/R)*r],
multiplies input r by w_N^(r*(j mod NS)*N/(NS*R)), and (unless it is the
last stage) writes output r to slot at(d) with d = (j/NS)*NS*R + j%NS + r*NS,
after which every thread reads its canonical elements back.  The model runs
that data movement with numpy for every size the library builds and checks:
  * the result is the DFT of the line (numpy.fft), so the index maps are a
    Stockham transform;
  * every exchange slot is inside the buffer the launcher sizes, and no two
    elements of one exchange share a slot (the lines' regions do not overlap);
  * the last stage leaves each thread its own canonical elements (what the
    z solve's in-register scaling and the x passes' direct stores rely on).
"""
import numpy as np
import pytest

SIZES = (32, 64, 96, 128, 192, 256, 384, 512, 768, 1024)


def reg_elems(n):
    return 8 if n & (n - 1) == 0 else 12


def pick_radix(rem, e):
    for r in (8, 4, 2, 3):
        if rem % r == 0 and e % r == 0:
            return r
    raise AssertionError(f"no radix for {rem} with {e} elements per thread")


def lines_per_cta(n):
    return 8 if n <= 256 else (4 if n <= 512 else 2)


def reg_rows(n):
    return n + n // 8


def pad(n):
    return n + (n >> 3)


def swz(n):
    return n ^ ((n >> 3) & 15)


def model_fft(x, direction, at, nslots):
    """Run the register-resident transform of the lines x[c, :] (direction
    -1 forward, +1 unnormalised inverse) through a shared buffer of nslots
    slots, with at(c, n) the slot of element n of line c."""
    nlines, n = x.shape
    e_ = reg_elems(n)
    tpc = n // e_
    w = np.exp(-2j * np.pi * np.arange(n) / n)  # the twiddle table tw[m] = e^{-2 pi i m/N}
    if direction > 0:
        w = np.conj(w)
    # v[c, t, m] = x[c, t + tpc*m]
    v = np.stack([x[:, t + tpc * np.arange(e_)] for t in range(tpc)], axis=1)
    ns = 1
    while ns < n:
        r_ = pick_radix(n // ns, e_)
        b_ = e_ // r_
        tstride = n // (ns * r_)
        out = np.empty_like(v)
        for b in range(b_):
            j = np.arange(tpc) + tpc * b
            jm = j % ns
            u = np.stack([v[:, :, b + b_ * r] * (w[(r * jm * tstride) % n] if ns > 1 else 1.0)
                          for r in range(r_)], axis=-1)
            d = np.fft.fft(u, axis=-1) if direction < 0 else np.fft.ifft(u, axis=-1) * r_
            for r in range(r_):
                out[:, :, b + b_ * r] = d[..., r]
        v = out
        if ns * r_ < n:
            s = np.full(nslots, np.nan + 0j)
            used = set()
            for c in range(nlines):
                for t in range(tpc):
                    for b in range(b_):
                        j = t + tpc * b
                        d0 = (j // ns) * ns * r_ + j % ns
                        for r in range(r_):
                            slot = at(c, d0 + r * ns)
                            assert 0 <= slot < nslots
                            assert slot not in used
                            used.add(slot)
                            s[slot] = v[c, t, b + b_ * r]
            for c in range(nlines):
                for t in range(tpc):
                    for m in range(e_):
                        v[c, t, m] = s[at(c, t + tpc * m)]
        ns *= r_
    # back to line order: element t + tpc*m of line c
    y = np.empty_like(x)
    for t in range(tpc):
        y[:, t + tpc * np.arange(e_)] = v[:, t, :]
    return y


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("elem", [16, 8])
def test_column_slab_layout(n, elem):
    """y passes and z solve: CC kx columns interleaved, slot pad(n)*CC + c,
    in an exchange buffer of reg_rows(N)*CC slots."""
    cc = lines_per_cta(n) * (1 if elem == 16 else 2)
    rng = np.random.default_rng(n + elem)
    x = rng.standard_normal((cc, n)) + 1j * rng.standard_normal((cc, n))
    at = lambda c, k: pad(k) * cc + c  # noqa: E731
    y = model_fft(x, -1, at, reg_rows(n) * cc)
    assert np.max(np.abs(y - np.fft.fft(x, axis=1))) < 1e-9 * np.max(np.abs(y))
    z = model_fft(y, +1, at, reg_rows(n) * cc)
    assert np.max(np.abs(z / n - x)) < 1e-12 * n


@pytest.mark.parametrize("n", SIZES)
def test_x_line_layouts(n):
    """x passes: FP64 lines at c*reg_rows(N) + pad(n), FP32 lines at
    c*N + swz(n); the fused x inverse + projection (n >= 256) adds one halo
    pair, P + 1 lines at c*reg_rows(N) + pad(n)."""
    p = lines_per_cta(n)
    rng = np.random.default_rng(n)
    cases = [(p, lambda c, k: c * reg_rows(n) + pad(k), p * reg_rows(n)),
             (p, lambda c, k: c * n + swz(k), p * n)]
    if n >= 256:
        cases.append((p + 1, lambda c, k: c * reg_rows(n) + pad(k), (p + 1) * reg_rows(n)))
    for nlines, at, nslots in cases:
        x = rng.standard_normal((nlines, n)) + 1j * rng.standard_normal((nlines, n))
        y = model_fft(x, +1, at, nslots)
        assert np.max(np.abs(y - np.fft.ifft(x, axis=1) * n)) < 1e-9 * np.max(np.abs(y))


@pytest.mark.parametrize("n", SIZES)
def test_fused_kernel_buffers_fit(n):
    """The fused kernel's p rows (2P+1 rows of N doubles) alias its exchange
    buffer ((P+1)*reg_rows(N) complex) and the previous plane's rows (2P x N)
    follow it; the whole stays inside 227 KB, and its thread count is whole
    warps (its block reduction shuffles full warps)."""
    if n < 256 or n & (n - 1):
        pytest.skip("fused only for power-of-two sizes from 256^3")
    p = lines_per_cta(n)
    xbytes = (p + 1) * reg_rows(n) * 16
    pbytes = (2 * p + 1) * n * 8
    smem = max(xbytes, pbytes) + 2 * p * n * 8
    assert smem <= 227 * 1024
    assert ((p + 1) * (n // 8)) % 32 == 0
