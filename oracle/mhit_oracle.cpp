// MHIT36 CPU ORACLE -- test infrastructure only.
//
// This file is the checker for the CUDA step in mhit36_b200/csrc.  It is a
// plain C++17/OpenMP restatement, in FP64, of one MHIT36 timestep as written in
// the reference (aroccon/MHIT36, multi/main.f90:329-977).  Only tests/, the
// smoke() entry and bench.py's CPU-baseline / reference legs may load it; the
// product library never links or calls it.
//
// Layout follows the reference module arrays (multi/module.f90:39-58,
// allocated at multi/main.f90:175-200): Fortran order (x fastest) with shape
// (nx, ny+2, nz+2), one halo cell in y and z, none in x.  On one rank every
// cuDecomp halo update (cudecompUpdateHalosX, periodic) is a periodic copy of
// the opposite interior plane, which `halo()` reproduces (y first, then z over
// all j so that edge/corner cells are filled too).
//
// Reference quirks that are reproduced on purpose:
//   * dx = lx/(nx-1) with x(i)=(i-1)dx (multi/readinput.f90:37,
//     multi/main.f90:150-153) -- grid_mode 0;
//   * spectral k^2 with integer k in the Poisson solve (multi/main.f90:154-159,
//     791-792) -- k2_mode 0;
//   * enum and the normal-vector guard are the float32 literal 1.e-16
//     (multi/readinput.f90:43, multi/main.f90:436);
//   * gamma = 1.0*gumax of the previous step, gumax = 1 before step 1
//     (multi/main.f90:325-327, 362);
//   * gumax is the SIGNED max of u,v,w over the whole halo'd arrays
//     (multi/main.f90:937-941);
//   * phi is advanced with explicit Euler (multi/main.f90:476), momentum with
//     Euler on the first step then AB2 (multi/main.f90:323-324, 666-668, 677-678).
// Extensions (absent from the reference, off by default): linear forcing
// rhs += A*u, an FD-modified k^2 (exact inverse of the 7-point Laplacian), and a
// consistent grid dx = lx/nx.
//
// The FFT is this file's own mixed-radix Stockham transform (radices 4,2,3,5),
// standing in for cuFFT Z2Z (forward e^{-i}, inverse e^{+i}, unnormalised),
// which the reference calls at multi/main.f90:750-812.

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

typedef std::complex<double> cplx;

extern "C" {

// Mirrors input.inp lines 1-16 (multi/readinput.f90:13-31) plus extensions.
typedef struct oracle_params {
  double dt, mu, rho;
  double f1, f2, f3, k0;
  double radius, sigma, epsr;
  double lin_force;   // extension: rhs += A*u (0 = off, as the reference)
  int k2_mode;        // 0 spectral (reference), 1 FD-modified
  int grid_mode;      // 0 reference dx=2pi/(N-1), 1 consistent dx=2pi/N
  int phase_field;    // 1 = ACDI on (#define phiflag 1, multi/main.f90:39)
  int tanh_identity;  // 1 = use tanh(psi/2eps)=(2phi-1)/(1+2enum) (not the reference)
  int phi_floor;      // 1 = psi from max(min(phi,1),0) (not the reference)
} oracle_params;

typedef struct oracle_diag {
  double umax;     // gumax after the step (signed max, multi/main.f90:937-941)
  double cfl;      // gumax*dt*dxi (multi/main.f90:942)
  double umean, vmean, wmean;  // means removed in the step (multi/main.f90:906-919)
  int step;        // steps taken so far
} oracle_diag;

}  // extern "C"

namespace {

// ---------------------------------------------------------------- FFT
struct FFTPlan {
  int n = 0;
  std::vector<int> radices;
  std::vector<cplx> tw_fwd, tw_inv;  // e^{-+2 pi i m / n}
  void init(int n_) {
    n = n_;
    radices.clear();
    int m = n;
    while (m % 4 == 0) { radices.push_back(4); m /= 4; }
    while (m % 2 == 0) { radices.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2) {
      while (m % p == 0) { radices.push_back(p); m /= p; }
    }
    tw_fwd.resize(n);
    tw_inv.resize(n);
    for (int i = 0; i < n; ++i) {
      long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)i / (long double)n;
      double c = (double)cosl(a), s = (double)sinl(a);
      tw_fwd[i] = cplx(c, -s);
      tw_inv[i] = cplx(c, s);
    }
  }
  // In-place transform of x (length n) using scratch y (length n).
  void run(cplx* x, cplx* y, int sign) const {
    const cplx* tw = (sign < 0) ? tw_fwd.data() : tw_inv.data();
    cplx* src = x;
    cplx* dst = y;
    int Ns = 1;
    for (int R : radices) {
      const int nR = n / R;
      const int tstride = n / (Ns * R);
      cplx v[32], o[32];
      for (int j = 0; j < nR; ++j) {
        const int jm = j % Ns;
        for (int r = 0; r < R; ++r) {
          cplx a = src[j + r * nR];
          if (r && jm) a *= tw[(r * jm * tstride) % n];
          v[r] = a;
        }
        for (int s = 0; s < R; ++s) {
          cplx acc = v[0];
          for (int r = 1; r < R; ++r) acc += v[r] * tw[((r * s) % R) * nR];
          o[s] = acc;
        }
        const int idxD = (j / Ns) * Ns * R + jm;
        for (int s = 0; s < R; ++s) dst[idxD + s * Ns] = o[s];
      }
      std::swap(src, dst);
      Ns *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cplx) * n);
  }
};

inline double f32lit(double v) { return (double)(float)v; }

struct Oracle {
  int nx, ny, nz;
  int sy, sz;   // halo'd extents ny+2, nz+2
  size_t ntot;  // nx*(ny+2)*(nz+2)
  oracle_params prm;
  double lx, dx, dxi, ddxi, rhoi, eps, epsi, enum_;
  double gumax, alpha, beta;
  int nstep;
  double last_means[3];
  std::vector<double> x, kx;
  std::vector<double> u, v, w, ustar, vstar, wstar, rhsu, rhsv, rhsw, rhsu_o, rhsv_o, rhsw_o;
  std::vector<double> rhsp, p;
  std::vector<double> phi, rhsphi, psidi, normx, normy, normz, chempot, gpx, gpy, gpz, fxst, fyst, fzst;
  std::vector<cplx> psi;  // complex Poisson work array, X-pencil layout
  FFTPlan planx, plany, planz;

  inline size_t id(int i, int j, int k) const {  // 1-based Fortran indices
    return (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)sy * (size_t)(k - 1));
  }

  void init(const oracle_params* p_, int n_) {
    prm = *p_;
    nx = ny = nz = n_;
    sy = ny + 2;
    sz = nz + 2;
    ntot = (size_t)nx * sy * sz;
    // multi/readinput.f90:34-43
    const double twopi = 8.0 * std::atan(1.0);
    lx = twopi;
    dx = (prm.grid_mode == 1) ? lx / nx : lx / (nx - 1);
    dxi = 1.0 / dx;
    ddxi = 1.0 / dx / dx;
    rhoi = 1.0 / prm.rho;
    eps = prm.epsr * dx;
    epsi = 1.0 / eps;
    enum_ = f32lit(1.e-16);
    // multi/main.f90:149-159
    x.assign(nx, 0.0);
    kx.assign(nx, 0.0);
    for (int i = 2; i <= nx; ++i) x[i - 1] = x[i - 2] + dx;
    for (int i = 1; i <= nx / 2; ++i) kx[i - 1] = (i - 1) * (twopi / lx);
    for (int i = nx / 2 + 1; i <= nx; ++i) kx[i - 1] = (i - 1 - nx) * (twopi / lx);
    auto z = [&](std::vector<double>& a) { a.assign(ntot, 0.0); };
    z(u); z(v); z(w); z(ustar); z(vstar); z(wstar); z(rhsu); z(rhsv); z(rhsw);
    z(rhsu_o); z(rhsv_o); z(rhsw_o); z(rhsp); z(p);
    if (prm.phase_field) {
      z(phi); z(rhsphi); z(psidi); z(normx); z(normy); z(normz); z(chempot);
      z(gpx); z(gpy); z(gpz); z(fxst); z(fyst); z(fzst);
    }
    psi.assign(ntot, cplx(0, 0));
    planx.init(nx); plany.init(ny); planz.init(nz);
    // multi/main.f90:323-327
    alpha = 1.0; beta = 0.0; gumax = 1.0;
    nstep = 0;
    last_means[0] = last_means[1] = last_means[2] = 0.0;
  }

  // Periodic halo copy in y then z (cudecompUpdateHalosX along axes 2, 3).
  template <class T>
  void halo(std::vector<T>& a) {
#pragma omp parallel for
    for (int k = 2; k <= nz + 1; ++k) {
      std::memcpy(&a[id(1, 1, k)], &a[id(1, ny + 1, k)], sizeof(T) * nx);
      std::memcpy(&a[id(1, ny + 2, k)], &a[id(1, 2, k)], sizeof(T) * nx);
    }
    const size_t plane = (size_t)nx * sy;
    std::memcpy(&a[id(1, 1, 1)], &a[id(1, 1, nz + 1)], sizeof(T) * plane);
    std::memcpy(&a[id(1, 1, nz + 2)], &a[id(1, 1, 2)], sizeof(T) * plane);
  }

  // ------------------------------------------------------------ phase field
  // multi/main.f90:338-486
  void phase_step() {
    const double gamma = 1.0 * gumax;  // multi/main.f90:362
    // A1 + A2: convection and diffusion (multi/main.f90:341-381)
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
          if (ip > nx) ip = 1;
          if (im < 1) im = nx;
          const double c = phi[id(i, j, k)];
          double r = -(u[id(ip, j, k)] * 0.5 * (phi[id(ip, j, k)] + c) - u[id(i, j, k)] * 0.5 * (c + phi[id(im, j, k)])) * dxi
                     - (v[id(i, jp, k)] * 0.5 * (phi[id(i, jp, k)] + c) - v[id(i, j, k)] * 0.5 * (c + phi[id(i, jm, k)])) * dxi
                     - (w[id(i, j, kp)] * 0.5 * (phi[id(i, j, kp)] + c) - w[id(i, j, k)] * 0.5 * (c + phi[id(i, j, km)])) * dxi;
          r = r + gamma * (eps * (phi[id(ip, j, k)] - 2.0 * c + phi[id(im, j, k)]) * ddxi
                           + eps * (phi[id(i, jp, k)] - 2.0 * c + phi[id(i, jm, k)]) * ddxi
                           + eps * (phi[id(i, j, kp)] - 2.0 * c + phi[id(i, j, km)]) * ddxi);
          rhsphi[id(i, j, k)] = r;
        }
    // A3: psi on all cells including halos (multi/main.f90:384-393)
#pragma omp parallel for
    for (size_t n = 0; n < ntot; ++n) {
      double val = std::min(phi[n], 1.0);
      if (prm.phi_floor) val = std::max(val, 0.0);
      psidi[n] = eps * std::log((val + enum_) / (1.0 - val + enum_));
    }
    // A4: raw gradient of psi (multi/main.f90:397-415)
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int ip = i + 1, im = i - 1;
          if (ip > nx) ip = 1;
          if (im < 1) im = nx;
          normx[id(i, j, k)] = psidi[id(ip, j, k)] - psidi[id(im, j, k)];
          normy[id(i, j, k)] = psidi[id(i, j + 1, k)] - psidi[id(i, j - 1, k)];
          normz[id(i, j, k)] = psidi[id(i, j, k + 1)] - psidi[id(i, j, k - 1)];
        }
    halo(normx); halo(normy); halo(normz);  // H1
    // A5: normalise on all cells (multi/main.f90:432-443); 1.0E-16 is a float32 literal
    const double tiny = f32lit(1.0E-16);
#pragma omp parallel for
    for (size_t n = 0; n < ntot; ++n) {
      const double a = normx[n], b = normy[n], c = normz[n];
      const double normod = 1.0 / (std::sqrt(a * a + b * b + c * c) + tiny);
      normx[n] = a * normod;
      normy[n] = b * normod;
      normz[n] = c * normod;
    }
    // A6: ACDI sharpening (multi/main.f90:446-469)
    auto g = [&](size_t n) -> double {
      double t;
      if (prm.tanh_identity) {
        double val = std::min(phi[n], 1.0);
        if (prm.phi_floor) val = std::max(val, 0.0);
        t = (2.0 * val - 1.0) * (1.0 / (1.0 + 2.0 * enum_));
      } else {
        t = std::tanh(0.5 * psidi[n] * epsi);
      }
      return 0.25 * (1.0 - t * t);
    };
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int ip = i + 1, im = i - 1;
          if (ip > nx) ip = 1;
          if (im < 1) im = nx;
          const size_t xp = id(ip, j, k), xm = id(im, j, k), yp = id(i, j + 1, k), ym = id(i, j - 1, k),
                       zp = id(i, j, k + 1), zm = id(i, j, k - 1);
          rhsphi[id(i, j, k)] = rhsphi[id(i, j, k)] -
              gamma * ((g(xp) * normx[xp] - g(xm) * normx[xm]) * 0.5 * dxi +
                       (g(yp) * normy[yp] - g(ym) * normy[ym]) * 0.5 * dxi +
                       (g(zp) * normz[zp] - g(zm) * normz[zm]) * 0.5 * dxi);
        }
    // A7: explicit Euler (multi/main.f90:472-480)
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) phi[id(i, j, k)] = phi[id(i, j, k)] + prm.dt * rhsphi[id(i, j, k)];
    halo(phi);  // H2
  }

  // ------------------------------------------------------------ momentum
  // multi/main.f90:510-696
  void momentum_step() {
    const double mu = prm.mu, dt = prm.dt;
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int ip = i + 1, im = i - 1;
          const int jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
          if (ip > nx) ip = 1;
          if (im < 1) im = nx;
          auto U = [&](int a, int b, int c) { return u[id(a, b, c)]; };
          auto V = [&](int a, int b, int c) { return v[id(a, b, c)]; };
          auto W = [&](int a, int b, int c) { return w[id(a, b, c)]; };
          // B1 convection, conservative form (multi/main.f90:527-549)
          double h11 = (U(ip, j, k) + U(i, j, k)) * (U(ip, j, k) + U(i, j, k)) - (U(i, j, k) + U(im, j, k)) * (U(i, j, k) + U(im, j, k));
          double h12 = (U(i, jp, k) + U(i, j, k)) * (V(i, jp, k) + V(im, jp, k)) - (U(i, j, k) + U(i, jm, k)) * (V(i, j, k) + V(im, j, k));
          double h13 = (U(i, j, kp) + U(i, j, k)) * (W(i, j, kp) + W(im, j, kp)) - (U(i, j, k) + U(i, j, km)) * (W(i, j, k) + W(im, j, k));
          double h21 = (U(ip, j, k) + U(ip, jm, k)) * (V(ip, j, k) + V(i, j, k)) - (U(i, j, k) + U(i, jm, k)) * (V(i, j, k) + V(im, j, k));
          double h22 = (V(i, jp, k) + V(i, j, k)) * (V(i, jp, k) + V(i, j, k)) - (V(i, j, k) + V(i, jm, k)) * (V(i, j, k) + V(i, jm, k));
          double h23 = (W(i, j, kp) + W(i, jm, kp)) * (V(i, j, kp) + V(i, j, k)) - (W(i, j, k) + W(i, jm, k)) * (V(i, j, k) + V(i, j, km));
          double h31 = (W(ip, j, k) + W(i, j, k)) * (U(ip, j, k) + U(ip, j, km)) - (W(i, j, k) + W(im, j, k)) * (U(i, j, k) + U(i, j, km));
          double h32 = (V(i, jp, k) + V(i, jp, km)) * (W(i, jp, k) + W(i, j, k)) - (V(i, j, k) + V(i, j, km)) * (W(i, j, k) + W(i, jm, k));
          double h33 = (W(i, j, kp) + W(i, j, k)) * (W(i, j, kp) + W(i, j, k)) - (W(i, j, k) + W(i, j, km)) * (W(i, j, k) + W(i, j, km));
          h11 = h11 * 0.25 * dxi; h12 = h12 * 0.25 * dxi; h13 = h13 * 0.25 * dxi;
          h21 = h21 * 0.25 * dxi; h22 = h22 * 0.25 * dxi; h23 = h23 * 0.25 * dxi;
          h31 = h31 * 0.25 * dxi; h32 = h32 * 0.25 * dxi; h33 = h33 * 0.25 * dxi;
          double ru = -(h11 + h12 + h13);
          double rv = -(h21 + h22 + h23);
          double rw = -(h31 + h32 + h33);
          // B2 viscous (multi/main.f90:567-578)
          h11 = mu * (U(ip, j, k) - 2.0 * U(i, j, k) + U(im, j, k)) * ddxi;
          h12 = mu * (U(i, jp, k) - 2.0 * U(i, j, k) + U(i, jm, k)) * ddxi;
          h13 = mu * (U(i, j, kp) - 2.0 * U(i, j, k) + U(i, j, km)) * ddxi;
          h21 = mu * (V(ip, j, k) - 2.0 * V(i, j, k) + V(im, j, k)) * ddxi;
          h22 = mu * (V(i, jp, k) - 2.0 * V(i, j, k) + V(i, jm, k)) * ddxi;
          h23 = mu * (V(i, j, kp) - 2.0 * V(i, j, k) + V(i, j, km)) * ddxi;
          h31 = mu * (W(ip, j, k) - 2.0 * W(i, j, k) + W(im, j, k)) * ddxi;
          h32 = mu * (W(i, jp, k) - 2.0 * W(i, j, k) + W(i, jm, k)) * ddxi;
          h33 = mu * (W(i, j, kp) - 2.0 * W(i, j, k) + W(i, j, km)) * ddxi;
          ru = ru + (h11 + h12 + h13) * rhoi;
          rv = rv + (h21 + h22 + h23) * rhoi;
          rw = rw + (h31 + h32 + h33) * rhoi;
          // B3 ABC forcing (multi/main.f90:584-600).  Coordinates use the
          // global interior index (jg = j-1 here), see the file header.
          const double xi = x[i - 1], xj = x[j - 2], xk = x[k - 2];
          ru = ru + prm.f3 * std::sin(prm.k0 * xk) + prm.f2 * std::cos(prm.k0 * xj);
          rv = rv + prm.f1 * std::sin(prm.k0 * xi) + prm.f3 * std::cos(prm.k0 * xk);
          rw = rw + prm.f2 * std::sin(prm.k0 * xj) + prm.f1 * std::cos(prm.k0 * xi);
          // Extension: linear forcing A*u on the staggered component itself.
          if (prm.lin_force != 0.0) {
            ru = ru + prm.lin_force * U(i, j, k);
            rv = rv + prm.lin_force * V(i, j, k);
            rw = rw + prm.lin_force * W(i, j, k);
          }
          rhsu[id(i, j, k)] = ru;
          rhsv[id(i, j, k)] = rv;
          rhsw[id(i, j, k)] = rw;
        }
    if (prm.phase_field) {
      const double sigma = prm.sigma;
      // B4 chemical potential, gradient and force at cell centres (multi/main.f90:606-626)
#pragma omp parallel for collapse(2)
      for (int k = 2; k <= nz + 1; ++k)
        for (int j = 2; j <= ny + 1; ++j)
          for (int i = 1; i <= nx; ++i) {
            int ip = i + 1, im = i - 1;
            const int jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
            if (ip > nx) ip = 1;
            if (im < 1) im = nx;
            const double c = phi[id(i, j, k)];
            const size_t n = id(i, j, k);
            chempot[n] = c * (1.0 - c) * (1.0 - 2.0 * c) * epsi -
                         eps * (phi[id(ip, j, k)] + phi[id(im, j, k)] + phi[id(i, jp, k)] + phi[id(i, jm, k)] +
                                phi[id(i, j, kp)] + phi[id(i, j, km)] - 6.0 * c) * ddxi;
            gpx[n] = 0.5 * (phi[id(ip, j, k)] - phi[id(im, j, k)]) * dxi;
            gpy[n] = 0.5 * (phi[id(i, jp, k)] - phi[id(i, jm, k)]) * dxi;
            gpz[n] = 0.5 * (phi[id(i, j, kp)] - phi[id(i, j, km)]) * dxi;
            fxst[n] = 6.0 * sigma * chempot[n] * gpx[n];
            fyst[n] = 6.0 * sigma * chempot[n] * gpy[n];
            fzst[n] = 6.0 * sigma * chempot[n] * gpz[n];
          }
      halo(fxst); halo(fyst); halo(fzst);  // H3
      // B5 face interpolation (multi/main.f90:645-657)
#pragma omp parallel for collapse(2)
      for (int k = 2; k <= nz + 1; ++k)
        for (int j = 2; j <= ny + 1; ++j)
          for (int i = 1; i <= nx; ++i) {
            int im = i - 1;
            if (im < 1) im = nx;
            const size_t n = id(i, j, k);
            rhsu[n] = rhsu[n] + 0.5 * (fxst[id(im, j, k)] + fxst[n]) * rhoi;
            rhsv[n] = rhsv[n] + 0.5 * (fyst[id(i, j - 1, k)] + fyst[n]) * rhoi;
            rhsw[n] = rhsw[n] + 0.5 * (fzst[id(i, j, k - 1)] + fzst[n]) * rhoi;
          }
    }
    // B6 AB2 / Euler (multi/main.f90:662-672), B7 (multi/main.f90:676-682)
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          const size_t n = id(i, j, k);
          ustar[n] = u[n] + dt * (alpha * rhsu[n] - beta * rhsu_o[n]);
          vstar[n] = v[n] + dt * (alpha * rhsv[n] - beta * rhsv_o[n]);
          wstar[n] = w[n] + dt * (alpha * rhsw[n] - beta * rhsw_o[n]);
        }
    alpha = 1.5;
    beta = 0.5;
    rhsu_o = rhsu;
    rhsv_o = rhsv;
    rhsw_o = rhsw;
    halo(ustar); halo(vstar); halo(wstar);  // H4
  }

  // ------------------------------------------------------------ Poisson
  double k2_at(int ig, int jg, int kg) const {  // 1-based wavenumber indices
    if (prm.k2_mode == 1) {
      const double pi = 4.0 * std::atan(1.0);
      const double sx = std::sin(pi * (ig - 1) / nx), sy_ = std::sin(pi * (jg - 1) / ny), sz_ = std::sin(pi * (kg - 1) / nz);
      const double c = 4.0 * ddxi;
      return c * (sx * sx) + c * (sy_ * sy_) + c * (sz_ * sz_);
    }
    return kx[ig - 1] * kx[ig - 1] + kx[jg - 1] * kx[jg - 1] + kx[kg - 1] * kx[kg - 1];
  }

  // 3D complex transform of the interior of psi (x, then y, then z lines).
  void fft3(int sign) {
    // The reference transforms halo rows along x too (multi/main.f90:134-135),
    // then cuDecomp drops them in the X->Y transpose; interior lines suffice.
#pragma omp parallel
    {
      std::vector<cplx> buf(std::max(nx, std::max(ny, nz))), scr(buf.size());
      if (sign < 0) {
        pass_x(buf, scr, sign);
#pragma omp barrier
        pass_y(buf, scr, sign);
#pragma omp barrier
        pass_z(buf, scr, sign);
      } else {
        pass_z(buf, scr, sign);
#pragma omp barrier
        pass_y(buf, scr, sign);
#pragma omp barrier
        pass_x(buf, scr, sign);
      }
    }
  }
  void pass_x(std::vector<cplx>& buf, std::vector<cplx>& scr, int sign) {
#pragma omp for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j) planx.run(&psi[id(1, j, k)], scr.data(), sign);
    (void)buf;  // x lines are contiguous and transformed in place
  }
  void pass_y(std::vector<cplx>& buf, std::vector<cplx>& scr, int sign) {
#pragma omp for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int i = 1; i <= nx; ++i) {
        for (int j = 0; j < ny; ++j) buf[j] = psi[id(i, j + 2, k)];
        plany.run(buf.data(), scr.data(), sign);
        for (int j = 0; j < ny; ++j) psi[id(i, j + 2, k)] = buf[j];
      }
  }
  void pass_z(std::vector<cplx>& buf, std::vector<cplx>& scr, int sign) {
#pragma omp for collapse(2)
    for (int j = 2; j <= ny + 1; ++j)
      for (int i = 1; i <= nx; ++i) {
        for (int k = 0; k < nz; ++k) buf[k] = psi[id(i, j, k + 2)];
        planz.run(buf.data(), scr.data(), sign);
        for (int k = 0; k < nz; ++k) psi[id(i, j, k + 2)] = buf[k];
      }
  }

  // rhsp (interior) -> p (all cells), multi/main.f90:732-850.
  void poisson() {
#pragma omp parallel for
    for (size_t n = 0; n < ntot; ++n) psi[n] = cplx(0.0, 0.0);
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) psi[id(i, j, k)] = cplx(rhsp[id(i, j, k)], 0.0);
    fft3(-1);
    const double nnn = (double)((int64_t)nx * (int64_t)ny * (int64_t)nz);
    // C1: divide by -k^2 and normalise (multi/main.f90:785-798)
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          const double k2 = k2_at(i, j - 1, k - 1);
          cplx& z = psi[id(i, j, k)];
          z = cplx(-z.real() / k2 / nnn, -z.imag() / k2 / nnn);
        }
    psi[id(1, 2, 2)] = cplx(0.0, 0.0);
    fft3(+1);
    halo(psi);  // H5
    // P3 (multi/main.f90:842-850)
#pragma omp parallel for
    for (size_t n = 0; n < ntot; ++n) p[n] = psi[n].real();
  }

  void pressure_step() {
    const double c = prm.rho * dxi / prm.dt;  // (rho*dxi/dt), multi/main.f90:723
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int ip = i + 1;
          if (ip > nx) ip = 1;
          double r = c * (ustar[id(ip, j, k)] - ustar[id(i, j, k)]);
          r = r + c * (vstar[id(i, j + 1, k)] - vstar[id(i, j, k)]);
          r = r + c * (wstar[id(i, j, k + 1)] - wstar[id(i, j, k)]);
          rhsp[id(i, j, k)] = r;
        }
    poisson();
  }

  // ------------------------------------------------------------ correction
  // multi/main.f90:869-946
  void correction_step() {
    const double dtr = prm.dt / prm.rho;
#pragma omp parallel for collapse(2)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          int im = i - 1;
          if (im < 1) im = nx;
          const size_t n = id(i, j, k);
          u[n] = ustar[n] - dtr * (p[n] - p[id(im, j, k)]) * dxi;
          v[n] = vstar[n] - dtr * (p[n] - p[id(i, j - 1, k)]) * dxi;
          w[n] = wstar[n] - dtr * (p[n] - p[id(i, j, k - 1)]) * dxi;
        }
    double su = 0, sv = 0, sw = 0;
#pragma omp parallel for collapse(2) reduction(+ : su, sv, sw)
    for (int k = 2; k <= nz + 1; ++k)
      for (int j = 2; j <= ny + 1; ++j)
        for (int i = 1; i <= nx; ++i) {
          const size_t n = id(i, j, k);
          su += u[n];
          sv += v[n];
          sw += w[n];
        }
    const double um = su / nx / ny / nz, vm = sv / nx / ny / nz, wm = sw / nx / ny / nz;
#pragma omp parallel for
    for (size_t n = 0; n < ntot; ++n) {
      u[n] = u[n] - um;
      v[n] = v[n] - vm;
      w[n] = w[n] - wm;
    }
    halo(u); halo(v); halo(w);  // H6
    double uc = -INFINITY, vc = -INFINITY, wc = -INFINITY;
#pragma omp parallel for reduction(max : uc, vc, wc)
    for (size_t n = 0; n < ntot; ++n) {
      uc = std::max(uc, u[n]);
      vc = std::max(vc, v[n]);
      wc = std::max(wc, w[n]);
    }
    gumax = std::max(wc, std::max(uc, vc));
    last_means[0] = um; last_means[1] = vm; last_means[2] = wm;
  }

  void step() {
    if (prm.phase_field) phase_step();
    momentum_step();
    pressure_step();
    correction_step();
    ++nstep;
  }

  // Raw interior (nx*ny*nz, x fastest) <-> halo'd arrays.
  void put(std::vector<double>& a, const double* src) {
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        std::memcpy(&a[id(1, j + 2, k + 2)], src + (size_t)nx * (j + (size_t)ny * k), sizeof(double) * nx);
    halo(a);
  }
  void get(const std::vector<double>& a, double* dst) const {
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        std::memcpy(dst + (size_t)nx * (j + (size_t)ny * k), &a[id(1, j + 2, k + 2)], sizeof(double) * nx);
  }
};

}  // namespace

extern "C" {

void* oracle_create(const oracle_params* p, int n) {
  if (n < 4 || (n % 2) != 0) return nullptr;
  Oracle* o = new Oracle();
  o->init(p, n);
  return o;
}

void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }

int oracle_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// u, v, w, phi: raw interior arrays (nx*ny*nz, x fastest); phi may be NULL.
void oracle_set_fields(void* h, const double* u, const double* v, const double* w, const double* phi) {
  Oracle* o = static_cast<Oracle*>(h);
  o->put(o->u, u);
  o->put(o->v, v);
  o->put(o->w, w);
  if (phi && o->prm.phase_field) o->put(o->phi, phi);
}

void oracle_get_fields(void* h, double* u, double* v, double* w, double* phi) {
  Oracle* o = static_cast<Oracle*>(h);
  if (u) o->get(o->u, u);
  if (v) o->get(o->v, v);
  if (w) o->get(o->w, w);
  if (phi && o->prm.phase_field) o->get(o->phi, phi);
}

void oracle_get_pressure(void* h, double* p) {
  Oracle* o = static_cast<Oracle*>(h);
  o->get(o->p, p);
}

void oracle_get_state(void* h, double* ustar, double* vstar, double* wstar, double* rhsu_o, double* rhsv_o,
                      double* rhsw_o) {
  Oracle* o = static_cast<Oracle*>(h);
  if (ustar) o->get(o->ustar, ustar);
  if (vstar) o->get(o->vstar, vstar);
  if (wstar) o->get(o->wstar, wstar);
  if (rhsu_o) o->get(o->rhsu_o, rhsu_o);
  if (rhsv_o) o->get(o->rhsv_o, rhsv_o);
  if (rhsw_o) o->get(o->rhsw_o, rhsw_o);
}

// Advance nsteps; stops early (returning 1) when the CFL exceeds `cfl_limit`
// after a step, as multi/main.f90:942-946 does with `stop`; 2 on a NaN.
int oracle_step(void* h, int nsteps, double cfl_limit, oracle_diag* d) {
  Oracle* o = static_cast<Oracle*>(h);
  int rc = 0;
  for (int s = 0; s < nsteps; ++s) {
    o->step();
    const double cou = o->gumax * o->prm.dt * o->dxi;
    if (!(cou == cou)) { rc = 2; break; }
    if (cou > cfl_limit) { rc = 1; break; }
  }
  if (d) {
    d->umax = o->gumax;
    d->cfl = o->gumax * o->prm.dt * o->dxi;
    d->umean = o->last_means[0];
    d->vmean = o->last_means[1];
    d->wmean = o->last_means[2];
    d->step = o->nstep;
  }
  return rc;
}

// Stand-alone Poisson solve: rhs (raw interior) -> p (raw interior), using
// the same FFT path and k^2 convention as the step.
void oracle_poisson(void* h, const double* rhs, double* p) {
  Oracle* o = static_cast<Oracle*>(h);
  o->put(o->rhsp, rhs);
  o->poisson();
  o->get(o->p, p);
}

// 1D transform of n complex values (interleaved re,im), sign -1 forward.
void oracle_fft1d(int n, double* data, int sign) {
  FFTPlan pl;
  pl.init(n);
  std::vector<cplx> scr(n);
  pl.run(reinterpret_cast<cplx*>(data), scr.data(), sign);
}

// Dissipation 2*nu*<S_ij S_ij> with centred differences and periodic wrap,
// following post/compute_diss/main.f90:72-117.  With pi_f32=1, pi is the
// default-real literal of post/compute_diss/module.f90:5 (float32-rounded),
// which the val/ curves were made with; dx = 2*pi/(n-1).
double oracle_dissipation(int n, const double* u, const double* v, const double* w, double nu, int pi_f32) {
  const double pi = pi_f32 ? (double)(float)3.14159265358979 : 3.14159265358979;
  const double lx = 2 * pi;
  const double dx = lx / (n - 1);
  const double dxi = 1.0 / dx;
  auto I = [n](int i, int j, int k) { return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * k); };
  double eps = 0.0;
#pragma omp parallel for collapse(2) reduction(+ : eps)
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int ip = (i + 1) % n, im = (i + n - 1) % n, jp = (j + 1) % n, jm = (j + n - 1) % n,
                  kp = (k + 1) % n, km = (k + n - 1) % n;
        const double dudx = (u[I(ip, j, k)] - u[I(im, j, k)]) * 0.5 * dxi;
        const double dudy = (u[I(i, jp, k)] - u[I(i, jm, k)]) * 0.5 * dxi;
        const double dudz = (u[I(i, j, kp)] - u[I(i, j, km)]) * 0.5 * dxi;
        const double dvdx = (v[I(ip, j, k)] - v[I(im, j, k)]) * 0.5 * dxi;
        const double dvdy = (v[I(i, jp, k)] - v[I(i, jm, k)]) * 0.5 * dxi;
        const double dvdz = (v[I(i, j, kp)] - v[I(i, j, km)]) * 0.5 * dxi;
        const double dwdx = (w[I(ip, j, k)] - w[I(im, j, k)]) * 0.5 * dxi;
        const double dwdy = (w[I(i, jp, k)] - w[I(i, jm, k)]) * 0.5 * dxi;
        const double dwdz = (w[I(i, j, kp)] - w[I(i, j, km)]) * 0.5 * dxi;
        const double S11 = dudx, S22 = dvdy, S33 = dwdz;
        const double S12 = 0.5 * (dudy + dvdx), S13 = 0.5 * (dudz + dwdx), S23 = 0.5 * (dvdz + dwdy);
        eps += S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
      }
  return 2 * nu * eps / n / n / n;
}

// Drop count and sizes, post/DropCountSize: cells with phi >= 0.5
// (get_interface.f90:15), the x-fastest scan starting a new drop at every
// foreground cell not yet taken (get_interface.f90:28-40), the flood fill over
// the 26 neighbours with periodic wrap (flood_fill.f90:1-127; iterative here,
// the recursion overflows the stack for large drops), and
// deq = dx*(6/pi*vol)^(1/3) (calculate_deq.f90:29-33).  Returns the count;
// the first `capacity` drops' cell counts and diameters go to cells / deq.
int oracle_drop_count(int n, const double* phi, int capacity, int64_t* cells, double* deq, double dx) {
  const size_t N3 = (size_t)n * n * n, nn = (size_t)n * n;
  std::vector<unsigned char> top(N3);
  for (size_t g = 0; g < N3; ++g) top[g] = phi[g] >= 0.5 ? 1 : 0;
  const double pi = 4.0 * std::atan(1.0), n6opi = 6.0 / pi;
  int count = 0;
  std::vector<size_t> stack;
  for (size_t g0 = 0; g0 < N3; ++g0) {
    if (!top[g0]) continue;
    ++count;
    int64_t vol = 0;
    top[g0] = 0;
    stack.assign(1, g0);
    while (!stack.empty()) {
      const size_t g = stack.back();
      stack.pop_back();
      ++vol;
      const int i = (int)(g % n), j = (int)((g / n) % n), k = (int)(g / nn);
      for (int dk = -1; dk <= 1; ++dk)
        for (int dj = -1; dj <= 1; ++dj)
          for (int di = -1; di <= 1; ++di) {
            if (!di && !dj && !dk) continue;
            const size_t nb = (size_t)((i + di + n) % n) + (size_t)n * ((j + dj + n) % n) + nn * ((k + dk + n) % n);
            if (top[nb]) {
              top[nb] = 0;
              stack.push_back(nb);
            }
          }
    }
    if (count <= capacity) {
      cells[count - 1] = vol;
      deq[count - 1] = dx * std::pow(n6opi * (double)vol, 1.0 / 3.0);
    }
  }
  return count;
}

}  // extern "C"
