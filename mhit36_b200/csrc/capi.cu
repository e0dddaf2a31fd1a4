// C ABI of libmhit (declared in include/mhit.h).
//
// A handle owns the resident device state of one simulation, one CUDA stream,
// and two CUDA graphs (one per parity of the phi ping-pong buffer) that hold
// the kernels of one timestep.  mhit_step replays them; step-dependent
// scalars (gamma, AB2 weights, the pending mean) live in a device control
// block, so no graph is ever re-captured and nothing crosses PCIe per step
// except the optional 100-byte diagnostics read.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <string>
#include <vector>

#include "internal.h"
#include "mhit.h"

using mhit::Ctrl;
using mhit::StepConst;

struct mhit_handle {
  int n = 0, precision = 0, phase_field = 0, device = 0;
  mhit_params prm;
  StepConst c;
  cudaStream_t st = nullptr;
  // FP64 state
  double *u = nullptr, *v = nullptr, *w = nullptr;
  double *us = nullptr, *vs = nullptr, *ws = nullptr;
  double *ru = nullptr, *rv = nullptr, *rw = nullptr;
  double* phi[2] = {nullptr, nullptr};
  double* p = nullptr;
  double2* spec = nullptr;
  double2* tw = nullptr;
  double* k2tab = nullptr;
  double *fsin = nullptr, *fcos = nullptr;
  double* partials = nullptr;
  int nparts = 0;
  Ctrl* ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned mirror
  long long nstep_host = 0;
  bool has_fields = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  size_t bytes = 0;
  std::vector<void*> allocs;
  std::string last_error;
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int cuda_fail(mhit_handle* h, cudaError_t e, const char* where) {
  if (h) {
    h->last_error = std::string(where) + ": " + cudaGetErrorString(e);
  }
  return e == cudaErrorMemoryAllocation ? MHIT_ERR_NOMEM : MHIT_ERR_CUDA;
}

#define CK(h, call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
  } while (0)

template <class P> cudaError_t dalloc(mhit_handle* h, P** ptr, size_t bytes) {
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e) return e;
  h->allocs.push_back(q);
  h->bytes += bytes;
  *ptr = static_cast<P*>(q);
  return cudaSuccess;
}

void free_all(mhit_handle* h) {
  for (int i = 0; i < 2; ++i)
    if (h->graph[i]) cudaGraphExecDestroy(h->graph[i]);
  for (void* q : h->allocs) cudaFree(q);
  h->allocs.clear();
  if (h->h_ctrl) cudaFreeHost(h->h_ctrl);
  if (h->st) cudaStreamDestroy(h->st);
}

bool size_supported(int n) {
  bool built = false;
#define MHIT_CASE(NN) built |= (n == NN);
  MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
  return built && mhit::stencil_size_ok(n);
}

mhit::StencilArgs<double> stencil_args(mhit_handle* h, int cur) {
  mhit::StencilArgs<double> a;
  a.u = h->u; a.v = h->v; a.w = h->w;
  a.phi_in = h->phi[cur];
  a.phi_out = h->phi[cur ^ 1];
  a.us = h->us; a.vs = h->vs; a.ws = h->ws;
  a.ru = h->ru; a.rv = h->rv; a.rw = h->rw;
  a.p = h->p;
  a.uo = h->u; a.vo = h->v; a.wo = h->w;
  a.partials = h->partials;
  a.fsin = h->fsin; a.fcos = h->fcos;
  a.ctrl = h->ctrl;
  a.c = h->c;
  return a;
}

// Enqueue the kernels of one step reading phi[cur] (9 launches with ACDI).
cudaError_t enqueue_step(mhit_handle* h, int cur) {
  mhit::StencilArgs<double> a = stencil_args(h, cur);
  cudaError_t e;
  if (h->phase_field) {
    if ((e = mhit::launch_phase<double>(a, h->st))) return e;
    a.phi_in = h->phi[cur ^ 1];  // momentum reads the updated phi
  }
  if ((e = mhit::launch_momentum<double>(a, h->phase_field != 0, h->st))) return e;
  mhit::PoissonArgs<double> pa;
  pa.us = h->us; pa.vs = h->vs; pa.ws = h->ws;
  pa.rhs = nullptr;
  pa.spec = h->spec;
  pa.p = h->p;
  pa.tw = h->tw;
  pa.k2tab = h->k2tab;
  pa.ctrl = h->ctrl;
  pa.cdiv = h->c.cdiv;
  if ((e = mhit::launch_poisson<double>(h->n, pa, h->st))) return e;
  if ((e = mhit::launch_project<double>(a, h->st))) return e;
  return mhit::launch_finalize(h->partials, h->nparts, h->ctrl, h->c, h->st);
}

cudaError_t build_graph(mhit_handle* h, int cur) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal);
  if (e) return e;
  cudaError_t e2 = enqueue_step(h, cur);
  e = cudaStreamEndCapture(h->st, &g);
  if (e2) {
    if (g) cudaGraphDestroy(g);
    return e2;
  }
  if (e) return e;
  e = cudaGraphInstantiate(&h->graph[cur], g, 0);
  cudaGraphDestroy(g);
  return e;
}

void reset_ctrl(mhit_handle* h) {
  Ctrl* c = h->h_ctrl;
  memset(c, 0, sizeof(Ctrl));
  c->gumax = 1.0;  // multi/main.f90:325
  c->alpha = 1.0;  // multi/main.f90:323-324
  c->beta = 0.0;
  c->cfl_limit = h->prm.cfl_limit;
}

int layout_ok(int layout) { return layout == MHIT_LAYOUT_RAW || layout == MHIT_LAYOUT_PIX_HALO; }

// host (layout) -> device raw, n^2 doubles per z plane.
cudaError_t upload(mhit_handle* h, double* dst, const double* src, int layout) {
  const int n = h->n;
  const size_t plane = (size_t)n * n;
  if (layout == MHIT_LAYOUT_RAW) return cudaMemcpyAsync(dst, src, plane * n * sizeof(double), cudaMemcpyHostToDevice, h->st);
  for (int k = 0; k < n; ++k) {
    const double* s = src + (size_t)n * (1 + (size_t)(n + 2) * (k + 1));
    cudaError_t e = cudaMemcpyAsync(dst + plane * k, s, plane * sizeof(double), cudaMemcpyHostToDevice, h->st);
    if (e) return e;
  }
  return cudaSuccess;
}

cudaError_t download(mhit_handle* h, double* dst, const double* src, int layout) {
  const int n = h->n;
  const size_t plane = (size_t)n * n;
  if (layout == MHIT_LAYOUT_RAW) return cudaMemcpyAsync(dst, src, plane * n * sizeof(double), cudaMemcpyDeviceToHost, h->st);
  for (int k = 0; k < n; ++k) {
    double* d = dst + (size_t)n * (1 + (size_t)(n + 2) * (k + 1));
    cudaError_t e = cudaMemcpyAsync(d, src + plane * k, plane * sizeof(double), cudaMemcpyDeviceToHost, h->st);
    if (e) return e;
  }
  return cudaSuccess;
}

// Periodic halo fill of a host (nx, ny+2, nz+2) array (after download).
void fill_halo_host(double* a, int n) {
  const size_t row = (size_t)n, sy = (size_t)n + 2;
  for (int k = 1; k <= n; ++k) {
    double* pl = a + row * sy * k;
    memcpy(pl, pl + row * n, row * sizeof(double));
    memcpy(pl + row * (n + 1), pl + row, row * sizeof(double));
  }
  memcpy(a, a + row * sy * n, row * sy * sizeof(double));
  memcpy(a + row * sy * (n + 1), a + row * sy, row * sy * sizeof(double));
}

void fill_diag(mhit_handle* h, mhit_diag* d) {
  if (!d) return;
  const Ctrl* c = h->h_ctrl;
  d->umax = c->gumax;
  d->cfl = c->cfl;
  d->umean = c->last_mean[0];
  d->vmean = c->last_mean[1];
  d->wmean = c->last_mean[2];
  d->gamma = 1.0 * c->gumax;
  d->step = c->nstep;
  d->status = c->status;
  d->reserved = 0;
}

cudaError_t pull_ctrl(mhit_handle* h) {
  cudaError_t e = cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->st);
  if (e) return e;
  return cudaStreamSynchronize(h->st);
}

}  // namespace

extern "C" {

void mhit_default_params(mhit_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  // multi/input.inp:1-16
  p->restart = 0; p->tstart = 0; p->tfin = 20000; p->dump = 1000;
  p->inflow = 0; p->inphi = 0;
  p->dt = 0.0002; p->mu = 0.006; p->rho = 1.0;
  p->f1 = 0.0; p->f2 = 0.0; p->f3 = 0.0; p->k0 = 2.0;
  p->radius = 0.5; p->sigma = 1.0; p->epsr = 1.0;
  p->lin_force = 0.0;
  p->k2_mode = MHIT_K2_SPECTRAL;
  p->grid_mode = MHIT_GRID_REFERENCE;
  p->cfl_limit = 7.0;
  p->tanh_identity = 0;
}

int mhit_size_supported(int n) { return size_supported(n) ? 1 : 0; }

const char* mhit_strerror(int s) {
  switch (s) {
    case MHIT_OK: return "ok";
    case MHIT_ERR_INVALID: return "invalid argument";
    case MHIT_ERR_CUDA: return "CUDA runtime error";
    case MHIT_ERR_NOMEM: return "device out of memory";
    case MHIT_ERR_CFL: return "CFL above the limit";
    case MHIT_ERR_NONFINITE: return "non-finite value in the velocity reductions";
    case MHIT_ERR_IO: return "field file missing or of the wrong size";
    case MHIT_ERR_UNSUPPORTED: return "unsupported grid size or option";
    case MHIT_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

const char* mhit_last_error(mhit_handle* h) { return h ? h->last_error.c_str() : ""; }

int mhit_create(const mhit_params* p, int nx, int ny, int nz, int precision, int phase_field, mhit_handle** out) {
  if (!p || !out) return MHIT_ERR_INVALID;
  *out = nullptr;
  if (nx != ny || nx != nz) return MHIT_ERR_UNSUPPORTED;  // ny = nz = nx (multi/module.f90:2-3)
  if (!size_supported(nx)) return MHIT_ERR_UNSUPPORTED;
  if (precision != MHIT_FP64) return MHIT_ERR_UNSUPPORTED;
  if (!(p->dt > 0) || !(p->rho > 0) || !(p->epsr > 0)) return MHIT_ERR_INVALID;
  mhit_handle* h = new mhit_handle();
  h->n = nx;
  h->precision = precision;
  h->phase_field = phase_field ? 1 : 0;
  h->prm = *p;
  if (!(h->prm.cfl_limit > 0)) h->prm.cfl_limit = 7.0;
  cudaGetDevice(&h->device);
  const int n = nx;
  // multi/readinput.f90:34-43 (dx per grid_mode)
  const double twopi = 8.0 * atan(1.0);
  const double lx = twopi;
  const double dx = (p->grid_mode == MHIT_GRID_CONSISTENT) ? lx / n : lx / (n - 1);
  StepConst& c = h->c;
  memset(&c, 0, sizeof(c));
  c.n = n;
  c.dt = p->dt; c.mu = p->mu; c.rho = p->rho;
  c.rhoi = 1.0 / p->rho;
  c.dxi = 1.0 / dx;
  c.ddxi = 1.0 / dx / dx;
  c.eps = p->epsr * dx;
  c.epsi = 1.0 / c.eps;
  c.enumv = (double)(float)1.e-16;  // single-precision literal, multi/readinput.f90:43
  c.tiny = (double)(float)1.0E-16;  // multi/main.f90:436
  c.sigma = p->sigma;
  c.lin_force = p->lin_force;
  c.f1 = p->f1; c.f2 = p->f2; c.f3 = p->f3;
  c.abc = (p->f1 != 0.0 || p->f2 != 0.0 || p->f3 != 0.0) ? 1 : 0;
  c.tanh_identity = p->tanh_identity ? 1 : 0;
  c.cdiv = p->rho * c.dxi / p->dt;
  c.dtr = p->dt / p->rho;

  int rc = MHIT_OK;
  auto fail = [&](cudaError_t e, const char* what) {
    rc = cuda_fail(h, e, what);
    return rc;
  };
  do {
    cudaError_t e;
    if ((e = mhit::prepare_stencils())) { fail(e, "prepare_stencils"); break; }
    if ((e = mhit::prepare_poisson(n))) { fail(e, "prepare_poisson"); break; }
    if ((e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking))) { fail(e, "stream"); break; }
    const size_t N3 = (size_t)n * n * n;
    const size_t fb = N3 * sizeof(double);
    double** fields[] = {&h->u, &h->v, &h->w, &h->us, &h->vs, &h->ws, &h->ru, &h->rv, &h->rw, &h->p};
    bool bad = false;
    for (double** f : fields) {
      if ((e = dalloc(h, f, fb))) { fail(e, "cudaMalloc field"); bad = true; break; }
    }
    if (bad) break;
    if (h->phase_field) {
      if ((e = dalloc(h, &h->phi[0], fb)) || (e = dalloc(h, &h->phi[1], fb))) { fail(e, "cudaMalloc phi"); break; }
    }
    const size_t pitch = mhit::spectrum_pitch(n);
    const size_t sb = (size_t)n * n * pitch * sizeof(double2);
    if ((e = dalloc(h, &h->spec, sb))) { fail(e, "cudaMalloc spectrum"); break; }
    if ((e = cudaMemsetAsync(h->spec, 0, sb, h->st))) { fail(e, "memset"); break; }
    h->nparts = mhit::project_partials(n);
    if ((e = dalloc(h, &h->partials, (size_t)h->nparts * 6 * sizeof(double)))) { fail(e, "cudaMalloc partials"); break; }
    if ((e = dalloc(h, &h->ctrl, sizeof(Ctrl)))) { fail(e, "cudaMalloc ctrl"); break; }
    if ((e = cudaMallocHost(&h->h_ctrl, sizeof(Ctrl)))) { fail(e, "cudaMallocHost"); break; }
    // tables: twiddles e^{-2 pi i m/n}, k^2, forcing sin/cos
    std::vector<double2> tw(n);
    for (int m = 0; m < n; ++m) {
      long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
      tw[m].x = (double)cosl(a);
      tw[m].y = -(double)sinl(a);
    }
    std::vector<double> k2(n), fs(n), fc(n), x(n);
    const double pi = 4.0 * atan(1.0);
    for (int m = 0; m < n; ++m) {
      if (p->k2_mode == MHIT_K2_FD) {
        const double s = sin(pi * m / n);
        k2[m] = (4.0 * c.ddxi) * (s * s);
      } else {
        // kx = (i-1)*(twopi/lx) or (i-1-nx)*(twopi/lx)   (multi/main.f90:154-159)
        const double kk = (m < n / 2 ? (double)m : (double)(m - n)) * (twopi / lx);
        k2[m] = kk * kk;
      }
    }
    x[0] = 0.0;  // multi/main.f90:150-153
    for (int m = 1; m < n; ++m) x[m] = x[m - 1] + dx;
    for (int m = 0; m < n; ++m) {
      fs[m] = sin(p->k0 * x[m]);
      fc[m] = cos(p->k0 * x[m]);
    }
    if ((e = dalloc(h, &h->tw, n * sizeof(double2))) || (e = dalloc(h, &h->k2tab, n * sizeof(double))) ||
        (e = dalloc(h, &h->fsin, n * sizeof(double))) || (e = dalloc(h, &h->fcos, n * sizeof(double)))) {
      fail(e, "cudaMalloc tables");
      break;
    }
    if ((e = cudaMemcpyAsync(h->tw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice, h->st)) ||
        (e = cudaMemcpyAsync(h->k2tab, k2.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->st)) ||
        (e = cudaMemcpyAsync(h->fsin, fs.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->st)) ||
        (e = cudaMemcpyAsync(h->fcos, fc.data(), n * sizeof(double), cudaMemcpyHostToDevice, h->st))) {
      fail(e, "upload tables");
      break;
    }
    reset_ctrl(h);
    if ((e = cudaMemcpyAsync(h->ctrl, h->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, h->st))) { fail(e, "ctrl"); break; }
    if ((e = cudaStreamSynchronize(h->st))) { fail(e, "sync"); break; }
  } while (0);
  if (rc != MHIT_OK) {
    fprintf(stderr, "mhit_create: %s\n", h->last_error.c_str());
    free_all(h);
    delete h;
    return rc;
  }
  *out = h;
  return MHIT_OK;
}

int mhit_destroy(mhit_handle* h) {
  if (!h) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  free_all(h);
  delete h;
  return MHIT_OK;
}

int mhit_set_fields(mhit_handle* h, const double* u, const double* v, const double* w, const double* phi,
                    int layout) {
  if (!h || !u || !v || !w || !layout_ok(layout)) return MHIT_ERR_INVALID;
  if (h->phase_field && !phi) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  const size_t fb = (size_t)h->n * h->n * h->n * sizeof(double);
  CK(h, upload(h, h->u, u, layout));
  CK(h, upload(h, h->v, v, layout));
  CK(h, upload(h, h->w, w, layout));
  if (h->phase_field) CK(h, upload(h, h->phi[0], phi, layout));
  // rhs_o starts at zero; beta = 0 on the first step (multi/main.f90:324)
  CK(h, cudaMemsetAsync(h->ru, 0, fb, h->st));
  CK(h, cudaMemsetAsync(h->rv, 0, fb, h->st));
  CK(h, cudaMemsetAsync(h->rw, 0, fb, h->st));
  CK(h, cudaMemsetAsync(h->p, 0, fb, h->st));
  reset_ctrl(h);
  CK(h, cudaMemcpyAsync(h->ctrl, h->h_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  h->nstep_host = 0;
  h->has_fields = true;
  return MHIT_OK;
}

int mhit_sync_state(mhit_handle* h) {
  if (!h) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  CK(h, mhit::launch_materialize<double>(h->u, h->v, h->w, h->n, h->ctrl, h->st));
  return MHIT_OK;
}

int mhit_get_fields(mhit_handle* h, double* u, double* v, double* w, double* phi, int layout) {
  if (!h || !layout_ok(layout)) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  CK(h, mhit::launch_materialize<double>(h->u, h->v, h->w, h->n, h->ctrl, h->st));
  CK(h, pull_ctrl(h));
  const int cur = (int)(h->h_ctrl->nstep & 1);
  if (u) CK(h, download(h, u, h->u, layout));
  if (v) CK(h, download(h, v, h->v, layout));
  if (w) CK(h, download(h, w, h->w, layout));
  if (phi && h->phase_field) CK(h, download(h, phi, h->phi[cur], layout));
  CK(h, cudaStreamSynchronize(h->st));
  if (layout == MHIT_LAYOUT_PIX_HALO) {
    double* outs[4] = {u, v, w, h->phase_field ? phi : nullptr};
    for (double* o : outs)
      if (o) fill_halo_host(o, h->n);
  }
  return MHIT_OK;
}

int mhit_get_pressure(mhit_handle* h, double* p, int layout) {
  if (!h || !p || !layout_ok(layout)) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  CK(h, download(h, p, h->p, layout));
  CK(h, cudaStreamSynchronize(h->st));
  if (layout == MHIT_LAYOUT_PIX_HALO) fill_halo_host(p, h->n);
  return MHIT_OK;
}

int mhit_step(mhit_handle* h, int nsteps, mhit_diag* out) {
  if (!h || nsteps < 0) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  for (int s = 0; s < nsteps; ++s) {
    const int cur = (int)(h->nstep_host & 1);
    if (!h->graph[cur]) CK(h, build_graph(h, cur));
    CK(h, cudaGraphLaunch(h->graph[cur], h->st));
    ++h->nstep_host;
  }
  CK(h, pull_ctrl(h));
  h->nstep_host = h->h_ctrl->nstep;  // fewer if a step raised the error status
  fill_diag(h, out);
  return h->h_ctrl->status;
}

// Enqueue `nsteps` steps without waiting or reading anything back.
int mhit_step_async(mhit_handle* h, int nsteps) {
  if (!h || nsteps < 0) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  for (int s = 0; s < nsteps; ++s) {
    const int cur = (int)(h->nstep_host & 1);
    if (!h->graph[cur]) CK(h, build_graph(h, cur));
    CK(h, cudaGraphLaunch(h->graph[cur], h->st));
    ++h->nstep_host;
  }
  return MHIT_OK;
}

int mhit_get_diag(mhit_handle* h, mhit_diag* out) {
  if (!h || !out) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  CK(h, pull_ctrl(h));
  h->nstep_host = h->h_ctrl->nstep;
  fill_diag(h, out);
  return MHIT_OK;
}

void* mhit_stream(mhit_handle* h) { return h ? (void*)h->st : nullptr; }

int mhit_device_state(mhit_handle* h, void** u, void** v, void** w, void** phi) {
  if (!h) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  if (u) *u = h->u;
  if (v) *v = h->v;
  if (w) *w = h->w;
  if (phi) {
    CK(h, pull_ctrl(h));
    *phi = h->phase_field ? (void*)h->phi[h->h_ctrl->nstep & 1] : nullptr;
  }
  return MHIT_OK;
}

int mhit_memory_bytes(mhit_handle* h, size_t* bytes) {
  if (!h || !bytes) return MHIT_ERR_INVALID;
  *bytes = h->bytes;
  return MHIT_OK;
}

int mhit_launches_per_step(mhit_handle* h, int* n) {
  if (!h || !n) return MHIT_ERR_INVALID;
  *n = (h->phase_field ? 1 : 0) + 1 + 5 + 1 + 1;
  return MHIT_OK;
}

// Run `reps` steps with every kernel launched on its own between CUDA events
// on the handle's stream; ms[k] = mean duration of stage k.  Stage names in
// launch order: phase (ACDI only), momentum, xfwd, yfwd, zsolve, yinv, xinv,
// project, finalize.
static const char* kStageNames[] = {"phase", "momentum", "xfwd", "yfwd", "zsolve", "yinv", "xinv", "project",
                                    "finalize"};

int mhit_profile_step(mhit_handle* h, int reps, double* ms, int* nstages) {
  if (!h || !ms || !nstages || reps < 1) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  const int NS = 9;
  cudaEvent_t ev[NS + 1];
  for (int i = 0; i <= NS; ++i) CK(h, cudaEventCreate(&ev[i]));
  double acc[NS] = {0};
  for (int r = 0; r < reps; ++r) {
    const int cur = (int)(h->nstep_host & 1);
    mhit::StencilArgs<double> a = stencil_args(h, cur);
    mhit::PoissonArgs<double> pa;
    pa.us = h->us; pa.vs = h->vs; pa.ws = h->ws; pa.rhs = nullptr; pa.spec = h->spec; pa.p = h->p;
    pa.tw = h->tw; pa.k2tab = h->k2tab; pa.ctrl = h->ctrl; pa.cdiv = h->c.cdiv;
    CK(h, cudaEventRecord(ev[0], h->st));
    if (h->phase_field) CK(h, mhit::launch_phase<double>(a, h->st));
    CK(h, cudaEventRecord(ev[1], h->st));
    if (h->phase_field) a.phi_in = h->phi[cur ^ 1];
    CK(h, mhit::launch_momentum<double>(a, h->phase_field != 0, h->st));
    CK(h, cudaEventRecord(ev[2], h->st));
    for (int stage = 0; stage < 5; ++stage) {
      CK(h, mhit::launch_poisson_stage<double>(h->n, pa, stage, h->st));
      CK(h, cudaEventRecord(ev[3 + stage], h->st));
    }
    CK(h, mhit::launch_project<double>(a, h->st));
    CK(h, cudaEventRecord(ev[8], h->st));
    CK(h, mhit::launch_finalize(h->partials, h->nparts, h->ctrl, h->c, h->st));
    CK(h, cudaEventRecord(ev[9], h->st));
    CK(h, cudaEventSynchronize(ev[9]));
    for (int i = 0; i < NS; ++i) {
      float t = 0;
      CK(h, cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
      acc[i] += t;
    }
    ++h->nstep_host;
  }
  for (int i = 0; i <= NS; ++i) cudaEventDestroy(ev[i]);
  for (int i = 0; i < NS; ++i) ms[i] = acc[i] / reps;
  *nstages = NS;
  CK(h, pull_ctrl(h));
  h->nstep_host = h->h_ctrl->nstep;
  return h->h_ctrl->status;
}

const char* mhit_stage_name(int k) { return (k >= 0 && k < 9) ? kStageNames[k] : ""; }

int mhit_poisson_device(mhit_handle* h, const double* rhs_dev, double* p_dev) {
  if (!h || !rhs_dev || !p_dev) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  mhit::PoissonArgs<double> pa;
  pa.us = pa.vs = pa.ws = nullptr;
  pa.rhs = rhs_dev;
  pa.spec = h->spec;
  pa.p = p_dev;
  pa.tw = h->tw;
  pa.k2tab = h->k2tab;
  pa.ctrl = nullptr;
  pa.cdiv = h->c.cdiv;
  CK(h, mhit::launch_poisson<double>(h->n, pa, h->st));
  return MHIT_OK;
}

int mhit_poisson(mhit_handle* h, const double* rhs, double* p) {
  if (!h || !rhs || !p) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  const size_t fb = (size_t)h->n * h->n * h->n * sizeof(double);
  CK(h, cudaMemcpyAsync(h->p, rhs, fb, cudaMemcpyHostToDevice, h->st));
  int rc = mhit_poisson_device(h, h->p, h->p);
  if (rc) return rc;
  CK(h, cudaMemcpyAsync(p, h->p, fb, cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  return MHIT_OK;
}

// ------------------------------------------------------------ save / load
// Sidecar for exact resume: header + rhs_o (3 raw fields).
struct Sidecar {
  char magic[8];  // "MHITSTA1"
  int32_t n, precision, phase_field, pad;
  int64_t nstep;
  double gumax, alpha, beta, cfl;
};

static int write_raw(const std::string& path, const double* a, size_t count) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return MHIT_ERR_IO;
  size_t wr = fwrite(a, sizeof(double), count, f);
  fclose(f);
  return wr == count ? MHIT_OK : MHIT_ERR_IO;
}

static int read_raw(const std::string& path, double* a, size_t count) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return MHIT_ERR_IO;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  if (sz != (long)(count * sizeof(double))) {
    fclose(f);
    return MHIT_ERR_IO;
  }
  size_t rd = fread(a, sizeof(double), count, f);
  fclose(f);
  return rd == count ? MHIT_OK : MHIT_ERR_IO;
}

static std::string fname(const char* dir, const char* base, int t) {
  char b[64];
  snprintf(b, sizeof(b), "/%s_%08d.dat", base, t);
  return std::string(dir) + b;
}

int mhit_save(mhit_handle* h, const char* dir, int t) {
  if (!h || !dir) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  const size_t N3 = (size_t)h->n * h->n * h->n;
  std::vector<double> buf(N3);
  double* host = buf.data();
  int rc;
  const char* names[3] = {"u", "v", "w"};
  double* dev[3] = {h->u, h->v, h->w};
  DeviceGuard g(h->device);
  CK(h, mhit::launch_materialize<double>(h->u, h->v, h->w, h->n, h->ctrl, h->st));
  CK(h, pull_ctrl(h));
  for (int f = 0; f < 3; ++f) {
    CK(h, cudaMemcpy(host, dev[f], N3 * sizeof(double), cudaMemcpyDeviceToHost));
    if ((rc = write_raw(fname(dir, names[f], t), host, N3))) return rc;
  }
  if (h->phase_field) {
    CK(h, cudaMemcpy(host, h->phi[h->h_ctrl->nstep & 1], N3 * sizeof(double), cudaMemcpyDeviceToHost));
    if ((rc = write_raw(fname(dir, "phi", t), host, N3))) return rc;
  }
  char b[64];
  snprintf(b, sizeof(b), "/state_%08d.bin", t);
  FILE* f = fopen((std::string(dir) + b).c_str(), "wb");
  if (!f) return MHIT_ERR_IO;
  Sidecar sc;
  memset(&sc, 0, sizeof(sc));
  memcpy(sc.magic, "MHITSTA1", 8);
  sc.n = h->n;
  sc.precision = h->precision;
  sc.phase_field = h->phase_field;
  sc.nstep = h->h_ctrl->nstep;
  sc.gumax = h->h_ctrl->gumax;
  sc.alpha = h->h_ctrl->alpha;
  sc.beta = h->h_ctrl->beta;
  sc.cfl = h->h_ctrl->cfl;
  bool ok = fwrite(&sc, sizeof(sc), 1, f) == 1;
  double* ro[3] = {h->ru, h->rv, h->rw};
  for (int q = 0; q < 3 && ok; ++q) {
    if (cudaMemcpy(host, ro[q], N3 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ok = false;
    else ok = fwrite(host, sizeof(double), N3, f) == N3;
  }
  fclose(f);
  return ok ? MHIT_OK : MHIT_ERR_IO;
}

int mhit_load(mhit_handle* h, const char* dir, int t) {
  if (!h || !dir) return MHIT_ERR_INVALID;
  const size_t N3 = (size_t)h->n * h->n * h->n;
  std::vector<double> bu(N3), bv(N3), bw(N3), bp;
  int rc;
  if ((rc = read_raw(fname(dir, "u", t), bu.data(), N3))) return rc;
  if ((rc = read_raw(fname(dir, "v", t), bv.data(), N3))) return rc;
  if ((rc = read_raw(fname(dir, "w", t), bw.data(), N3))) return rc;
  if (h->phase_field) {
    bp.resize(N3);
    if ((rc = read_raw(fname(dir, "phi", t), bp.data(), N3))) return rc;
  }
  if ((rc = mhit_set_fields(h, bu.data(), bv.data(), bw.data(), h->phase_field ? bp.data() : nullptr,
                            MHIT_LAYOUT_RAW)))
    return rc;
  char b[64];
  snprintf(b, sizeof(b), "/state_%08d.bin", t);
  FILE* f = fopen((std::string(dir) + b).c_str(), "rb");
  if (!f) return MHIT_OK;  // reference restart: Euler first step, gumax = 1
  Sidecar sc;
  bool ok = fread(&sc, sizeof(sc), 1, f) == 1 && memcmp(sc.magic, "MHITSTA1", 8) == 0 && sc.n == h->n;
  double* ro[3] = {h->ru, h->rv, h->rw};
  DeviceGuard g(h->device);
  for (int q = 0; q < 3 && ok; ++q) {
    ok = fread(bu.data(), sizeof(double), N3, f) == N3;
    if (ok) ok = cudaMemcpy(ro[q], bu.data(), N3 * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  fclose(f);
  if (!ok) return MHIT_ERR_IO;
  // phi was uploaded into phi[0]; keep the parity convention phi[nstep & 1]
  if (h->phase_field && (sc.nstep & 1))
    CK(h, cudaMemcpyAsync(h->phi[1], h->phi[0], N3 * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
  Ctrl* c = h->h_ctrl;
  c->gumax = sc.gumax;
  c->alpha = sc.alpha;
  c->beta = sc.beta;
  c->cfl = sc.cfl;
  c->nstep = sc.nstep;
  CK(h, cudaMemcpyAsync(h->ctrl, c, sizeof(Ctrl), cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  h->nstep_host = sc.nstep;
  return MHIT_OK;
}

}  // extern "C"
