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
#include <algorithm>
#include <functional>
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
  // FP32 refinement form state (u, v, w, ustar, rhs_o, phi in FP32; the
  // Poisson solve is an FP32 solve p0 plus an FP32 correction solve dp of the
  // FP64 residual)
  float *fu = nullptr, *fv = nullptr, *fw = nullptr;
  float *fus = nullptr, *fvs = nullptr, *fws = nullptr;
  float *fru = nullptr, *frv = nullptr, *frw = nullptr;
  float* fphi[2] = {nullptr, nullptr};
  float *fp0 = nullptr, *fdp = nullptr;
  float2* fspec = nullptr;
  float2* ftw = nullptr;
  double* k2tab = nullptr;
  double *fsin = nullptr, *fcos = nullptr;
  double* partials = nullptr;
  int nparts = 0;
  // FP64 step with the fused x inverse + projection: p is not stored by the
  // step; the spectrum still holds the last step's y-inverse output, from
  // which mhit_get_pressure recomputes p.
  bool p_in_spec = false;
  // FP32 refinement form with the fused x inverse + projection: dp is not
  // stored by the step; the spectrum holds the last correction solve's
  // y-inverse output, from which dp (for the pressure and the divergence
  // check) is recomputed on request.
  bool dp_in_spec = false;
  bool have_step = false;     // a step ran since the fields were set (ustar, p0 are its own)
  double* div_out = nullptr;  // device: max |div u| of the FP64 projection (FP32 refine form)
  double* stat_partials = nullptr;
  double* stat_out = nullptr;
  double* h_stat = nullptr;  // pinned
  Ctrl* ctrl = nullptr;
  Ctrl* h_ctrl = nullptr;  // pinned mirror
  long long nstep_host = 0;
  bool has_fields = false;
  // drop counting scratch (allocated on first use)
  int* ccl_lab = nullptr;
  int* ccl_cnt = nullptr;
  int2* ccl_roots = nullptr;
  int* ccl_counter = nullptr;
  int ccl_cap = 0;
  int kz = 0;   // stencil z chunk (0: default)
  int mty = 0;  // momentum tile height (0: default for the grid size)
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
  if (h->h_stat) cudaFreeHost(h->h_stat);
  if (h->st) cudaStreamDestroy(h->st);
}

bool size_supported(int n) {
  bool built = false;
#define MHIT_CASE(NN) built |= (n == NN);
  MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
  return built && mhit::stencil_size_ok(n);
}

template <class T> struct Buffers;
template <> struct Buffers<double> {
  static mhit::StencilArgs<double> args(mhit_handle* h, int cur) {
    mhit::StencilArgs<double> a;
    a.u = h->u; a.v = h->v; a.w = h->w;
    a.phi_in = h->phi[cur];
    a.phi_out = h->phi[cur ^ 1];
    a.us = h->us; a.vs = h->vs; a.ws = h->ws;
    a.ru = h->ru; a.rv = h->rv; a.rw = h->rw;
    a.p = h->p;
    a.uo = h->u; a.vo = h->v; a.wo = h->w;
    return a;
  }
};
template <> struct Buffers<float> {
  static mhit::StencilArgs<float> args(mhit_handle* h, int cur) {
    mhit::StencilArgs<float> a;
    a.u = h->fu; a.v = h->fv; a.w = h->fw;
    a.phi_in = h->fphi[cur];
    a.phi_out = h->fphi[cur ^ 1];
    a.us = h->fus; a.vs = h->fvs; a.ws = h->fws;
    a.ru = h->fru; a.rv = h->frv; a.rw = h->frw;
    a.p = h->fp0;
    a.uo = h->fu; a.vo = h->fv; a.wo = h->fw;
    return a;
  }
};

template <class T> mhit::StencilArgs<T> stencil_args(mhit_handle* h, int cur) {
  mhit::StencilArgs<T> a = Buffers<T>::args(h, cur);
  a.partials = h->partials;
  a.fsin = h->fsin;
  a.fcos = h->fcos;
  a.ctrl = h->ctrl;
  a.c = h->c;
  return a;
}

typedef std::pair<const char*, std::function<cudaError_t()>> Stage;

// The kernels of one step reading phi[cur], in launch order.
//   FP64: [phase] momentum xfwd yfwd zsolve yinv xinv project finalize
//   FP32 refine: [phase] momentum, solve 1 (xfwd yfwd zsolve yinv xinv -> p0),
//     solve 2 of the FP64 residual (xres yfwd2 zsolve2 yinv2 xinv2 -> dp),
//     project (FP64), finalize
std::vector<Stage> step_stages(mhit_handle* h, int cur) {
  std::vector<Stage> v;
  cudaStream_t st = h->st;
  const int n = h->n;
  const int kz = h->kz, mty = h->mty ? h->mty : mhit::default_mty(n, h->precision != MHIT_FP64);
  const bool pf = h->phase_field != 0;
  static const char* pnames[5] = {"xfwd", "yfwd", "zsolve", "yinv", "xinv"};
  static const char* rnames[5] = {"xres", "yfwd2", "zsolve2", "yinv2", "xinv2"};
  if (h->precision == MHIT_FP64) {
    mhit::StencilArgs<double> a = stencil_args<double>(h, cur);
    mhit::StencilArgs<double> am = a;
    if (pf) {
      v.push_back({"phase", [a, st, kz] { return mhit::launch_phase<double>(a, st, kz); }});
      am.phi_in = h->phi[cur ^ 1];  // momentum reads the updated phi
    }
    v.push_back({"momentum", [am, pf, st, kz, mty] { return mhit::launch_momentum<double>(am, pf, st, kz, mty); }});
    mhit::PoissonArgs<double> pa;
    pa.us = h->us; pa.vs = h->vs; pa.ws = h->ws;
    pa.spec = h->spec; pa.p = h->p; pa.tw = h->tw; pa.k2tab = h->k2tab; pa.ctrl = h->ctrl;
    pa.cdiv = h->c.cdiv; pa.ddxi = h->c.ddxi;
    const bool fused = mhit::fused_projection(n) != 0;
    for (int k = 0; k < (fused ? 4 : 5); ++k)
      v.push_back({pnames[k], [pa, n, k, st] { return mhit::launch_poisson_stage<double>(n, pa, k, st); }});
    if (fused)
      v.push_back({"xinvproj", [pa, a, n, st] { return mhit::launch_xinv_project(n, pa, a, st); }});
    else
      v.push_back({"project", [a, st] { return mhit::launch_project<double>(a, st); }});
    Ctrl* ctrl = h->ctrl;
    double* part = h->partials;
    int np = h->nparts;
    StepConst c = h->c;
    v.push_back({"finalize", [part, np, ctrl, c, st] { return mhit::launch_finalize(part, np, 6, ctrl, c, st); }});
  } else {
    mhit::StencilArgs<float> a = stencil_args<float>(h, cur);
    mhit::StencilArgs<float> am = a;
    if (pf) {
      v.push_back({"phase", [a, st, kz] { return mhit::launch_phase<float>(a, st, kz); }});
      am.phi_in = h->fphi[cur ^ 1];
    }
    v.push_back({"momentum", [am, pf, st, kz, mty] { return mhit::launch_momentum<float>(am, pf, st, kz, mty); }});
    mhit::PoissonArgs<float> pa;
    pa.us = h->fus; pa.vs = h->fvs; pa.ws = h->fws;
    pa.spec = h->fspec; pa.p = h->fp0; pa.tw = h->ftw; pa.k2tab = h->k2tab; pa.ctrl = h->ctrl;
    pa.cdiv = h->c.cdiv; pa.ddxi = h->c.ddxi;
    for (int k = 0; k < 5; ++k)
      v.push_back({pnames[k], [pa, n, k, st] { return mhit::launch_poisson_stage<float>(n, pa, k, st); }});
    mhit::PoissonArgs<float> pr = pa;
    pr.pres = h->fp0;  // residual r - L(p0) in FP64
    pr.p = h->fdp;
    const bool fused = mhit::fused_projection(n) != 0;
    for (int k = 0; k < (fused ? 4 : 5); ++k)
      v.push_back({rnames[k], [pr, n, k, st] { return mhit::launch_poisson_stage<float>(n, pr, k, st); }});
    float* dp = h->fdp;
    if (fused)
      v.push_back({"xinvproj", [pr, a, n, st] { return mhit::launch_xinv_project<float>(n, pr, a, st); }});
    else
      v.push_back({"project", [a, dp, st] { return mhit::launch_project_refine(a, dp, st); }});
    Ctrl* ctrl = h->ctrl;
    double* part = h->partials;
    int np = h->nparts;
    StepConst c = h->c;
    const int stride = fused ? 6 : 7;
    v.push_back({"finalize", [part, np, ctrl, c, st, stride] {
                   return mhit::launch_finalize(part, np, stride, ctrl, c, st);
                 }});
  }
  return v;
}

cudaError_t enqueue_step(mhit_handle* h, int cur) {
  for (auto& stg : step_stages(h, cur)) {
    cudaError_t e = stg.second();
    if (e) return e;
  }
  return cudaSuccess;
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

// A device field of either form: FP64 or FP32 storage, raw layout.
struct DevField {
  void* ptr;
  bool f32;
};

// host float64 (layout) -> device field; FP32 fields are rounded on the host.
cudaError_t put_field(mhit_handle* h, DevField d, const double* src, int layout) {
  if (!d.f32) return upload(h, static_cast<double*>(d.ptr), src, layout);
  const int n = h->n;
  const size_t plane = (size_t)n * n;
  std::vector<float> tmp(plane * n);
  for (int k = 0; k < n; ++k) {
    const double* s = (layout == MHIT_LAYOUT_RAW) ? src + plane * k : src + (size_t)n * (1 + (size_t)(n + 2) * (k + 1));
    float* t = tmp.data() + plane * k;
    for (size_t q = 0; q < plane; ++q) t[q] = (float)s[q];
  }
  cudaError_t e = cudaMemcpyAsync(d.ptr, tmp.data(), tmp.size() * sizeof(float), cudaMemcpyHostToDevice, h->st);
  if (e) return e;
  return cudaStreamSynchronize(h->st);  // tmp dies here
}

// device field -> host float64 (layout); synchronous for FP32 fields.
cudaError_t get_field(mhit_handle* h, double* dst, DevField d, int layout) {
  if (!d.f32) return download(h, dst, static_cast<const double*>(d.ptr), layout);
  const int n = h->n;
  const size_t plane = (size_t)n * n;
  std::vector<float> tmp(plane * n);
  cudaError_t e = cudaMemcpyAsync(tmp.data(), d.ptr, tmp.size() * sizeof(float), cudaMemcpyDeviceToHost, h->st);
  if (e) return e;
  if ((e = cudaStreamSynchronize(h->st))) return e;
  for (int k = 0; k < n; ++k) {
    double* t = (layout == MHIT_LAYOUT_RAW) ? dst + plane * k : dst + (size_t)n * (1 + (size_t)(n + 2) * (k + 1));
    const float* s = tmp.data() + plane * k;
    for (size_t q = 0; q < plane; ++q) t[q] = (double)s[q];
  }
  return cudaSuccess;
}

bool f32(mhit_handle* h) { return h->precision == MHIT_FP32_REFINE; }
DevField fu(mhit_handle* h) { return f32(h) ? DevField{h->fu, true} : DevField{h->u, false}; }
DevField fv(mhit_handle* h) { return f32(h) ? DevField{h->fv, true} : DevField{h->v, false}; }
DevField fw(mhit_handle* h) { return f32(h) ? DevField{h->fw, true} : DevField{h->w, false}; }
DevField fphi(mhit_handle* h, int cur) { return f32(h) ? DevField{h->fphi[cur], true} : DevField{h->phi[cur], false}; }
DevField frhs_o(mhit_handle* h, int q) {
  if (f32(h)) return DevField{q == 0 ? h->fru : (q == 1 ? h->frv : h->frw), true};
  return DevField{q == 0 ? h->ru : (q == 1 ? h->rv : h->rw), false};
}
size_t elem_size(mhit_handle* h) { return f32(h) ? sizeof(float) : sizeof(double); }

cudaError_t materialize(mhit_handle* h) {
  if (f32(h)) return mhit::launch_materialize<float>(h->fu, h->fv, h->fw, h->n, h->ctrl, h->st);
  return mhit::launch_materialize<double>(h->u, h->v, h->w, h->n, h->ctrl, h->st);
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
  d->max_div = c->max_div;
  d->step = c->nstep;
  d->status = c->status;
  d->reserved = 0;
}

cudaError_t pull_ctrl(mhit_handle* h) {
  cudaError_t e = cudaMemcpyAsync(h->h_ctrl, h->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, h->st);
  if (e) return e;
  return cudaStreamSynchronize(h->st);
}

bool refine_fused(mhit_handle* h) { return f32(h) && mhit::fused_projection(h->n); }

// FP32 refinement form with the fused projection: dp = x inverse of the
// last correction solve's spectrum, into the dp buffer.
cudaError_t materialize_dp(mhit_handle* h) {
  if (!h->dp_in_spec) return cudaSuccess;
  mhit::PoissonArgs<float> pr;
  pr.spec = h->fspec;
  pr.p = h->fdp;
  pr.tw = h->ftw;
  pr.k2tab = h->k2tab;
  pr.ctrl = nullptr;
  cudaError_t e = mhit::launch_poisson_stage<float>(h->n, pr, 4, h->st);
  if (!e) h->dp_in_spec = false;
  return e;
}

// max |div u| of the last step's FP64 projection (FP32 refinement form),
// measured from the stored ustar, p0 and dp; -1 before the first step.
cudaError_t refine_max_div(mhit_handle* h, double* out) {
  *out = h->h_ctrl->max_div;
  if (!refine_fused(h) || !h->have_step) return cudaSuccess;
  cudaError_t e = materialize_dp(h);
  if (e) return e;
  const int cur = (int)(h->h_ctrl->nstep & 1);
  if ((e = mhit::launch_refine_divergence(stencil_args<float>(h, cur), h->fdp, h->div_out, h->st))) return e;
  if ((e = cudaMemcpyAsync(h->h_stat, h->div_out, sizeof(double), cudaMemcpyDeviceToHost, h->st))) return e;
  if ((e = cudaStreamSynchronize(h->st))) return e;
  *out = h->h_stat[0];
  return cudaSuccess;
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
  p->tanh_identity = 1;
  p->phi_floor = 1;
}

int mhit_size_supported(int n) { return size_supported(n) ? 1 : 0; }

int mhit_check_bounded_wait(int arrive, long long limit_cycles, int* status_out) {
  if (!status_out || limit_cycles <= 0) return MHIT_ERR_INVALID;
  int* d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return MHIT_ERR_NOMEM;
  int rc = MHIT_OK;
  if (mhit::launch_wait_check(arrive, limit_cycles, d, 0) != cudaSuccess ||
      cudaMemcpy(status_out, d, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = MHIT_ERR_CUDA;
  cudaFree(d);
  return rc;
}

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
    case MHIT_ERR_SCRATCH_LIMIT: return "grid larger than the fixed scratch of the allocation-free entry point";
    case MHIT_ERR_TIMEOUT: return "a kernel's bounded wait for staged data gave up";
    default: return "unknown status";
  }
}

const char* mhit_last_error(mhit_handle* h) { return h ? h->last_error.c_str() : ""; }

int mhit_create(const mhit_params* p, int nx, int ny, int nz, int precision, int phase_field, mhit_handle** out) {
  if (!p || !out) return MHIT_ERR_INVALID;
  *out = nullptr;
  if (nx != ny || nx != nz) return MHIT_ERR_UNSUPPORTED;  // ny = nz = nx (multi/module.f90:2-3)
  if (!size_supported(nx)) return MHIT_ERR_UNSUPPORTED;
  if (precision != MHIT_FP64 && precision != MHIT_FP32_REFINE) return MHIT_ERR_UNSUPPORTED;
  // One FP32 correction solve converges only when the solve inverts the FD
  // Laplacian exactly, i.e. with the FD-modified k^2.
  if (precision == MHIT_FP32_REFINE && p->k2_mode != MHIT_K2_FD) return MHIT_ERR_UNSUPPORTED;
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
  c.phi_floor = p->phi_floor ? 1 : 0;
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
    const size_t pitch = mhit::spectrum_pitch(n, precision != MHIT_FP64);
    bool bad = false;
    if (precision == MHIT_FP64) {
      const size_t fb = N3 * sizeof(double);
      double** fields[] = {&h->u, &h->v, &h->w, &h->us, &h->vs, &h->ws, &h->ru, &h->rv, &h->rw, &h->p};
      for (double** f : fields) {
        if ((e = dalloc(h, f, fb))) { fail(e, "cudaMalloc field"); bad = true; break; }
      }
      if (bad) break;
      if (h->phase_field) {
        if ((e = dalloc(h, &h->phi[0], fb)) || (e = dalloc(h, &h->phi[1], fb))) { fail(e, "cudaMalloc phi"); break; }
      }
      const size_t sb = (size_t)n * n * pitch * sizeof(double2);
      if ((e = dalloc(h, &h->spec, sb))) { fail(e, "cudaMalloc spectrum"); break; }
      if ((e = cudaMemsetAsync(h->spec, 0, sb, h->st))) { fail(e, "memset"); break; }
    } else {
      const size_t fb = N3 * sizeof(float);
      float** fields[] = {&h->fu, &h->fv, &h->fw, &h->fus, &h->fvs, &h->fws, &h->fru, &h->frv, &h->frw,
                          &h->fp0, &h->fdp};
      for (float** f : fields) {
        if ((e = dalloc(h, f, fb))) { fail(e, "cudaMalloc field"); bad = true; break; }
      }
      if (bad) break;
      if (h->phase_field) {
        if ((e = dalloc(h, &h->fphi[0], fb)) || (e = dalloc(h, &h->fphi[1], fb))) { fail(e, "cudaMalloc phi"); break; }
      }
      const size_t sb = (size_t)n * n * pitch * sizeof(float2);
      if ((e = dalloc(h, &h->fspec, sb))) { fail(e, "cudaMalloc spectrum"); break; }
      if ((e = cudaMemsetAsync(h->fspec, 0, sb, h->st))) { fail(e, "memset"); break; }
      if ((e = cudaMemsetAsync(h->fp0, 0, fb, h->st)) || (e = cudaMemsetAsync(h->fdp, 0, fb, h->st))) {
        fail(e, "memset");
        break;
      }
    }
    h->nparts = mhit::fused_projection(n) ? mhit::xinv_project_partials(n) : mhit::project_partials(n);
    if ((e = dalloc(h, &h->partials, (size_t)mhit::partials_capacity(n) * 7 * sizeof(double)))) {
      fail(e, "cudaMalloc partials");
      break;
    }
    if ((e = dalloc(h, &h->ctrl, sizeof(Ctrl)))) { fail(e, "cudaMalloc ctrl"); break; }
    if ((e = dalloc(h, &h->div_out, sizeof(double)))) { fail(e, "cudaMalloc div"); break; }
    if ((e = dalloc(h, &h->stat_partials, (size_t)mhit::stats_partials(n) * 8 * sizeof(double))) ||
        (e = dalloc(h, &h->stat_out, 8 * sizeof(double))) || (e = cudaMallocHost(&h->h_stat, 8 * sizeof(double)))) {
      fail(e, "cudaMalloc stats");
      break;
    }
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
    std::vector<float2> twf(n);
    for (int m = 0; m < n; ++m) {
      long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
      twf[m].x = (float)cosl(a);
      twf[m].y = -(float)sinl(a);
    }
    if ((e = dalloc(h, &h->ftw, n * sizeof(float2))) ||
        (e = cudaMemcpyAsync(h->ftw, twf.data(), n * sizeof(float2), cudaMemcpyHostToDevice, h->st))) {
      fail(e, "twiddles");
      break;
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
  const size_t fb = (size_t)h->n * h->n * h->n * elem_size(h);
  CK(h, put_field(h, fu(h), u, layout));
  CK(h, put_field(h, fv(h), v, layout));
  CK(h, put_field(h, fw(h), w, layout));
  if (h->phase_field) CK(h, put_field(h, fphi(h, 0), phi, layout));
  // rhs_o starts at zero; beta = 0 on the first step (multi/main.f90:324)
  for (int q = 0; q < 3; ++q) CK(h, cudaMemsetAsync(frhs_o(h, q).ptr, 0, fb, h->st));
  if (f32(h)) {
    CK(h, cudaMemsetAsync(h->fp0, 0, fb, h->st));
    CK(h, cudaMemsetAsync(h->fdp, 0, fb, h->st));
  } else {
    CK(h, cudaMemsetAsync(h->p, 0, fb, h->st));
    h->p_in_spec = false;
  }
  h->dp_in_spec = false;
  h->have_step = false;
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
  CK(h, materialize(h));
  return MHIT_OK;
}

int mhit_get_fields(mhit_handle* h, double* u, double* v, double* w, double* phi, int layout) {
  if (!h || !layout_ok(layout)) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  CK(h, materialize(h));
  CK(h, pull_ctrl(h));
  const int cur = (int)(h->h_ctrl->nstep & 1);
  if (u) CK(h, get_field(h, u, fu(h), layout));
  if (v) CK(h, get_field(h, v, fv(h), layout));
  if (w) CK(h, get_field(h, w, fw(h), layout));
  if (phi && h->phase_field) CK(h, get_field(h, phi, fphi(h, cur), layout));
  CK(h, cudaStreamSynchronize(h->st));
  if (layout == MHIT_LAYOUT_PIX_HALO) {
    double* outs[4] = {u, v, w, h->phase_field ? phi : nullptr};
    for (double* o : outs)
      if (o) fill_halo_host(o, h->n);
  }
  return MHIT_OK;
}

// The FP32 form's pressure is p0 + dp, summed in FP64 on the host.
int mhit_get_pressure(mhit_handle* h, double* p, int layout) {
  if (!h || !p || !layout_ok(layout)) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  if (f32(h)) {
    CK(h, materialize_dp(h));
    const size_t N3 = (size_t)h->n * h->n * h->n;
    std::vector<double> a(N3), b(N3);
    CK(h, get_field(h, a.data(), DevField{h->fp0, true}, MHIT_LAYOUT_RAW));
    CK(h, get_field(h, b.data(), DevField{h->fdp, true}, MHIT_LAYOUT_RAW));
    for (size_t q = 0; q < N3; ++q) a[q] += b[q];
    const size_t plane = (size_t)h->n * h->n;
    for (int k = 0; k < h->n; ++k) {
      double* t = (layout == MHIT_LAYOUT_RAW) ? p + plane * k : p + (size_t)h->n * (1 + (size_t)(h->n + 2) * (k + 1));
      memcpy(t, a.data() + plane * k, plane * sizeof(double));
    }
  } else {
    if (h->p_in_spec) {  // the last step's pressure: x inverse of its spectrum
      mhit::PoissonArgs<double> pa;
      pa.spec = h->spec;
      pa.p = h->p;
      pa.tw = h->tw;
      pa.k2tab = h->k2tab;
      pa.ctrl = nullptr;
      CK(h, mhit::launch_poisson_stage<double>(h->n, pa, 4, h->st));
      h->p_in_spec = false;
    }
    CK(h, download(h, p, h->p, layout));
    CK(h, cudaStreamSynchronize(h->st));
  }
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
    h->p_in_spec = !f32(h) && mhit::fused_projection(h->n);
    h->dp_in_spec = refine_fused(h);
    h->have_step = true;
  }
  CK(h, pull_ctrl(h));
  h->nstep_host = h->h_ctrl->nstep;  // fewer if a step raised the error status
  fill_diag(h, out);
  if (out) CK(h, refine_max_div(h, &out->max_div));
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
    h->p_in_spec = !f32(h) && mhit::fused_projection(h->n);
    h->dp_in_spec = refine_fused(h);
    h->have_step = true;
  }
  return MHIT_OK;
}

int mhit_get_diag(mhit_handle* h, mhit_diag* out) {
  if (!h || !out) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  CK(h, pull_ctrl(h));
  h->nstep_host = h->h_ctrl->nstep;
  fill_diag(h, out);
  CK(h, refine_max_div(h, &out->max_div));
  return MHIT_OK;
}

int mhit_diagnostics(mhit_handle* h, int pi_f32, mhit_stats* out) {
  if (!h || !out) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  CK(h, pull_ctrl(h));
  const int n = h->n;
  const int cur = (int)(h->h_ctrl->nstep & 1);
  double dxi_d = h->c.dxi;
  if (pi_f32) {
    const double pi32 = (double)(float)3.14159265358979;  // post/compute_diss/module.f90:5
    dxi_d = 1.0 / ((2 * pi32) / (n - 1));
  }
  if (f32(h))
    CK(h, mhit::launch_stats<float>(h->fu, h->fv, h->fw, h->phase_field ? h->fphi[cur] : nullptr, h->ctrl, n,
                                    h->c.dxi, dxi_d, h->stat_partials, h->stat_out, h->st));
  else
    CK(h, mhit::launch_stats<double>(h->u, h->v, h->w, h->phase_field ? h->phi[cur] : nullptr, h->ctrl, n,
                                     h->c.dxi, dxi_d, h->stat_partials, h->stat_out, h->st));
  CK(h, cudaMemcpyAsync(h->h_stat, h->stat_out, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  const double nd = (double)n, n3 = nd * nd * nd;
  const double* r = h->h_stat;
  out->ke = 0.5 * r[0] / n3;
  out->dissipation = 2 * (h->prm.mu / h->prm.rho) * r[1] / nd / nd / nd;
  out->max_div = r[2];
  out->phi_sum = h->phase_field ? r[3] : 0.0;
  out->phi_min = h->phase_field ? r[4] : 0.0;
  out->phi_max = h->phase_field ? r[5] : 0.0;
  out->umean = r[6] / n3;
  out->reserved = 0;
  return MHIT_OK;
}

void* mhit_stream(mhit_handle* h) { return h ? (void*)h->st : nullptr; }

int mhit_device_state(mhit_handle* h, void** u, void** v, void** w, void** phi) {
  if (!h) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  if (u) *u = fu(h).ptr;
  if (v) *v = fv(h).ptr;
  if (w) *w = fw(h).ptr;
  if (phi) {
    CK(h, pull_ctrl(h));
    *phi = h->phase_field ? fphi(h, (int)(h->h_ctrl->nstep & 1)).ptr : nullptr;
  }
  return MHIT_OK;
}

// Drop count and sizes of the current phi (post/DropCountSize): components of
// phi >= 0.5, 26-connected with periodic wrap, in the reference's scan order.
int mhit_drop_count(mhit_handle* h, int capacity, int* ndrops, int64_t* cells, double* deq) {
  if (!h || !ndrops || capacity < 0 || (capacity > 0 && (!cells || !deq))) return MHIT_ERR_INVALID;
  if (!h->phase_field) return MHIT_ERR_STATE;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  const int n = h->n;
  const size_t N3 = (size_t)n * n * n;
  if (!h->ccl_lab) {
    h->ccl_cap = 1 << 20;
    CK(h, dalloc(h, &h->ccl_lab, N3 * sizeof(int)));
    CK(h, dalloc(h, &h->ccl_cnt, N3 * sizeof(int)));
    CK(h, dalloc(h, &h->ccl_roots, (size_t)h->ccl_cap * sizeof(int2)));
    CK(h, dalloc(h, &h->ccl_counter, 2 * sizeof(int)));
  }
  CK(h, pull_ctrl(h));
  const int cur = (int)(h->h_ctrl->nstep & 1);
  if (f32(h))
    CK(h, mhit::launch_dropcount<float>(h->fphi[cur], n, h->ccl_lab, h->ccl_cnt, h->ccl_roots, h->ccl_cap,
                                        h->ccl_counter, h->st));
  else
    CK(h, mhit::launch_dropcount<double>(h->phi[cur], n, h->ccl_lab, h->ccl_cnt, h->ccl_roots, h->ccl_cap,
                                         h->ccl_counter, h->st));
  int cnt[2] = {0, 0};
  CK(h, cudaMemcpyAsync(cnt, h->ccl_counter, sizeof(cnt), cudaMemcpyDeviceToHost, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  if (cnt[1]) return MHIT_ERR_CUDA;
  if (cnt[0] > h->ccl_cap) return MHIT_ERR_UNSUPPORTED;  // more components than the root list holds
  std::vector<int2> roots(cnt[0]);
  if (cnt[0] > 0)
    CK(h, cudaMemcpy(roots.data(), h->ccl_roots, cnt[0] * sizeof(int2), cudaMemcpyDeviceToHost));
  std::sort(roots.begin(), roots.end(), [](const int2& a, const int2& b) { return a.x < b.x; });
  const double pi = 4.0 * atan(1.0), n6opi = 6.0 / pi;  // post/DropCountSize/module.f90:3-5
  const double dx = 1.0 / h->c.dxi;
  for (int q = 0; q < cnt[0] && q < capacity; ++q) {
    cells[q] = roots[q].y;
    deq[q] = dx * pow(n6opi * (double)roots[q].y, 1.0 / 3.0);  // calculate_deq.f90:33
  }
  *ndrops = cnt[0];
  return MHIT_OK;
}

// Tile shapes of the stencil kernels: z chunk kz (a divisor of n, 0 =
// default 32) and momentum tile height mty (8 or 16, 0 = default for n).
// Results do not depend on them; the step graphs are re-captured.
int mhit_set_tiles(mhit_handle* h, int kz, int mty) {
  if (!h) return MHIT_ERR_INVALID;
  if (kz != 0 && !mhit::stencil_kz_ok(h->n, kz)) return MHIT_ERR_INVALID;
  if (mty != 0 && mty != 8 && mty != 16) return MHIT_ERR_INVALID;
  DeviceGuard g(h->device);
  CK(h, cudaStreamSynchronize(h->st));
  for (int i = 0; i < 2; ++i)
    if (h->graph[i]) {
      cudaGraphExecDestroy(h->graph[i]);
      h->graph[i] = nullptr;
    }
  h->kz = kz;
  h->mty = mty;
  return MHIT_OK;
}

int mhit_memory_bytes(mhit_handle* h, size_t* bytes) {
  if (!h || !bytes) return MHIT_ERR_INVALID;
  *bytes = h->bytes;
  return MHIT_OK;
}

int mhit_launches_per_step(mhit_handle* h, int* n) {
  if (!h || !n) return MHIT_ERR_INVALID;
  *n = (int)step_stages(h, 0).size();
  return MHIT_OK;
}

// Run `reps` steps with every kernel launched on its own between CUDA events
// on the handle's stream; ms[k] = mean duration of stage k (names from
// mhit_stage_name, in launch order).
int mhit_profile_step(mhit_handle* h, int reps, double* ms, int* nstages) {
  if (!h || !ms || !nstages || reps < 1) return MHIT_ERR_INVALID;
  if (!h->has_fields) return MHIT_ERR_STATE;
  DeviceGuard g(h->device);
  const int NS = (int)step_stages(h, 0).size();
  std::vector<cudaEvent_t> ev(NS + 1);
  for (int i = 0; i <= NS; ++i) CK(h, cudaEventCreate(&ev[i]));
  std::vector<double> acc(NS, 0.0);
  for (int r = 0; r < reps; ++r) {
    const int cur = (int)(h->nstep_host & 1);
    std::vector<Stage> stages = step_stages(h, cur);
    CK(h, cudaEventRecord(ev[0], h->st));
    for (int i = 0; i < NS; ++i) {
      CK(h, stages[i].second());
      CK(h, cudaEventRecord(ev[i + 1], h->st));
    }
    CK(h, cudaEventSynchronize(ev[NS]));
    h->p_in_spec = !f32(h) && mhit::fused_projection(h->n);
    h->dp_in_spec = refine_fused(h);
    h->have_step = true;
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

const char* mhit_stage_name(mhit_handle* h, int k) {
  if (!h) return "";
  std::vector<Stage> st = step_stages(h, 0);
  return (k >= 0 && k < (int)st.size()) ? st[k].first : "";
}

int mhit_poisson_device(mhit_handle* h, const double* rhs_dev, double* p_dev) {
  if (!h || !rhs_dev || !p_dev) return MHIT_ERR_INVALID;
  if (f32(h)) return MHIT_ERR_UNSUPPORTED;  // the FP64 stand-alone solve needs the FP64 spectrum
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
  pa.ddxi = h->c.ddxi;
  if (h->p_in_spec) {
    // keep the last step's pressure: recompute it before the spectrum is
    // reused, unless the caller's buffers are the pressure buffer itself
    if (rhs_dev != h->p && p_dev != h->p) {
      mhit::PoissonArgs<double> px = pa;
      px.p = h->p;
      CK(h, mhit::launch_poisson_stage<double>(h->n, px, 4, h->st));
    }
    h->p_in_spec = false;
  }
  CK(h, mhit::launch_poisson<double>(h->n, pa, h->st));
  return MHIT_OK;
}

int mhit_poisson(mhit_handle* h, const double* rhs, double* p) {
  if (!h || !rhs || !p) return MHIT_ERR_INVALID;
  if (f32(h)) return MHIT_ERR_UNSUPPORTED;
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
  DevField dev[3] = {fu(h), fv(h), fw(h)};
  DeviceGuard g(h->device);
  CK(h, materialize(h));
  CK(h, pull_ctrl(h));
  for (int q = 0; q < 3; ++q) {
    CK(h, get_field(h, host, dev[q], MHIT_LAYOUT_RAW));
    CK(h, cudaStreamSynchronize(h->st));
    if ((rc = write_raw(fname(dir, names[q], t), host, N3))) return rc;
  }
  if (h->phase_field) {
    CK(h, get_field(h, host, fphi(h, (int)(h->h_ctrl->nstep & 1)), MHIT_LAYOUT_RAW));
    CK(h, cudaStreamSynchronize(h->st));
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
  for (int q = 0; q < 3 && ok; ++q) {
    if (get_field(h, host, frhs_o(h, q), MHIT_LAYOUT_RAW) != cudaSuccess ||
        cudaStreamSynchronize(h->st) != cudaSuccess)
      ok = false;
    else
      ok = fwrite(host, sizeof(double), N3, f) == N3;
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
  DeviceGuard g(h->device);
  for (int q = 0; q < 3 && ok; ++q) {
    ok = fread(bu.data(), sizeof(double), N3, f) == N3;
    if (ok) ok = put_field(h, frhs_o(h, q), bu.data(), MHIT_LAYOUT_RAW) == cudaSuccess;
  }
  fclose(f);
  if (!ok) return MHIT_ERR_IO;
  CK(h, cudaStreamSynchronize(h->st));
  // phi was uploaded into slot 0; keep the parity convention phi[nstep & 1]
  if (h->phase_field && (sc.nstep & 1))
    CK(h, cudaMemcpyAsync(fphi(h, 1).ptr, fphi(h, 0).ptr, N3 * elem_size(h), cudaMemcpyDeviceToDevice, h->st));
  Ctrl* c = h->h_ctrl;
  c->gumax = sc.gumax;
  c->alpha = sc.alpha;
  c->beta = sc.beta;
  c->cfl = sc.cfl;
  c->nstep = sc.nstep;
  CK(h, cudaMemcpyAsync(h->ctrl, c, sizeof(Ctrl), cudaMemcpyHostToDevice, h->st));
  CK(h, cudaStreamSynchronize(h->st));
  h->nstep_host = sc.nstep;
  h->have_step = false;
  return MHIT_OK;
}

}  // extern "C"
