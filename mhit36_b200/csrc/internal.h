// Internal launcher interface between the C ABI (capi.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "common.cuh"

// Grid sizes with built kernels (N^3 cells, N a multiple of 32 with radices 2/3).
#define MHIT_FOR_SIZES(X) X(32) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

namespace mhit {

template <class T> struct PoissonArgs {
  const T* us = nullptr;  // divergence inputs (ustar, vstar, wstar) or nullptr
  const T* vs = nullptr;
  const T* ws = nullptr;
  const T* rhs = nullptr;  // explicit RHS (stand-alone solve) or nullptr
  typename C2<T>::t* spec = nullptr;
  T* p = nullptr;
  const typename C2<T>::t* tw = nullptr;
  const double* k2tab = nullptr;
  const Ctrl* ctrl = nullptr;
  double cdiv = 0;         // rho*dxi/dt
  const T* pres = nullptr;  // refinement: first-solve pressure p0 (residual RHS) or nullptr
  double ddxi = 0;         // 1/dx^2 for the residual Laplacian
};

template <class T> cudaError_t launch_poisson(int n, const PoissonArgs<T>& a, cudaStream_t st);
// One of the five Poisson kernels (0 xfwd, 1 yfwd, 2 zsolve, 3 yinv, 4 xinv).
template <class T> cudaError_t launch_poisson_stage(int n, const PoissonArgs<T>& a, int stage, cudaStream_t st);
cudaError_t prepare_poisson(int n);
size_t spectrum_pitch(int n);

template <class T> struct StencilArgs {
  const T* u;
  const T* v;
  const T* w;
  const T* phi_in;
  T* phi_out;
  T* us;
  T* vs;
  T* ws;
  T* ru;
  T* rv;
  T* rw;
  const T* p;  // pressure (FP64 form) or first-solve p0 (FP32 refine)
  T* uo;
  T* vo;
  T* wo;
  double* partials;
  const double* fsin;  // sin(k0*x(g)), g = 0..N-1
  const double* fcos;  // cos(k0*x(g))
  Ctrl* ctrl;
  StepConst c;
};

template <class T> cudaError_t launch_phase(const StencilArgs<T>& a, cudaStream_t st);
template <class T> cudaError_t launch_momentum(const StencilArgs<T>& a, bool phase_field, cudaStream_t st);
template <class T> cudaError_t launch_project(const StencilArgs<T>& a, cudaStream_t st);
// FP32 refinement form: p = p0 + dp, projection and max|div u| in FP64.
cudaError_t launch_project_refine(const StencilArgs<float>& a, const float* dp, cudaStream_t st);
int project_refine_partials(int n);
cudaError_t launch_finalize(const double* partials, int nparts, int stride, Ctrl* ctrl, StepConst c,
                            cudaStream_t st);
template <class T> cudaError_t launch_materialize(T* u, T* v, T* w, int n, Ctrl* ctrl, cudaStream_t st);
cudaError_t prepare_stencils();
int project_partials(int n);
int stencil_size_ok(int n);

template <class T>
cudaError_t launch_stats(const T* u, const T* v, const T* w, const T* phi, const Ctrl* ctrl, int n, double dxi_c,
                         double dxi_d, double* partials, double* out, cudaStream_t st);
int stats_partials(int n);

}  // namespace mhit
