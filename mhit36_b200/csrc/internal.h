// Internal launcher interface between the C ABI (capi.cu) and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include "common.cuh"

// Grid sizes with built kernels (N^3 cells, N a multiple of 32 with radices 2/3).
#define MHIT_FOR_SIZES(X) X(32) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

namespace mhit {

template <class T> struct PoissonArgs {
  const T* us;  // divergence inputs (ustar, vstar, wstar) or nullptr
  const T* vs;
  const T* ws;
  const T* rhs;  // explicit RHS (stand-alone solve) or nullptr
  typename C2<T>::t* spec;
  T* p;
  const typename C2<T>::t* tw;
  const double* k2tab;
  const Ctrl* ctrl;
  T cdiv;
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
  const T* p;
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
cudaError_t launch_finalize(const double* partials, int nparts, Ctrl* ctrl, StepConst c, cudaStream_t st);
template <class T> cudaError_t launch_materialize(T* u, T* v, T* w, int n, Ctrl* ctrl, cudaStream_t st);
cudaError_t prepare_stencils();
int project_partials(int n);
int stencil_size_ok(int n);

}  // namespace mhit
