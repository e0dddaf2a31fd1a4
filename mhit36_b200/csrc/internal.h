// Internal launcher interface between the C ABI (capi.cu) and the kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
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
// Row pitch (complex elements) of the half spectrum of the FP64 (fp32 = 0) or FP32 form.
size_t spectrum_pitch(int n, int fp32);

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

// Tensor maps of the momentum kernel's staged fields (2D views of an n^3
// field: x by y*z rows).
struct PlaneMaps {
  CUtensorMap u, v, w, phi;
};
// Tensor maps of a served-ensemble slot, kept in its device table entry:
// the momentum kernel's boxes per tile height (8, 16) and phi parity, the
// phase kernel's phi box per parity, and the column passes' spectrum views
// (y passes, z solve).  Written by a kernel, so readers acquire them through
// the tensor-map proxy before use.
struct SlotMaps {
  PlaneMaps mom[2][2];
  CUtensorMap phase_phi[2];
  CUtensorMap col_y, col_z;
};

// One resident simulation of a served ensemble: the batched kernels read
// their arguments from a device array of these, one per slot of a class.
template <class T> struct SlotArgs {
  StencilArgs<T> st;    // phi_in / phi_out are chosen on the device by step parity
  PoissonArgs<T> po;    // the Poisson solve (FP32 form: first solve -> p0)
  PoissonArgs<T> pr;    // FP32 form: correction solve of the FP64 residual -> dp
  T* phi[2];
  float* dp;            // FP32 form: correction pressure
  int active;           // 0: every kernel of this slot returns at once
  int pad_;
  SlotMaps maps;        // tensor maps of this slot's fields (encoded on the host)
};

// Batched launches over `nslots` slots of one class (grid size n).  kz is
// the stencil kernels' z chunk (chosen by the autotuner).
template <class T> cudaError_t launch_phase_batched(const SlotArgs<T>* slots, int nslots, int n, int kz, cudaStream_t st);
template <class T>
cudaError_t launch_momentum_batched(const SlotArgs<T>* slots, int nslots, int n, int kz, bool pf, cudaStream_t st,
                                   int mty);
template <class T> cudaError_t launch_project_batched(const SlotArgs<T>* slots, int nslots, int n, cudaStream_t st);
cudaError_t launch_finalize_batched(const SlotArgs<double>* slots, int nslots, int n, cudaStream_t st);
cudaError_t launch_finalize_batched_f32(const SlotArgs<float>* slots, int nslots, int n, cudaStream_t st);
// Poisson stage (0..4) for every slot; `which` 0 = po, 1 = pr.
template <class T>
cudaError_t launch_poisson_stage_batched(const SlotArgs<T>* slots, int nslots, int n, int stage, int which,
                                         cudaStream_t st);
int stencil_kz_ok(int n, int kz);

// kz: z chunk of the stencil kernels (0 = default); mty: momentum tile height (8 or 16).
template <class T> cudaError_t launch_phase(const StencilArgs<T>& a, cudaStream_t st, int kz);
template <class T>
cudaError_t launch_momentum(const StencilArgs<T>& a, bool phase_field, cudaStream_t st, int kz, int mty);
int default_mty(int n, int fp32);
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
// The x inverse fused into the projection (power-of-two n >= 256): one
// kernel after the y inverse pass, writing its own partials (stride 6).
// FP64 step: pa is the solve; FP32 refinement form: pa is the correction
// solve, whose x inverse dp is added to the stored p0 (a.p).
int fused_projection(int n);
int xinv_project_partials(int n);
template <class T>
cudaError_t launch_xinv_project(int n, const PoissonArgs<T>& pa, const StencilArgs<T>& a, cudaStream_t st);
template <class T>
cudaError_t launch_xinv_project_batched(const SlotArgs<T>* slots, int nslots, int n, cudaStream_t st);
// FP32 refinement form: max |div u| of the FP64 projection u = ustar -
// dt/rho*grad(p0 + dp) from the stored ustar, p0 and dp, into *out (one
// double on the device; the forward-difference divergence of
// multi/main.f90:723-725).
// Tensor map of 8-byte elements (tiled, no swizzle): dims innermost first,
// strides[rank-1] in bytes, box per dim.
cudaError_t encode_tensor_map(CUtensorMap* m, int rank, const void* base, const uint64_t* dims,
                              const uint64_t* strides, const uint32_t* box, int elem_bytes = 8);
// A slot's tensor maps from its table entry's field pointers (n^3 grid).
template <class T> cudaError_t encode_slot_maps(SlotArgs<T>* a, int n, bool phase_field);
// The column passes' spectrum views of a slot (part of encode_slot_maps).
template <class T> cudaError_t encode_column_maps(SlotMaps* m, const void* spec, int n);
// One-warp self-check of the bounded barrier wait (writes 0 or MHIT_ERR_TIMEOUT).
cudaError_t launch_wait_check(int arrive, long long limit_cycles, int* out_dev, cudaStream_t st);
cudaError_t launch_refine_divergence(const StencilArgs<float>& a, const float* dp, double* out, cudaStream_t st);
// Partials the FP64 step's projection writes, and the buffer size that
// holds either projection's partials (stride 7).
inline int step_partials_fp64(int n) { return fused_projection(n) ? xinv_project_partials(n) : project_partials(n); }
inline int partials_capacity(int n) {
  return project_partials(n) > xinv_project_partials(n) ? project_partials(n) : xinv_project_partials(n);
}

template <class T>
cudaError_t launch_stats(const T* u, const T* v, const T* w, const T* phi, const Ctrl* ctrl, int n, double dxi_c,
                         double dxi_d, double* partials, double* out, cudaStream_t st);
int stats_partials(int n);

template <class T>
cudaError_t launch_dropcount(const T* phi, int n, int* lab, int* cnt, int2* roots, int cap, int* d_counter,
                             cudaStream_t st);

}  // namespace mhit
