// FFT Poisson solve of the MHIT36 step on one B200 (replaces
// multi/main.f90:715-850: divergence, rhsp -> rhsp_complex, cuFFT Z2Z along
// x/y/z with cuDecomp transposes, -1/k^2/(nx*ny*nz), inverse, real part).
//
// Design:
//   * The pressure RHS is real, so the x transform is real-to-complex: two
//     real lines (y = j, j+1) are packed as one complex line, transformed,
//     and split by Hermitian symmetry into two half spectra of N/2+1 modes.
//     The reference transforms the full complex field (2x the work).
//   * Spectrum layout in HBM: spec[kz][ky][kx], kx fastest, row pitch PITCH
//     complex (N/2+1 rounded up to the column chunk CC), so a chunk of CC
//     kx columns is one 128-byte row segment.  The y and z passes stage a
//     CC x N slab in shared memory, transform along the slow axis there, and
//     write it back in place: no transposes in HBM at all (the reference does
//     four cuDecomp transposes per solve, multi/main.f90:754-810).
//   * The z pass fuses forward FFT, the k^2 division and the inverse FFT.
//   * The inverse x pass is complex-to-real for two lines at once.
#include <cuda_runtime.h>
#include "common.cuh"
#include "fft.cuh"
#include "internal.h"

namespace mhit {

template <int N> struct PCfg {
  // Lines per CTA: 2048/N (at most 8), so that the first radix-8 stage gives
  // every one of the 256 threads exactly one butterfly (registers stay under
  // the 85 that three resident CTAs per SM allow).
  static constexpr int L = (N <= 256) ? 8 : ((N <= 512) ? 4 : 2);
  static constexpr int P = L;   // line pairs per CTA (x passes)
  static constexpr int CC = L;  // kx columns per CTA (y/z passes)
  static constexpr int NT = 256;
  static constexpr int PITCH = ((N / 2 + 1) + CC - 1) / CC * CC;
  static constexpr int NCHUNK = PITCH / CC;
};

// ---------------------------------------------------------------- x forward
// MODE 0: rhs = (rho*dxi/dt) * forward-difference divergence of (us,vs,ws)
// (multi/main.f90:715-729), evaluated in FP64.
// MODE 1: rhs read from `rhs` (stand-alone solve).
// MODE 2: refinement residual r - L(p0) in FP64, r as in MODE 0 and L the
// 7-point Laplacian (the operator whose symbol the FD-modified k^2 inverts).
template <int N, int MODE, class T>
__device__ __forceinline__ double xfwd_rhs(const T* __restrict__ us, const T* __restrict__ vs,
                                          const T* __restrict__ ws, const T* __restrict__ rhs,
                                          const T* __restrict__ p0, double cdiv, double ddxi, int n, int j,
                                          int k) {
  const size_t a = gidx(n, j, k, N);
  if (MODE == 1) return (double)rhs[a];
  const int ip = (n + 1 == N) ? 0 : n + 1;
  const int jp = (j + 1 == N) ? 0 : j + 1;
  const int kp = (k + 1 == N) ? 0 : k + 1;
  double r = cdiv * ((double)us[gidx(ip, j, k, N)] - (double)us[a]);
  r = r + cdiv * ((double)vs[gidx(n, jp, k, N)] - (double)vs[a]);
  r = r + cdiv * ((double)ws[gidx(n, j, kp, N)] - (double)ws[a]);
  if (MODE == 2) {
    const int im = n ? n - 1 : N - 1, jm = j ? j - 1 : N - 1, km = k ? k - 1 : N - 1;
    const double c = (double)p0[a];
    const double lap = ((double)p0[gidx(ip, j, k, N)] - 2.0 * c + (double)p0[gidx(im, j, k, N)]) * ddxi +
                       ((double)p0[gidx(n, jp, k, N)] - 2.0 * c + (double)p0[gidx(n, jm, k, N)]) * ddxi +
                       ((double)p0[gidx(n, j, kp, N)] - 2.0 * c + (double)p0[gidx(n, j, km, N)]) * ddxi;
    r = r - lap;
  }
  return r;
}

template <int N, int MODE, class T>
__global__ void __launch_bounds__(256, 3) xfwd_kernel(const T* __restrict__ us, const T* __restrict__ vs,
                                                  const T* __restrict__ ws, const T* __restrict__ rhs,
                                                  const T* __restrict__ p0,
                                                  typename C2<T>::t* __restrict__ spec,
                                                  const typename C2<T>::t* __restrict__ tw,
                                                  const Ctrl* __restrict__ ctrl, double cdiv, double ddxi) {
  typedef typename C2<T>::t C;
  typedef PCfg<N> G;
  constexpr int P = G::P, NT = G::NT;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int j0 = blockIdx.x * (2 * P);
  const int k = blockIdx.y;
  for (int wi = threadIdx.x; wi < P * N; wi += NT) {
    const int p = wi % P, n = wi / P;
    const int ja = j0 + 2 * p;
    C z;
    z.x = (T)xfwd_rhs<N, MODE, T>(us, vs, ws, rhs, p0, cdiv, ddxi, n, ja, k);
    z.y = (T)xfwd_rhs<N, MODE, T>(us, vs, ws, rhs, p0, cdiv, ddxi, n, ja + 1, k);
    s[n * P + p] = z;
  }
  __syncthreads();
  smem_fft<N, P, NT, -1>(s, tw);
  const T half = (T)0.5;
  for (int wi = threadIdx.x; wi < P * (N / 2 + 1); wi += NT) {
    const int p = wi % P, m = wi / P;
    const int ja = j0 + 2 * p;
    const C zm = s[m * P + p];
    const C zr = s[((m == 0) ? 0 : (N - m)) * P + p];
    C A, B;
    A.x = half * (zm.x + zr.x);
    A.y = half * (zm.y - zr.y);
    B.x = half * (zm.y + zr.y);
    B.y = -half * (zm.x - zr.x);
    C* row = spec + ((size_t)k * N + ja) * G::PITCH;
    row[m] = A;
    row[G::PITCH + m] = B;
  }
}

// ---------------------------------------------------------------- y pass
template <int N, int DIR, class T>
__global__ void __launch_bounds__(256, 3) ypass_kernel(typename C2<T>::t* __restrict__ spec,
                                                   const typename C2<T>::t* __restrict__ tw,
                                                   const Ctrl* __restrict__ ctrl) {
  typedef typename C2<T>::t C;
  typedef PCfg<N> G;
  constexpr int CC = G::CC, NT = G::NT;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  C* base = spec + (size_t)blockIdx.y * N * G::PITCH + blockIdx.x * CC;
  for (int wi = threadIdx.x; wi < CC * N; wi += NT) {
    const int l = wi % CC, n = wi / CC;
    s[wi] = base[(size_t)n * G::PITCH + l];
  }
  __syncthreads();
  smem_fft<N, CC, NT, DIR>(s, tw);
  for (int wi = threadIdx.x; wi < CC * N; wi += NT) {
    const int l = wi % CC, n = wi / CC;
    base[(size_t)n * G::PITCH + l] = s[wi];
  }
}

// ---------------------------------------------------------------- z pass
// Forward z FFT, psi = -psi/k2/(nx*ny*nz) with psi(0,0,0) = 0
// (multi/main.f90:785-798), inverse z FFT, all in shared memory.
// k2tab[m] holds kx(m)^2 (spectral) or (4/dx^2) sin^2(pi m/N) (FD-modified).
template <int N, class T>
__global__ void __launch_bounds__(256, 3) zsolve_kernel(typename C2<T>::t* __restrict__ spec,
                                                    const typename C2<T>::t* __restrict__ tw,
                                                    const double* __restrict__ k2tab,
                                                    const Ctrl* __restrict__ ctrl) {
  typedef typename C2<T>::t C;
  typedef PCfg<N> G;
  constexpr int CC = G::CC, NT = G::NT;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int jy = blockIdx.y;
  const int m0 = blockIdx.x * CC;
  C* base = spec + (size_t)jy * G::PITCH + m0;
  const size_t zstride = (size_t)N * G::PITCH;
  for (int wi = threadIdx.x; wi < CC * N; wi += NT) {
    const int l = wi % CC, n = wi / CC;
    s[wi] = base[(size_t)n * zstride + l];
  }
  __syncthreads();
  smem_fft<N, CC, NT, -1>(s, tw);
  const double nnn = (double)((long long)N * (long long)N * (long long)N);
  const double k2y = k2tab[jy];
  for (int wi = threadIdx.x; wi < CC * N; wi += NT) {
    const int l = wi % CC, n = wi / CC;
    const int m = m0 + l;
    C v = s[wi];
    if (m > N / 2 || (m == 0 && jy == 0 && n == 0)) {
      v.x = 0;
      v.y = 0;
    } else {
      const double k2 = (k2tab[m] + k2y) + k2tab[n];
      v.x = (T)(-(double)v.x / k2 / nnn);
      v.y = (T)(-(double)v.y / k2 / nnn);
    }
    s[wi] = v;
  }
  __syncthreads();
  smem_fft<N, CC, NT, +1>(s, tw);
  for (int wi = threadIdx.x; wi < CC * N; wi += NT) {
    const int l = wi % CC, n = wi / CC;
    base[(size_t)n * zstride + l] = s[wi];
  }
}

// ---------------------------------------------------------------- x inverse
// Complex-to-real x transform of two lines at once; writes p
// (multi/main.f90:812, 842-850: p = real(psi)).
template <int N, class T>
__global__ void __launch_bounds__(256, 3) xinv_kernel(const typename C2<T>::t* __restrict__ spec, T* __restrict__ p,
                                                  const typename C2<T>::t* __restrict__ tw,
                                                  const Ctrl* __restrict__ ctrl) {
  typedef typename C2<T>::t C;
  typedef PCfg<N> G;
  constexpr int P = G::P, NT = G::NT;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int j0 = blockIdx.x * (2 * P);
  const int k = blockIdx.y;
  for (int wi = threadIdx.x; wi < P * (N / 2 + 1); wi += NT) {
    const int q = wi % P, m = wi / P;
    const C* row = spec + ((size_t)k * N + j0 + 2 * q) * G::PITCH;
    C A = row[m];
    C B = row[G::PITCH + m];
    if (m == 0 || m == N / 2) {
      A.y = 0;
      B.y = 0;
    }
    C z;
    z.x = A.x - B.y;
    z.y = A.y + B.x;
    s[m * P + q] = z;
    if (m > 0 && m < N / 2) {
      C zc;
      zc.x = A.x + B.y;
      zc.y = B.x - A.y;
      s[(N - m) * P + q] = zc;
    }
  }
  __syncthreads();
  smem_fft<N, P, NT, +1>(s, tw);
  for (int wi = threadIdx.x; wi < P * N; wi += NT) {
    const int q = wi % P, n = wi / P;
    const int ja = j0 + 2 * q;
    const C z = s[n * P + q];
    p[gidx(n, ja, k, N)] = z.x;
    p[gidx(n, ja + 1, k, N)] = z.y;
  }
}

// ---------------------------------------------------------------- launchers
template <int N, class T> static size_t xsmem() { return (size_t)N * PCfg<N>::P * sizeof(typename C2<T>::t); }
template <int N, class T> static size_t csmem() { return (size_t)N * PCfg<N>::CC * sizeof(typename C2<T>::t); }

template <int N, class T> static cudaError_t set_attrs() {
  cudaError_t e;
  const int xs = (int)xsmem<N, T>(), cs = (int)csmem<N, T>();
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 0, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 2, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xinv_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(ypass_kernel<N, -1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs))) return e;
  if ((e = cudaFuncSetAttribute(ypass_kernel<N, 1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs))) return e;
  if ((e = cudaFuncSetAttribute(zsolve_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, cs))) return e;
  return cudaSuccess;
}

template <int N, class T>
static void launch_xfwd(const PoissonArgs<T>& a, cudaStream_t st) {
  typedef PCfg<N> G;
  const dim3 gx(N / (2 * G::P), N);
  const size_t xs = xsmem<N, T>();
  if (a.rhs)
    xfwd_kernel<N, 1, T><<<gx, G::NT, xs, st>>>(nullptr, nullptr, nullptr, a.rhs, nullptr, a.spec, a.tw, a.ctrl,
                                                a.cdiv, a.ddxi);
  else if (a.pres)
    xfwd_kernel<N, 2, T><<<gx, G::NT, xs, st>>>(a.us, a.vs, a.ws, nullptr, a.pres, a.spec, a.tw, a.ctrl, a.cdiv,
                                                a.ddxi);
  else
    xfwd_kernel<N, 0, T><<<gx, G::NT, xs, st>>>(a.us, a.vs, a.ws, nullptr, nullptr, a.spec, a.tw, a.ctrl, a.cdiv,
                                                a.ddxi);
}

template <int N, class T>
static cudaError_t poisson_run(const PoissonArgs<T>& a, cudaStream_t st) {
  typedef PCfg<N> G;
  const dim3 gx(N / (2 * G::P), N), gc(G::NCHUNK, N);
  const size_t xs = xsmem<N, T>(), cs = csmem<N, T>();
  launch_xfwd<N, T>(a, st);
  ypass_kernel<N, -1, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.ctrl);
  zsolve_kernel<N, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.k2tab, a.ctrl);
  ypass_kernel<N, 1, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.ctrl);
  xinv_kernel<N, T><<<gx, G::NT, xs, st>>>(a.spec, a.p, a.tw, a.ctrl);
  return cudaGetLastError();
}

template <int N, class T>
static cudaError_t poisson_stage(const PoissonArgs<T>& a, int stage, cudaStream_t st) {
  typedef PCfg<N> G;
  const dim3 gx(N / (2 * G::P), N), gc(G::NCHUNK, N);
  const size_t xs = xsmem<N, T>(), cs = csmem<N, T>();
  switch (stage) {
    case 0: launch_xfwd<N, T>(a, st); break;
    case 1: ypass_kernel<N, -1, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.ctrl); break;
    case 2: zsolve_kernel<N, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.k2tab, a.ctrl); break;
    case 3: ypass_kernel<N, 1, T><<<gc, G::NT, cs, st>>>(a.spec, a.tw, a.ctrl); break;
    case 4: xinv_kernel<N, T><<<gx, G::NT, xs, st>>>(a.spec, a.p, a.tw, a.ctrl); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_poisson_stage(int n, const PoissonArgs<T>& a, int stage, cudaStream_t st) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return poisson_stage<NN, T>(a, stage, st);
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_poisson_stage<double>(int, const PoissonArgs<double>&, int, cudaStream_t);
template cudaError_t launch_poisson_stage<float>(int, const PoissonArgs<float>&, int, cudaStream_t);

// Opt the kernels of size n into their dynamic shared memory (once per
// device and size; must precede graph capture).
cudaError_t prepare_poisson(int n) {
  switch (n) {
#define MHIT_CASE(NN)                                   \
  case NN: {                                            \
    cudaError_t e = set_attrs<NN, double>();            \
    return e ? e : set_attrs<NN, float>();              \
  }
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

template <class T>
cudaError_t launch_poisson(int n, const PoissonArgs<T>& a, cudaStream_t st) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return poisson_run<NN, T>(a, st);
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

size_t spectrum_pitch(int n) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return PCfg<NN>::PITCH;
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return 0;
  }
}

template cudaError_t launch_poisson<double>(int, const PoissonArgs<double>&, cudaStream_t);
template cudaError_t launch_poisson<float>(int, const PoissonArgs<float>&, cudaStream_t);

}  // namespace mhit
