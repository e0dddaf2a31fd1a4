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
//     kx columns is one 32-128-byte row segment.  The y and z passes hold a
//     CC x N slab of columns in registers (register-resident lines, fft.cuh),
//     transform along the slow axis and write it back in place: no
//     transposes in HBM at all (the reference does four cuDecomp transposes
//     per solve, multi/main.f90:754-810).
//   * The z pass fuses forward FFT, the k^2 division and the inverse FFT.
//   * The inverse x pass is complex-to-real for two lines at once.
#include <cuda_runtime.h>
#include <algorithm>
#include "common.cuh"
#include "fft.cuh"
#include <string.h>
#include "internal.h"

namespace mhit {

template <int N, class T = double> struct PCfg {
  // Lines per CTA: 2048/N (at most 8), so that the first radix-8 stage gives
  // every one of the 256 threads exactly one butterfly (registers stay under
  // the 85 that three resident CTAs per SM allow).  The FP32 column passes
  // take twice as many kx columns (two butterflies per thread), so that a
  // chunk is still a 64-128-byte row segment of the half spectrum (measured
  // 20-25% faster on B200 at 512^3; the x passes are faster with 2048/N).
  static constexpr int L = (N <= 256) ? 8 : ((N <= 512) ? 4 : 2);
  static constexpr int P = L;                               // line pairs per CTA (x passes)
  static constexpr int CC = (sizeof(T) == 8) ? L : 2 * L;   // kx columns per CTA (y/z passes)
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

// ---------------------------------------------------------------- column slabs
// The y passes and the z solve walk (column chunk, line) slabs of the half
// spectrum.  KIND 0/1: y pass forward/inverse; KIND 2: z solve.
struct ColSlab {
  void* spec;        // slab base (the chunk's first element)
  size_t stride;     // distance between consecutive elements of a column (complex)
  const void* tw;
  const double* k2tab;
  int jy;            // z solve: the ky index of the slab
  int m0;            // z solve: first kx of the chunk
  int chunk, line;   // the slab's column chunk and line (y pass: kz; z solve: ky)
  bool live;         // false: skip (inactive slot or stopped simulation)
  bool gmap;         // map lives in an ensemble slot table (acquire it first)
  const CUtensorMap* map;  // the spectrum view the prefetch boxes come from
  Ctrl* ctrl;        // where a prefetch wait that gives up records the timeout
};

// The z solve's per-mode factor -1/(k^2 nx ny nz) (multi/main.f90:792), for
// d = k^2 nx ny nz > 0.  FP64: the quotient by Newton-Raphson from the PTX
// reciprocal approximation (rcp.approx.ftz.f64, two iterations and a
// remainder correction; branch-free, unlike the IEEE division with its
// special-case path), applied in FP64.  FP32 solves (the refinement form):
// the single-precision reciprocal, whose relative error (about 1e-7) is of
// the order of the FP32 transform's own rounding, which the FP64 residual
// and correction solve remove.
template <class T> __device__ __forceinline__ T scale_factor(double d);
template <> __device__ __forceinline__ double scale_factor<double>(double d) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
  double e = fma(-d, y, 1.0);
  y = fma(y, e, y);
  e = fma(-d, y, 1.0);
  y = fma(y, e, y);
  return -fma(fma(-d, y, 1.0), y, y);
}
template <> __device__ __forceinline__ float scale_factor<float>(double d) { return -__frcp_rn((float)d); }

// Slab `it` of a single simulation.
template <int N, int KIND, class T>
__device__ __forceinline__ ColSlab slab_single(typename C2<T>::t* spec, const void* tw, const double* k2tab,
                                               const Ctrl* ctrl, int it) {
  typedef PCfg<N, T> G;
  ColSlab sl;
  const int chunk = it % G::NCHUNK, line = it / G::NCHUNK;
  sl.chunk = chunk;
  sl.line = line;
  sl.gmap = false;
  sl.map = nullptr;
  sl.ctrl = const_cast<Ctrl*>(ctrl);
  sl.live = !(ctrl && ctrl->status);
  sl.tw = tw;
  sl.k2tab = k2tab;
  sl.m0 = chunk * G::CC;
  if (KIND == 2) {
    sl.spec = spec + (size_t)line * G::PITCH + chunk * G::CC;
    sl.stride = (size_t)N * G::PITCH;
    sl.jy = line;
  } else {
    sl.spec = spec + (size_t)line * N * G::PITCH + chunk * G::CC;
    sl.stride = G::PITCH;
    sl.jy = 0;
  }
  return sl;
}

// ---------------------------------------------------------------- register column passes
// The y passes and the z solve on register-resident lines (reg_fft_stages,
// E = 8 elements per thread for power-of-two N, 12 for N = 3*2^k).  A CTA of
// CC*N/E threads holds a slab of CC kx columns; thread (c, t) loads the E
// elements t + (N/E)*m of column c straight from HBM into registers and
// stores them back from registers, and in the z
// solve the -1/(k^2 N^3) scaling and the first inverse stage run on the
// registers the forward transform left.  Shared memory carries only the
// exchanges between stages: 4 accesses per element for a y pass at 512^3
// (10 through the staged transform) and 8 for the z solve (18).  The CTAs
// are persistent, so that the twiddle table is copied to shared memory once
// per CTA.
template <int N, class T> struct RCfg {
  static constexpr int CC = PCfg<N, T>::CC;
  static constexpr int E = reg_elems(N);
  static constexpr int NT = CC * (N / E);
  // Register caps per thread (via the resident CTAs per SM the kernels are
  // built for): FP64 y passes 80 (3 CTAs of 256 threads), FP64 z solve 128
  // (a cap of 80 spilled and measured 24% slower), FP32 y passes 40 (3 CTAs
  // of 512 threads; 512^3: 0.245 -> 0.234 ms against 64), FP32 z solve 64
  // (2 CTAs; 0.537 -> 0.494 ms against 40, where it spilled).
  // The next slab is prefetched into shared memory while the current one is
  // transformed, by one thread issuing tensor-map box loads (the single
  // solve's map is a kernel parameter, an ensemble slot's sits in its table
  // entry).  FP64 (512^3): y passes 0.48 -> 0.41 ms and z solve 0.94 ->
  // 0.88 ms with per-element cp.async, 0.42 -> 0.40 and 0.86 -> 0.76 ms with
  // the box loads instead.  FP32: the z solve 0.495 -> 0.438 ms with the box
  // loads; the y passes run without a prefetch (0.235 against 0.248 ms with
  // it).  The twiddle table sits in shared memory for every pass (reading it
  // through L1 measured slower for the y passes and no faster for the z
  // solve).
  static constexpr bool pf_single(int kind) { return sizeof(T) == 8 || kind == 2; }
  // the ensemble's batched passes: FP64 only (the FP32 batched z solve spills
  // with the prefetch, and its served stream ran 28% slower)
  static constexpr bool pf_batched(int) { return sizeof(T) == 8; }
  static constexpr bool stw(int) { return true; }
  // (12 elements per thread: y passes 128 in FP64 and 80 in FP32, z solves
  // 168 and 128.)
  static constexpr int minb(int kind) {
    const int r = E == 8 ? (sizeof(T) == 8 ? (kind == 2 ? 128 : 80) : (kind == 2 ? 64 : 40))
                         : (sizeof(T) == 8 ? (kind == 2 ? 168 : 128) : (kind == 2 ? 128 : 80));
    return 65536 / (NT * r) > 1 ? 65536 / (NT * r) : 1;
  }
};

// Rows of a prefetch box (the slab's N lines in N/BH boxes of at most 256).
template <int N> __host__ __device__ constexpr int rcol_box_rows() { return N <= 256 ? N : (N % 256 == 0 ? 256 : N / 2); }

template <int N, int KIND, class T, bool PF = RCfg<N, T>::pf_single(KIND)>
static size_t rcolsmem() {  // exchange buffer, twiddle table, prefetch buffer
  typedef RCfg<N, T> R;
  // prefetch buffer rounded to a 128-byte boundary, then its barrier
  const size_t head = ((size_t)reg_rows(N) * R::CC + (R::stw(KIND) ? N : 0)) * sizeof(typename C2<T>::t);
  if (!PF) return head;
  return (head + 127) / 128 * 128 + (size_t)R::E * R::NT * sizeof(typename C2<T>::t) + 8;
}

template <int N, int KIND, class T, bool PF, bool TMA, class Getter>
__device__ __forceinline__ void rcol_run(int total, const typename C2<T>::t* __restrict__ gtw, Getter get) {
  typedef typename C2<T>::t C;
  constexpr int CC = RCfg<N, T>::CC, E = RCfg<N, T>::E, TPC = N / E;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int NT = RCfg<N, T>::NT;
  C* s = reinterpret_cast<C*>(smem_raw);
  C* stw = s + reg_rows(N) * CC;
  constexpr size_t HEAD = ((size_t)reg_rows(N) * CC + (RCfg<N, T>::stw(KIND) ? N : 0)) * sizeof(C);
  C* pbuf = reinterpret_cast<C*>(smem_raw + (PF ? (HEAD + 127) / 128 * 128 : HEAD));
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(pbuf + E * NT);
  if ((int)blockIdx.x >= total) return;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      mbar_init(bar, 1);
      mbar_init_fence();
    }
    __syncthreads();
  }
  unsigned phase = 0;
  bool pend = false;  // a box load of the next slab is in flight (the same in every thread)
  const C* tw = gtw;
  if constexpr (RCfg<N, T>::stw(KIND)) {
    for (int q = threadIdx.x; q < N; q += NT) stw[q] = gtw[q];
    __syncthreads();
    tw = stw;
  }
  const int c = threadIdx.x % CC, t = threadIdx.x / CC;
  const auto at = [c](int n) { return reg_pad(n) * CC + c; };
  // prefetch: each thread copies its own eight elements of the next slab into
  // its own slots (m*NT + tid), so only its own cp.async wait orders them
  // (TMA: one thread loads the whole slab, N/BH boxes of CC columns x BH
  // lines, into the same cells: element (line n, column c) at n*CC + c)
  auto prefetch = [&](const ColSlab& ps) {
    if constexpr (TMA) {
      if (ps.live) {
        if (threadIdx.x == 0) {
          constexpr int BH = rcol_box_rows<N>();
          const CUtensorMap* map = ps.map;
          if (ps.gmap) tensormap_acquire(map);
          mbar_arrive_expect_tx(bar, (unsigned)(E * NT * sizeof(C)));
          const int x = ps.chunk * CC * 2;
#pragma unroll
          for (int b = 0; b < N / BH; ++b) {
            if (KIND == 2) tma_load_3d(pbuf + b * BH * CC, map, x, ps.line, b * BH, bar);
            else tma_load_2d(pbuf + b * BH * CC, map, x, ps.line * N + b * BH, bar);
          }
        }
        pend = true;
      }
    } else {
      if (ps.live) {
        const C* pc = static_cast<const C*>(ps.spec) + c;
#pragma unroll
        for (int m = 0; m < E; ++m)
          cp_async_elem(pbuf + m * NT + threadIdx.x, pc + (size_t)(t + TPC * m) * ps.stride);
      }
      cp_async_commit();
    }
  };
  ColSlab nx;
  if constexpr (PF) {
    nx = get(blockIdx.x);
    prefetch(nx);
  }
  for (int it = blockIdx.x; it < total; it += gridDim.x) {
    C v[E];
    ColSlab sl;
    if constexpr (PF) {
      sl = nx;
      if constexpr (TMA) {
        if (pend) {
          if (!mbar_wait(bar, phase, kWaitCycles) && sl.ctrl) atomicCAS(&sl.ctrl->status, 0, kStatusTimeout);
          phase ^= 1u;
          pend = false;
        }
      } else {
        cp_async_wait<0>();
      }
      if (sl.live) {
#pragma unroll
        for (int m = 0; m < E; ++m) v[m] = pbuf[m * NT + threadIdx.x];
      }
      nx.live = false;
      if (it + (int)gridDim.x < total) nx = get(it + gridDim.x);
      if constexpr (TMA) __syncthreads();  // every thread has read the buffer the next box fills
      prefetch(nx);
      if (!sl.live) continue;
    } else {
      sl = get(it);
      if (!sl.live) continue;  // the same for every thread of the CTA
      const C* lc = static_cast<const C*>(sl.spec) + c;
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = lc[(size_t)(t + TPC * m) * sl.stride];
    }
    C* col = static_cast<C*>(sl.spec) + c;
    if (KIND == 0) {
      reg_fft_stages<N, 1, -1>(v, s, tw, t, at);
    } else if (KIND == 1) {
      reg_fft_stages<N, 1, +1>(v, s, tw, t, at);
    } else {
      // forward z FFT, then -psi/k2/(nx*ny*nz) per mode (multi/main.f90:792,
      // one reciprocal per mode; mode (0,0,0) and the pitch padding beyond
      // kx = N/2 set to 0), then the inverse z FFT
      reg_fft_stages<N, 1, -1>(v, s, tw, t, at);
      const double nnn = (double)((long long)N * (long long)N * (long long)N);
      const double* k2tab = sl.k2tab;
      const int mx = sl.m0 + c, jy = sl.jy;
      const double k2xy = k2tab[min(mx, N - 1)] + k2tab[jy];
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int n = t + TPC * m;
        if (mx > N / 2 || (mx == 0 && jy == 0 && n == 0)) {
          v[m].x = 0;
          v[m].y = 0;
        } else {
          const double k2 = k2xy + k2tab[n];
          const T f = scale_factor<T>(k2 * nnn);
          v[m].x = v[m].x * f;
          v[m].y = v[m].y * f;
        }
      }
      reg_fft_stages<N, 1, +1>(v, s, tw, t, at);
    }
#pragma unroll
    for (int m = 0; m < E; ++m) col[(size_t)(t + TPC * m) * sl.stride] = v[m];
  }
}

template <int N, int KIND, class T>
__global__ void __launch_bounds__(RCfg<N, T>::NT, RCfg<N, T>::minb(KIND)) rcol_kernel(typename C2<T>::t* __restrict__ spec,
                                                              const typename C2<T>::t* __restrict__ tw,
                                                              const double* __restrict__ k2tab,
                                                              const Ctrl* __restrict__ ctrl,
                                                              const __grid_constant__ CUtensorMap map) {
  typedef PCfg<N, T> G;
  constexpr bool PFS = RCfg<N, T>::pf_single(KIND);
  rcol_run<N, KIND, T, PFS, PFS>(G::NCHUNK * N, tw, [&](int it) {
    ColSlab s = slab_single<N, KIND, T>(spec, tw, k2tab, ctrl, it);
    s.map = &map;
    return s;
  });
}

template <int N, int KIND, class T>
__global__ void __launch_bounds__(RCfg<N, T>::NT, RCfg<N, T>::minb(KIND)) rcol_kernel_b(const SlotArgs<T>* __restrict__ slots, int nslots,
                                                                int which) {
  typedef PCfg<N, T> G;
  const int per = G::NCHUNK * N;
  const typename C2<T>::t* tw = nullptr;
  for (int q = 0; q < nslots && !tw; ++q)
    if (slots[q].active) tw = (which ? slots[q].pr : slots[q].po).tw;
  if (!tw) return;
  constexpr bool PFB = RCfg<N, T>::pf_batched(KIND);
  rcol_run<N, KIND, T, PFB, PFB>(per * nslots, tw, [&](int it) {
    const int sl = it / per;
    const PoissonArgs<T>& a = which ? slots[sl].pr : slots[sl].po;
    ColSlab s;
    if (!slots[sl].active) {
      s.live = false;
      return s;
    }
    s = slab_single<N, KIND, T>(a.spec, a.tw, a.k2tab, a.ctrl, it - sl * per);
    s.map = KIND == 2 ? &slots[sl].maps.col_z : &slots[sl].maps.col_y;
    s.gmap = true;
    return s;
  });
}

// ---------------------------------------------------------------- register x passes
// The x passes on register-resident lines (reg_fft_stages), P*N/E threads
// per CTA, thread (q, t) holding elements t + (N/E)*m of line pair q.  x inverse: each thread reads the two half spectra at
// min(n, N - n) for its own elements n straight into registers, so the
// unpacking takes no shared-memory pass (the mirrored half reads a row
// segment another warp reads too, an L1/L2 hit); the transformed line goes
// from registers to p.  x forward: the divergence of each thread's
// elements is computed straight into registers; the transformed line is
// written once to shared memory for the Hermitian split, which needs modes
// m and N - m together.
template <int N, class T> struct XCfg {
  static constexpr int E = reg_elems(N);
  static constexpr int NT = PCfg<N, T>::P * (N / E);
  // exchange slots of a line (see reg_pad / reg_swz) and the line stride
  static constexpr int LS = sizeof(T) == 8 ? reg_rows(N) : N;
  static __device__ __forceinline__ int slot(int n) { return sizeof(T) == 8 ? reg_pad(n) : reg_swz(n); }
};

template <int N, class T>
__device__ __forceinline__ void xinv_reg_body(const typename C2<T>::t* __restrict__ spec, T* __restrict__ p,
                                              const typename C2<T>::t* __restrict__ tw,
                                              const Ctrl* __restrict__ ctrl, int bx, int by) {
  typedef typename C2<T>::t C;
  typedef PCfg<N, T> G;
  constexpr int E = XCfg<N, T>::E, TPC = N / E;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int t = threadIdx.x % TPC, q = threadIdx.x / TPC;
  const int k = by, ja = bx * (2 * G::P) + 2 * q;
  const C* row = spec + ((size_t)k * N + ja) * G::PITCH;
  C A[E], B[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = t + TPC * m;
    const int h = (n <= N / 2) ? n : N - n;
    A[m] = row[h];
    B[m] = row[G::PITCH + h];
  }
  // z = A + iB on modes 0..N/2 and its Hermitian mirror above (the imaginary
  // parts of modes 0 and N/2 dropped)
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = t + TPC * m;
    C a = A[m], b = B[m];
    if (n == 0 || n == N / 2) {
      a.y = 0;
      b.y = 0;
    }
    if (n <= N / 2) {
      v[m].x = a.x - b.y;
      v[m].y = a.y + b.x;
    } else {
      v[m].x = a.x + b.y;
      v[m].y = b.x - a.y;
    }
  }
  const int base = q * XCfg<N, T>::LS;
  reg_fft_stages<N, 1, +1>(v, s, tw, t, [base](int n) { return base + XCfg<N, T>::slot(n); });
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = t + TPC * m;
    p[gidx(n, ja, k, N)] = v[m].x;
    p[gidx(n, ja + 1, k, N)] = v[m].y;
  }
}

template <int N, int MODE, class T>
__device__ __forceinline__ void xfwd_reg_body(const T* __restrict__ us, const T* __restrict__ vs,
                                              const T* __restrict__ ws, const T* __restrict__ rhs,
                                              const T* __restrict__ p0, typename C2<T>::t* __restrict__ spec,
                                              const typename C2<T>::t* __restrict__ tw,
                                              const Ctrl* __restrict__ ctrl, double cdiv, double ddxi, int bx,
                                              int by) {
  typedef typename C2<T>::t C;
  typedef PCfg<N, T> G;
  constexpr int E = XCfg<N, T>::E, TPC = N / E, M = N / 2 + 1;
  if (ctrl && ctrl->status) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* s = reinterpret_cast<C*>(smem_raw);
  const int t = threadIdx.x % TPC, q = threadIdx.x / TPC;
  const int k = by, j0 = bx * (2 * G::P);
  const int ja = j0 + 2 * q;
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int n = t + TPC * m;
    v[m].x = (T)xfwd_rhs<N, MODE, T>(us, vs, ws, rhs, p0, cdiv, ddxi, n, ja, k);
    v[m].y = (T)xfwd_rhs<N, MODE, T>(us, vs, ws, rhs, p0, cdiv, ddxi, n, ja + 1, k);
  }
  const int base = q * XCfg<N, T>::LS;
  const auto at = [base](int n) { return base + XCfg<N, T>::slot(n); };
  reg_fft_stages<N, 1, -1>(v, s, tw, t, at);
#pragma unroll
  for (int m = 0; m < E; ++m) s[at(t + TPC * m)] = v[m];
  __syncthreads();
  const T half = (T)0.5;
  for (int wi = threadIdx.x; wi < G::P * M; wi += XCfg<N, T>::NT) {
    const int m = wi % M, pq = wi / M;
    const int jb = j0 + 2 * pq;
    const C zm = s[pq * XCfg<N, T>::LS + XCfg<N, T>::slot(m)];
    const int mr = (m == 0) ? 0 : (N - m);
    const C zr = s[pq * XCfg<N, T>::LS + XCfg<N, T>::slot(mr)];
    C Am, Bm;
    Am.x = half * (zm.x + zr.x);
    Am.y = half * (zm.y - zr.y);
    Bm.x = half * (zm.y + zr.y);
    Bm.y = -half * (zm.x - zr.x);
    C* orow = spec + ((size_t)k * N + jb) * G::PITCH;
    orow[m] = Am;
    orow[G::PITCH + m] = Bm;
  }
}

// ---------------------------------------------------------------- x inverse fused with the projection
// Power-of-two N >= 256 (C2 + R1 of multi/main.f90:812-903 in one pass): the
// pressure never goes to HBM.  A CTA owns the output rows j0 .. j0+2P-1 of
// a chunk of KZ planes and marches through them.  Per plane it runs the x
// inverse of its P line pairs plus one halo pair below (rows j0-2, j0-1;
// the projection's backward difference in y needs row j0-1), puts the
// plane's pressure rows into shared memory, and projects the plane:
//   u = ustar - dt/rho*(p - p(i-1))*dxi, v with p(j-1), w with p(k-1),
// where p(k-1) is the previous plane's rows, kept in a second buffer (the
// chunk starts one plane early to fill it).  Per-CTA FP64 sums and maxima
// as in project_body, in a fixed order.
//   * FP64 step (T = double): p is the x inverse of the spectrum.  The x
//     inverse is xinv_reg_body's arithmetic and the projection
//     project_body's, so u, v, w and the pressure (recomputed from the
//     spectrum on request) are the same bits as the unfused kernels give;
//     only the grouping of the sums that make the means differs.  Traffic
//     per point: the half spectrum (8.06 B, plus the halo rows, mostly L2
//     hits) + ustar, vstar, wstar + u, v, w: the 280 B/pt schedule instead
//     of 296.
//   * FP32 refinement form (T = float): the spectrum is the correction
//     solve's; its x inverse is dp, and the pressure p = p0 + dp is formed
//     in FP64 from the first solve's stored p0.  The projection runs in FP64
//     and rounds u, v, w to FP32 when storing them (project_refine_body's
//     arithmetic, without its forward-difference divergence, which
//     refine_divergence measures on request from the same stored inputs).
//     dp never goes to HBM: 32 B/pt instead of the 40 of the separate x
//     inverse and projection.
template <int N, class T> struct XPCfg {
  static constexpr bool ON = (N & (N - 1)) == 0 && N >= 256;  // power-of-two sizes (8 elements per thread)
  static constexpr int P = PCfg<N, T>::P;
  static constexpr int TPC = N / 8;
  static constexpr int NT = (P + 1) * TPC;  // a multiple of 32 for N >= 256
  static constexpr int KZ = N >= 512 ? 16 : 8;
  static constexpr size_t XBYTES = (size_t)(P + 1) * XCfg<N, T>::LS * sizeof(typename C2<T>::t);  // exchange
  static constexpr size_t PBYTES = (size_t)(2 * P + 1) * N * sizeof(double);  // plane's p rows
  static constexpr size_t ABYTES = XBYTES > PBYTES ? XBYTES : PBYTES;        // the two alias
  static constexpr size_t SMEM = ABYTES + (size_t)2 * P * N * sizeof(double);  // + previous plane
  static constexpr int PARTS = (N / (2 * P)) * (N / KZ);
};

template <int N, class T>
__device__ __forceinline__ void xinvproj_body(const typename C2<T>::t* __restrict__ spec,
                                              const typename C2<T>::t* __restrict__ tw, const StencilArgs<T>& a,
                                              int bx, int bz, int gx) {
  typedef typename C2<T>::t C;
  typedef XPCfg<N, T> X;
  constexpr bool REF = sizeof(T) == 4;  // FP32 refinement form: p = p0 + dp
  constexpr int P = X::P, TPC = X::TPC, NT = X::NT, KZ = X::KZ;
  constexpr size_t PITCH = PCfg<N, T>::PITCH;
  static_assert(NT % 32 == 0, "whole warps");
  if (a.ctrl->status) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* sx = reinterpret_cast<C*>(smem_raw);
  double* sp = reinterpret_cast<double*>(smem_raw);  // the plane's p rows, after its transform
  double* spp = reinterpret_cast<double*>(smem_raw + X::ABYTES);  // the previous plane's rows
  const int t = threadIdx.x % TPC, q = threadIdx.x / TPC;        // q == P: the halo pair
  const int j0 = bx * (2 * P), k0 = bz * KZ;
  const int ja = (q < P) ? j0 + 2 * q : (j0 - 2 + N) % N;
  const double dtr = a.c.dtr, dxi = a.c.dxi;
  const size_t nn = (size_t)N * N;
  const T* __restrict__ us = a.us;
  const T* __restrict__ vs = a.vs;
  const T* __restrict__ ws = a.ws;
  T* __restrict__ uo_ = a.uo;
  T* __restrict__ vo_ = a.vo;
  T* __restrict__ wo_ = a.wo;
  constexpr int PIT = (2 * P * N + NT - 1) / NT;  // projection points per thread and plane
  constexpr int PG = 4;
  double su = 0, sv = 0, sw = 0;
  double xu = -INFINITY, xv = -INFINITY, xw = -INFINITY;
  const int base = q * XCfg<N, T>::LS;
  const auto at = [base](int n) { return base + XCfg<N, T>::slot(n); };
  for (int kk = k0 - 1; kk < k0 + KZ; ++kk) {
    const int kw = (kk + N) % N;
    // (1) x inverse of the plane's line pairs (xinv_reg_body)
    const C* row = spec + ((size_t)kw * N + ja) * PITCH;
    C A[8], B[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int n = t + TPC * m;
      const int h = (n <= N / 2) ? n : N - n;
      A[m] = row[h];
      B[m] = row[PITCH + h];
    }
    // FP32 refinement form: the first solve's p0 on the same two rows
    T pa0[8], pb0[8];
    if constexpr (REF) {
      const T* __restrict__ p0 = a.p;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const size_t g = (size_t)(t + TPC * m) + (size_t)N * ja + nn * kw;
        pa0[m] = (q < P) ? p0[g] : (T)0;
        pb0[m] = p0[g + N];
      }
    }
    C v[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int n = t + TPC * m;
      C ca = A[m], cb = B[m];
      if (n == 0 || n == N / 2) {
        ca.y = 0;
        cb.y = 0;
      }
      if (n <= N / 2) {
        v[m].x = ca.x - cb.y;
        v[m].y = ca.y + cb.x;
      } else {
        v[m].x = ca.x + cb.y;
        v[m].y = cb.x - ca.y;
      }
    }
    reg_fft_stages<N, 1, +1>(v, sx, tw, t, at);  // ends with a barrier: sx is free
    // (2) the plane's p rows: row 0 = j0-1 (second line of the halo pair),
    // rows 1 .. 2P = j0 .. j0+2P-1
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int n = t + TPC * m;
      if constexpr (REF) {
        const double pa = (double)pa0[m] + (double)v[m].x, pb = (double)pb0[m] + (double)v[m].y;
        if (q < P) {
          sp[(2 * q + 1) * N + n] = pa;
          sp[(2 * q + 2) * N + n] = pb;
        } else {
          sp[n] = pb;
        }
      } else {
        if (q < P) {
          sp[(2 * q + 1) * N + n] = v[m].x;
          sp[(2 * q + 2) * N + n] = v[m].y;
        } else {
          sp[n] = v[m].y;
        }
      }
    }
    __syncthreads();
    // (3) projection of plane kw (the chunk's first pass only fills spp).
    // A thread's points are tid + NT*it; they are taken in groups of PG
    // whose ustar/vstar/wstar loads are all issued before the group's
    // arithmetic and stores (ustar and u are distinct arrays), so that a
    // group costs one memory latency rather than PG.
    if (kk >= k0) {
#pragma unroll 1
      for (int it0 = 0; it0 < PIT; it0 += PG) {
        T lu[PG], lv[PG], lw[PG];
#pragma unroll
        for (int c = 0; c < PG; ++c) {
          const int pi = threadIdx.x + NT * (it0 + c);
          if (pi < 2 * P * N) {
            const int x = pi % N, r = pi / N;
            const size_t g = (size_t)x + (size_t)N * (j0 + r) + nn * kw;
            lu[c] = us[g];
            lv[c] = vs[g];
            lw[c] = ws[g];
          }
        }
#pragma unroll
        for (int c = 0; c < PG; ++c) {
          const int pi = threadIdx.x + NT * (it0 + c);
          if (pi < 2 * P * N) {
            const int x = pi % N, r = pi / N;
            const double pc = sp[(r + 1) * N + x];
            const double pxm = sp[(r + 1) * N + (x ? x - 1 : N - 1)];
            const double pym = sp[r * N + x];
            const double pzm = spp[r * N + x];
            const size_t g = (size_t)x + (size_t)N * (j0 + r) + nn * kw;
            const double uo = (double)lu[c] - dtr * (pc - pxm) * dxi;
            const double vo = (double)lv[c] - dtr * (pc - pym) * dxi;
            const double wo = (double)lw[c] - dtr * (pc - pzm) * dxi;
            uo_[g] = (T)uo;
            vo_[g] = (T)vo;
            wo_[g] = (T)wo;
            su += uo;
            sv += vo;
            sw += wo;
            xu = fmax(xu, uo);
            xv = fmax(xv, vo);
            xw = fmax(xw, wo);
            // NaN must not vanish in fmax: fold it into the sums too
            if (uo != uo || vo != vo || wo != wo) su = NAN;
            spp[r * N + x] = pc;
          }
        }
      }
    } else {
      for (int pi = threadIdx.x; pi < 2 * P * N; pi += NT) spp[pi] = sp[N + pi];
    }
    __syncthreads();  // sp (which aliases sx) is free for the next transform
  }
  // deterministic block reduction: xor-shuffle in warps, then warps in order
  double vals[6] = {su, sv, sw, xu, xv, xw};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) vals[c] += __shfl_xor_sync(0xffffffffu, vals[c], o);
#pragma unroll
    for (int c = 3; c < 6; ++c) vals[c] = fmax(vals[c], __shfl_xor_sync(0xffffffffu, vals[c], o));
  }
  __shared__ double red[NT / 32][6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 6; ++c) red[wid][c] = vals[c];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r6[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) r6[c] = red[0][c];
    for (int w = 1; w < NT / 32; ++w) {
      for (int c = 0; c < 3; ++c) r6[c] += red[w][c];
      for (int c = 3; c < 6; ++c) r6[c] = fmax(r6[c], red[w][c]);
    }
    const size_t b = (size_t)bx + (size_t)gx * bz;
    for (int c = 0; c < 6; ++c) a.partials[b * 6 + c] = r6[c];
  }
}

template <int N, class T>
__global__ void __launch_bounds__(XPCfg<N, T>::NT, 2) xinvproj_kernel(const typename C2<T>::t* __restrict__ spec,
                                                                      const typename C2<T>::t* __restrict__ tw,
                                                                      StencilArgs<T> a) {
  if constexpr (XPCfg<N, T>::ON) xinvproj_body<N, T>(spec, tw, a, blockIdx.x, blockIdx.y, gridDim.x);
}
// Batched: the FP64 step transforms the slot's spectrum, the FP32
// refinement form its correction spectrum.
template <int N, class T>
__global__ void __launch_bounds__(XPCfg<N, T>::NT, 2) xinvproj_kernel_b(const SlotArgs<T>* __restrict__ slots,
                                                                        int zch) {
  if constexpr (XPCfg<N, T>::ON) {
    const int sl = blockIdx.y / zch;
    if (!slots[sl].active) return;
    const PoissonArgs<T>& pa = (sizeof(T) == 4) ? slots[sl].pr : slots[sl].po;
    xinvproj_body<N, T>(pa.spec, pa.tw, slots[sl].st, blockIdx.x, blockIdx.y - sl * zch, gridDim.x);
  }
}

// ---------------------------------------------------------------- entry points
// Single solve: block coordinates are the grid's.
// x passes: 3 CTAs of up to 256 threads per SM with 8 elements per thread, 2
// with 12 (their registers); 4 for the FP32 divergence pass (64 registers,
// no spill: 0.469 -> 0.446 ms at 512^3 on B200).
template <int N, int MODE, class T> __host__ __device__ constexpr int xfwd_min_blocks() {
  return reg_elems(N) == 8 ? (sizeof(T) == 4 && MODE != 2 ? 4 : 3) : 2;
}
template <int N, int MODE, class T>
__global__ void __launch_bounds__(256, xfwd_min_blocks<N, MODE, T>()) xfwd_kernel(const T* __restrict__ us, const T* __restrict__ vs,
                                                  const T* __restrict__ ws, const T* __restrict__ rhs,
                                                  const T* __restrict__ p0, typename C2<T>::t* __restrict__ spec,
                                                  const typename C2<T>::t* __restrict__ tw,
                                                  const Ctrl* __restrict__ ctrl, double cdiv, double ddxi) {
  xfwd_reg_body<N, MODE, T>(us, vs, ws, rhs, p0, spec, tw, ctrl, cdiv, ddxi, blockIdx.x, blockIdx.y);
}
template <int N, class T>
__global__ void __launch_bounds__(256, reg_elems(N) == 8 ? 3 : 2) xinv_kernel(const typename C2<T>::t* __restrict__ spec, T* __restrict__ p,
                                                  const typename C2<T>::t* __restrict__ tw,
                                                  const Ctrl* __restrict__ ctrl) {
  xinv_reg_body<N, T>(spec, p, tw, ctrl, blockIdx.x, blockIdx.y);
}

// Batched over the slots of a served ensemble: grid y = slot * N + plane.
// `which` selects the slot's first (0) or correction (1) solve.
template <int N, int MODE, class T>
__global__ void __launch_bounds__(256, xfwd_min_blocks<N, MODE, T>()) xfwd_kernel_b(const SlotArgs<T>* __restrict__ slots, int which) {
  const int sl = blockIdx.y / N;
  if (!slots[sl].active) return;
  const PoissonArgs<T>& a = which ? slots[sl].pr : slots[sl].po;
  xfwd_reg_body<N, MODE, T>(a.us, a.vs, a.ws, a.rhs, a.pres, a.spec, a.tw, a.ctrl, a.cdiv, a.ddxi, blockIdx.x,
                            blockIdx.y - sl * N);
}
template <int N, class T>
__global__ void __launch_bounds__(256, reg_elems(N) == 8 ? 3 : 2) xinv_kernel_b(const SlotArgs<T>* __restrict__ slots, int which) {
  const int sl = blockIdx.y / N;
  if (!slots[sl].active) return;
  const PoissonArgs<T>& a = which ? slots[sl].pr : slots[sl].po;
  xinv_reg_body<N, T>(a.spec, a.p, a.tw, a.ctrl, blockIdx.x, blockIdx.y - sl * N);
}

// ---------------------------------------------------------------- launchers
template <int N, class T> static size_t xsmem() {
  return (size_t)PCfg<N, T>::P * XCfg<N, T>::LS * sizeof(typename C2<T>::t);
}

// Persistent grid of the column passes: resident CTAs per SM (occupancy)
// times the SM count.
template <int N, int KIND, class T, bool BATCHED> static int rcolgrid() {
  static int grid = 0;
  if (!grid) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (BATCHED)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rcol_kernel_b<N, KIND, T>, RCfg<N, T>::NT,
                                                    rcolsmem<N, KIND, T, RCfg<N, T>::pf_batched(KIND)>());
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rcol_kernel<N, KIND, T>, RCfg<N, T>::NT,
                                                    rcolsmem<N, KIND, T, RCfg<N, T>::pf_single(KIND)>());
    grid = std::max(1, sms) * std::max(1, per);
  }
  return grid;
}

// Column pass KIND of one solve / of the slots of an ensemble class.
// Where the single solve prefetches (pf_single): a tensor map of the half
// spectrum as reals, (2*PITCH, N*N rows) for the y passes and (2*PITCH, N,
// N) for the z solve, boxes of CC columns by BH lines.
// The spectrum view column pass KIND prefetches from (where it prefetches):
// the half spectrum as reals, (2*PITCH, N*N rows) for the y passes and
// (2*PITCH, N, N) for the z solve, boxes of CC columns by BH lines.
template <int N, int KIND, class T> static cudaError_t col_map(CUtensorMap* map, const void* spec) {
  typedef PCfg<N, T> G;
  memset(map, 0, sizeof(*map));
  if constexpr (!RCfg<N, T>::pf_single(KIND)) return cudaSuccess;
  const uint64_t row = (uint64_t)G::PITCH * sizeof(typename C2<T>::t);
  const uint32_t bh = (uint32_t)rcol_box_rows<N>(), bw = (uint32_t)(2 * G::CC);
  if (KIND == 2) {
    const uint64_t dims[3] = {(uint64_t)2 * G::PITCH, (uint64_t)N, (uint64_t)N};
    const uint64_t strides[2] = {row, row * N};
    const uint32_t box[3] = {bw, 1, bh};
    return encode_tensor_map(map, 3, spec, dims, strides, box, (int)sizeof(T));
  }
  const uint64_t dims[2] = {(uint64_t)2 * G::PITCH, (uint64_t)N * N};
  const uint64_t strides[1] = {row};
  const uint32_t box[2] = {bw, bh};
  return encode_tensor_map(map, 2, spec, dims, strides, box, (int)sizeof(T));
}

template <int N, int KIND, class T> static void launch_col(const PoissonArgs<T>& a, cudaStream_t st) {
  CUtensorMap map;
  if (col_map<N, KIND, T>(&map, a.spec)) {  // surfaces as the launch error of an empty grid
    rcol_kernel<N, KIND, T><<<0, 1, 0, st>>>(a.spec, a.tw, a.k2tab, a.ctrl, map);
    return;
  }
  rcol_kernel<N, KIND, T><<<rcolgrid<N, KIND, T, false>(), RCfg<N, T>::NT, rcolsmem<N, KIND, T>(), st>>>(
      a.spec, a.tw, a.k2tab, a.ctrl, map);
}
template <int N, int KIND, class T>
static void launch_col_b(const SlotArgs<T>* slots, int nslots, int which, cudaStream_t st) {
  rcol_kernel_b<N, KIND, T><<<rcolgrid<N, KIND, T, true>(), RCfg<N, T>::NT,
                               rcolsmem<N, KIND, T, RCfg<N, T>::pf_batched(KIND)>(), st>>>(
      slots, nslots, which);
}

template <int N, class T> static cudaError_t set_attrs() {
  cudaError_t e;
  const int xs = (int)xsmem<N, T>();
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 0, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 1, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel<N, 2, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xinv_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel_b<N, 0, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xfwd_kernel_b<N, 2, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  if ((e = cudaFuncSetAttribute(xinv_kernel_b<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs))) return e;
  {
    const int r0 = (int)rcolsmem<N, 0, T, RCfg<N, T>::pf_batched(0)>(),
              r1 = (int)rcolsmem<N, 1, T, RCfg<N, T>::pf_batched(1)>(),
              r2 = (int)rcolsmem<N, 2, T, RCfg<N, T>::pf_batched(2)>();
    const cudaFuncAttribute A = cudaFuncAttributeMaxDynamicSharedMemorySize;
    const int q0 = (int)rcolsmem<N, 0, T, RCfg<N, T>::pf_single(0)>(),
              q1 = (int)rcolsmem<N, 1, T, RCfg<N, T>::pf_single(1)>(),
              q2 = (int)rcolsmem<N, 2, T, RCfg<N, T>::pf_single(2)>();
    if ((e = cudaFuncSetAttribute(rcol_kernel<N, 0, T>, A, q0))) return e;
    if ((e = cudaFuncSetAttribute(rcol_kernel<N, 1, T>, A, q1))) return e;
    if ((e = cudaFuncSetAttribute(rcol_kernel<N, 2, T>, A, q2))) return e;
    if ((e = cudaFuncSetAttribute(rcol_kernel_b<N, 0, T>, A, r0))) return e;
    if ((e = cudaFuncSetAttribute(rcol_kernel_b<N, 1, T>, A, r1))) return e;
    if ((e = cudaFuncSetAttribute(rcol_kernel_b<N, 2, T>, A, r2))) return e;
  }
  if constexpr (XPCfg<N, T>::ON) {
    const int xs2 = (int)XPCfg<N, T>::SMEM;
    if ((e = cudaFuncSetAttribute(xinvproj_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs2))) return e;
    if ((e = cudaFuncSetAttribute(xinvproj_kernel_b<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, xs2)))
      return e;
  }
  return cudaSuccess;
}

template <int N, class T>
static void launch_xfwd(const PoissonArgs<T>& a, cudaStream_t st) {
  typedef PCfg<N, T> G;
  const dim3 gx(N / (2 * G::P), N);
  const size_t xs = xsmem<N, T>();
  if (a.rhs)
    xfwd_kernel<N, 1, T><<<gx, XCfg<N, T>::NT, xs, st>>>(nullptr, nullptr, nullptr, a.rhs, nullptr, a.spec, a.tw, a.ctrl,
                                                a.cdiv, a.ddxi);
  else if (a.pres)
    xfwd_kernel<N, 2, T><<<gx, XCfg<N, T>::NT, xs, st>>>(a.us, a.vs, a.ws, nullptr, a.pres, a.spec, a.tw, a.ctrl, a.cdiv,
                                                a.ddxi);
  else
    xfwd_kernel<N, 0, T><<<gx, XCfg<N, T>::NT, xs, st>>>(a.us, a.vs, a.ws, nullptr, nullptr, a.spec, a.tw, a.ctrl, a.cdiv,
                                                a.ddxi);
}

template <int N, class T>
static cudaError_t poisson_run(const PoissonArgs<T>& a, cudaStream_t st) {
  typedef PCfg<N, T> G;
  const dim3 gx(N / (2 * G::P), N);
  const size_t xs = xsmem<N, T>();
  launch_xfwd<N, T>(a, st);
  launch_col<N, 0, T>(a, st);
  launch_col<N, 2, T>(a, st);
  launch_col<N, 1, T>(a, st);
  xinv_kernel<N, T><<<gx, XCfg<N, T>::NT, xs, st>>>(a.spec, a.p, a.tw, a.ctrl);
  return cudaGetLastError();
}

template <int N, class T>
static cudaError_t xinvproj_run(const PoissonArgs<T>& pa, const StencilArgs<T>& a, cudaStream_t st) {
  if constexpr (XPCfg<N, T>::ON) {
    const dim3 grid(N / (2 * XPCfg<N, T>::P), N / XPCfg<N, T>::KZ);
    xinvproj_kernel<N, T><<<grid, XPCfg<N, T>::NT, XPCfg<N, T>::SMEM, st>>>(pa.spec, pa.tw, a);
    return cudaGetLastError();
  }
  return cudaErrorInvalidValue;
}
template <int N, class T>
static cudaError_t xinvproj_run_b(const SlotArgs<T>* slots, int nslots, cudaStream_t st) {
  if constexpr (XPCfg<N, T>::ON) {
    const dim3 grid(N / (2 * XPCfg<N, T>::P), (N / XPCfg<N, T>::KZ) * nslots);
    xinvproj_kernel_b<N, T><<<grid, XPCfg<N, T>::NT, XPCfg<N, T>::SMEM, st>>>(slots, N / XPCfg<N, T>::KZ);
    return cudaGetLastError();
  }
  return cudaErrorInvalidValue;
}

template <int N, class T>
static cudaError_t poisson_stage(const PoissonArgs<T>& a, int stage, cudaStream_t st) {
  typedef PCfg<N, T> G;
  const dim3 gx(N / (2 * G::P), N);
  const size_t xs = xsmem<N, T>();
  switch (stage) {
    case 0: launch_xfwd<N, T>(a, st); break;
    case 1: launch_col<N, 0, T>(a, st); break;
    case 2: launch_col<N, 2, T>(a, st); break;
    case 3: launch_col<N, 1, T>(a, st); break;
    case 4: xinv_kernel<N, T><<<gx, XCfg<N, T>::NT, xs, st>>>(a.spec, a.p, a.tw, a.ctrl); break;
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
template <class T> cudaError_t encode_column_maps(SlotMaps* m, const void* spec, int n) {
  cudaError_t e;
  switch (n) {
#define CM_CASE(NN)                                                        \
  case NN:                                                                 \
    if ((e = col_map<NN, 0, T>(&m->col_y, spec))) return e;                \
    return col_map<NN, 2, T>(&m->col_z, spec);
    MHIT_FOR_SIZES(CM_CASE)
#undef CM_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
template cudaError_t encode_column_maps<double>(SlotMaps*, const void*, int);
template cudaError_t encode_column_maps<float>(SlotMaps*, const void*, int);

template cudaError_t launch_poisson_stage<double>(int, const PoissonArgs<double>&, int, cudaStream_t);
template cudaError_t launch_poisson_stage<float>(int, const PoissonArgs<float>&, int, cudaStream_t);

template <int N, class T>
static cudaError_t poisson_stage_b(const SlotArgs<T>* slots, int nslots, int stage, int which, cudaStream_t st) {
  typedef PCfg<N, T> G;
  const dim3 gx(N / (2 * G::P), N * nslots);
  const size_t xs = xsmem<N, T>();
  switch (stage) {
    case 0:
      if (which)
        xfwd_kernel_b<N, 2, T><<<gx, XCfg<N, T>::NT, xs, st>>>(slots, 1);
      else
        xfwd_kernel_b<N, 0, T><<<gx, XCfg<N, T>::NT, xs, st>>>(slots, 0);
      break;
    case 1: launch_col_b<N, 0, T>(slots, nslots, which, st); break;
    case 2: launch_col_b<N, 2, T>(slots, nslots, which, st); break;
    case 3: launch_col_b<N, 1, T>(slots, nslots, which, st); break;
    case 4: xinv_kernel_b<N, T><<<gx, XCfg<N, T>::NT, xs, st>>>(slots, which); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_poisson_stage_batched(const SlotArgs<T>* slots, int nslots, int n, int stage, int which,
                                         cudaStream_t st) {
  if ((long long)n * nslots > 65535) return cudaErrorInvalidConfiguration;
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return poisson_stage_b<NN, T>(slots, nslots, stage, which, st);
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_poisson_stage_batched<double>(const SlotArgs<double>*, int, int, int, int, cudaStream_t);
template cudaError_t launch_poisson_stage_batched<float>(const SlotArgs<float>*, int, int, int, int, cudaStream_t);

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

template <class T>
cudaError_t launch_xinv_project(int n, const PoissonArgs<T>& pa, const StencilArgs<T>& a, cudaStream_t st) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return xinvproj_run<NN, T>(pa, a, st);
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_xinv_project<double>(int, const PoissonArgs<double>&, const StencilArgs<double>&,
                                                 cudaStream_t);
template cudaError_t launch_xinv_project<float>(int, const PoissonArgs<float>&, const StencilArgs<float>&,
                                                cudaStream_t);

template <class T>
cudaError_t launch_xinv_project_batched(const SlotArgs<T>* slots, int nslots, int n, cudaStream_t st) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return xinvproj_run_b<NN, T>(slots, nslots, st);
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_xinv_project_batched<double>(const SlotArgs<double>*, int, int, cudaStream_t);
template cudaError_t launch_xinv_project_batched<float>(const SlotArgs<float>*, int, int, cudaStream_t);

int fused_projection(int n) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return (XPCfg<NN, double>::ON && XPCfg<NN, float>::ON) ? 1 : 0;
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return 0;
  }
}

int xinv_project_partials(int n) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return XPCfg<NN, double>::ON ? XPCfg<NN, double>::PARTS : 0;
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return 0;
  }
}

size_t spectrum_pitch(int n, int fp32) {
  switch (n) {
#define MHIT_CASE(NN) \
  case NN:            \
    return fp32 ? PCfg<NN, float>::PITCH : PCfg<NN, double>::PITCH;
    MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
    default:
      return 0;
  }
}

template cudaError_t launch_poisson<double>(int, const PoissonArgs<double>&, cudaStream_t);
template cudaError_t launch_poisson<float>(int, const PoissonArgs<float>&, cudaStream_t);

}  // namespace mhit
