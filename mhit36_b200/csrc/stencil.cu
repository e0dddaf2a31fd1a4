// Stencil kernels of the MHIT36 step on one B200: the ACDI phase-field update,
// the momentum RHS + AB2 predictor, the projection with the mean/max
// reductions, and the one-block finalize.
//
// Fields are stored without halo cells, x fastest (n^3 values); periodic
// neighbours come from index wrap.  On one rank this is exactly what the
// reference's cuDecomp halo updates (periodic, multi/main.f90:418-429,
// 483-486, 630-641, 685-696, 817-818, 923-934) provide, so none of the 28 halo
// calls of a reference step has a counterpart here.
//
// Both stencil kernels march a TX x TY column tile through a chunk of KZ z
// planes ("2.5D" blocking): each z plane of every input is read from HBM once
// per tile (plus its x/y halo ring, mostly L2 hits), kept in a small ring of
// shared-memory planes, and every intermediate the reference materialises in
// HBM (psidi, normx/y/z, rhsphi, rhsu/v/w, chempot, gradphi*, f*st) lives
// only in shared memory or registers.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include "common.cuh"
#include "internal.h"

namespace mhit {

constexpr int TX = 32, TY = 8, NT = TX * TY;

// Default z chunk of the stencil kernels: 64 planes from 512^3 up (measured
// 2-3% faster than 32 there on B200; the grid still has >= 13 waves), 32
// below, so that smaller grids keep enough CTAs.
static int pick_kz(int n) { return n >= 512 ? 64 : (n >= 32 ? 32 : n); }

// Momentum tile height.  Both tiles run 256 threads; the 16-row tile gives
// each thread two rows.  Measured on B200 at 512^3: FP64 8 rows 3.06 ms,
// 16 rows 4.18 ms (128 registers); FP32 8 rows 2.00 ms, 16 rows 1.87 ms.
int default_mty(int n, int fp32) { return (n >= 16 && fp32) ? 16 : 8; }

// ============================================================ psi arithmetic
// psi = eps*log(a/b) (A3) is the phase kernel's most expensive expression.
// FP64: a/b by Newton-Raphson from the PTX reciprocal approximation
// (rcp.approx.ftz.f64, two iterations and a remainder correction: the
// correctly rounded quotient for these operands, which are normal numbers
// in [1e-16, 1 + 1e-16]), and the logarithm by P. T. P. Tang's table-driven
// method ("Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16(4), 1990): x = 2^k m, m in
// [1, 2), F = 1 + j/128 nearest to m, r = (m - F)/F with |r| <= 2^-8, and
// log x = k ln2 + log F + log(1 + r), the last by its Taylor series to r^7
// (truncation below 2^-59 relative).  log F and ln2 are double-double
// values computed on the host in long double.  Both are branch-free, so the
// psi of a thread's elements overlap.  Measured against CUDA's log and
// division on B200 over 134M phase-field values: at most 2 ulp apart, and
// 1.45x faster.  FP32: the hardware approximations __fdividef and __logf
// (about 1 ulp of psi on these operands).
constexpr int LOGTAB = 3 * 129 + 2;  // 1/F, log F (hi), log F (lo), then ln2 (hi, lo)
__device__ double g_log_table[LOGTAB];

__device__ __forceinline__ double div_nr(double a, double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  const double q = a * y;
  return fma(fma(-b, q, a), y, q);
}

// log x for positive normal x; tab = g_log_table (in shared memory)
__device__ __forceinline__ double tang_log(double x, const double* __restrict__ tab) {
  const int hi = __double2hiint(x), lo = __double2loint(x);
  const int k = (hi >> 20) - 1023;
  const int mant = hi & 0x000fffff;
  const int j = (mant + (1 << 12)) >> 13;  // nearest j/128, 0..128
  const double m = __hiloint2double(mant | 0x3ff00000, lo);
  const double r = (m - (1.0 + (double)j * (1.0 / 128))) * tab[j];  // m - F is exact
  double p = fma(r, 1.0 / 7, -1.0 / 6);
  p = fma(p, r, 0.2);
  p = fma(p, r, -0.25);
  p = fma(p, r, 1.0 / 3);
  p = fma(p, r, -0.5);
  p = fma(p, r * r, r);
  const double kd = (double)k;
  return fma(kd, tab[3 * 129], tab[129 + j]) + (fma(kd, tab[3 * 129 + 1], tab[2 * 129 + j]) + p);
}

template <class T> struct PsiMath;
template <> struct PsiMath<double> {
  static constexpr int TAB = LOGTAB;  // table entries staged in shared memory
  static __device__ __forceinline__ double log_ratio(double a, double b, const double* tab) {
    return tang_log(div_nr(a, b), tab);
  }
};
template <> struct PsiMath<float> {
  static constexpr int TAB = 0;
  static __device__ __forceinline__ float log_ratio(float a, float b, const double*) { return __logf(__fdividef(a, b)); }
};

// The table of tang_log, once per device (before any graph capture).
static cudaError_t upload_log_table() {
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e) return e;
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  double t[LOGTAB];
  for (int j = 0; j <= 128; ++j) {
    const long double F = 1.0L + (long double)j / 128.0L;
    const long double l = logl(F);
    t[j] = (double)(1.0L / F);
    t[129 + j] = (double)l;
    t[2 * 129 + j] = (double)(l - (long double)t[129 + j]);
  }
  const long double ln2 = logl(2.0L);
  t[3 * 129] = (double)ln2;
  t[3 * 129 + 1] = (double)(ln2 - (long double)t[3 * 129]);
  if ((e = cudaMemcpyToSymbol(g_log_table, t, sizeof(t)))) return e;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return cudaSuccess;
}

// ============================================================ phase field
// ACDI step A1..A7 (multi/main.f90:341-480) fused into one kernel:
//   psi = eps*log((min(phi,1)+enum)/(1-min(phi,1)+enum))      (A3)
//   n   = grad(psi) / (|grad(psi)| + 1e-16f)                  (A4, A5)
//   F   = 0.25*(1 - tanh(psi/(2 eps))^2) * n                  (A6 flux)
//   rhs = -div(u phi_face) + gamma*eps*lap(phi) - gamma*div_c(F)   (A1, A2, A6)
//   phi_new = phi + dt*rhs                                    (A7)
// psi needs phi on a radius-2 neighbourhood; it is computed per plane on the
// tile plus a 2-cell ring, F on the tile plus a 1-cell ring.
// Tile 32 x 16 with two output rows per thread (rows ty and ty + 8, 256
// threads): the per-plane barriers, ring bookkeeping and copy issue are
// shared by two points, and the psi / F loops run three rounds per thread
// (B200, 512^3 FP64: 2.61 -> 2.36 ms against one row per thread).
constexpr int PTY = 16;            // phase tile height
constexpr int PPT = 2;             // output rows per thread (rows ty + h*PTY/PPT)
constexpr int PNT = TX * PTY / PPT;  // phase threads per CTA
// Resident CTAs per SM the phase kernel is built for: 2 in FP64 (its FP64
// registers), 4 in FP32 (64 registers; 512^3: 1.57 -> 1.37 ms against 2).
template <class T> __host__ __device__ constexpr int phase_min_blocks() { return sizeof(T) == 4 ? 4 : 2; }

// Momentum ring depth (planes per field): planes m-2 .. m+1, one in flight.
// (A 5-plane ring with two planes in flight measured 30% slower on B200 at
// 512^3: it leaves fewer CTAs per SM.)
__host__ __device__ constexpr int momentum_ring(int) { return 4; }
// Resident CTAs per SM the momentum kernel is built for: what its shared
// memory allows with ACDI (3 with 8-row tiles), 4 without; registers follow.
// FP32 16-row tiles: 3 (80 registers, no spill; 1.73 -> 1.62 ms at 512^3 on
// B200 against 2), FP64 16-row tiles 2 (128 registers).
template <class T> __host__ __device__ constexpr int momentum_min_blocks(bool pf, int mty) {
  return mty == 8 ? (pf ? 3 : 4) : (sizeof(T) == 4 ? 3 : 2);
}

// Staged-plane geometry of the momentum kernel.  A staged plane is a box of
// cells whose first column lies XS cells left of the tile, XS cells being 16
// bytes, so that a tensor-map box load starts on a 16-byte boundary: UX x UY
// cells for the velocities (the tile and its 1-cell ring), EX x EY for phi
// (2-cell ring), widths rounded up to 16 bytes.  Ring slots are 128-byte
// multiples; the slot barriers follow the force ring.
template <class T, int TYv> struct MomGeo {
  static constexpr int XS = 16 / (int)sizeof(T);
  static constexpr int AL = 128 / (int)sizeof(T);
  static constexpr int UX = (XS + TX + 1 + XS - 1) / XS * XS, UY = TYv + 2, UE = UX * UY;
  static constexpr int EX = (XS + TX + 2 + XS - 1) / XS * XS, EY = TYv + 4, PE = EX * EY;
  static constexpr int USL = (UE + AL - 1) / AL * AL, PSL = (PE + AL - 1) / AL * AL;
  static constexpr int QE = (TX + 1) * (TYv + 1);
  static __host__ __device__ constexpr size_t bar_offset(bool pf, int ns) {
    return ((sizeof(T) * (3 * ns * USL + (pf ? ns * PSL + 6 * QE : 0))) + 7) / 8 * 8;
  }
  static __host__ __device__ constexpr unsigned tx_bytes(bool pf) {
    return (unsigned)(sizeof(T) * (3 * UE + (pf ? PE : 0)));
  }
  // every box of the tile inside the n x n plane
  static __host__ __device__ bool interior(int x0, int y0, int n, bool pf) {
    const int bw = UX > EX ? UX : EX, r = pf ? 2 : 1;
    return x0 >= XS && x0 - XS + bw <= n && y0 >= r && y0 + TYv + r <= n;
  }
};
static_assert(MomGeo<double, 8>::UX == 36 && MomGeo<double, 8>::EX == 36, "FP64 staged box widths");
static_assert(MomGeo<float, 16>::UX == 40 && MomGeo<float, 16>::EX == 40, "FP32 staged box widths");

// Staged phi planes of the phase kernel: the tile and its 2-cell ring in a
// box starting XS cells (16 bytes) left of the tile, row pitch EX.
template <class T> struct PhaseGeo {
  static constexpr int XS = 16 / (int)sizeof(T);
  static constexpr int EX = (XS + TX + 2 + XS - 1) / XS * XS, EY = PTY + 4;
  static constexpr int AL = 128 / (int)sizeof(T);
  static constexpr int PSL = (EX * EY + AL - 1) / AL * AL;
  static __host__ __device__ constexpr unsigned tx_bytes() { return (unsigned)(sizeof(T) * EX * EY); }
  static __host__ __device__ bool interior(int x0, int y0, int n) {
    return x0 >= XS && x0 - XS + EX <= n && y0 >= 2 && y0 + PTY + 2 <= n;
  }
};
static_assert(PhaseGeo<double>::EX == 36 && PhaseGeo<float>::EX == 40, "staged phi box widths");


// 1/(sqrt(s) + tiny) for s > 0, the normalisation of A5.  With r = rsqrt(s),
// 1/(sqrt(s) + tiny) = r/(1 + tiny*r) = r - tiny*r^2 + r*O((tiny*r)^2); the
// first-order form is used while tiny*r < 2^-30, where the dropped term is
// below 2^-60 r (far under an ulp), and the direct formula otherwise.
template <class T>
__device__ __forceinline__ T inv_norm_plus(T s, T tiny) {
  const T r = rsqrt(s);
  const T tr = tiny * r;
  if (tr < (T)9.3e-10) return fma(-tr, r, r);
  return (T)1 / (sqrt(s) + tiny);
}

// phimap: a __grid_constant__ parameter (single simulation), or a map in the
// ensemble's slot table (gmaps: acquired through the tensor-map proxy first).
template <class T, bool TMA>
__device__ __forceinline__ void phase_body(const StencilArgs<T>& a, int KZ, int bx, int by, int bz,
                                           const CUtensorMap* __restrict__ phimap, bool gmaps) {
  if (a.ctrl->status) return;
  constexpr int TY = PTY, NT = PNT;
  // The psi ring covers the tile and its 2-cell ring (LX x EY cells); phi and
  // psi planes are stored with row pitch EX and the ring's first column at
  // OFF (the staged phi box starts XS cells left of the tile, 16 bytes).
  typedef PhaseGeo<T> PG;
  constexpr int LX = TX + 4, EY = TY + 4, PE = LX * EY, EX = PG::EX, OFF = PG::XS - 2, SL = PG::PSL;
  constexpr int FX = TX + 2, FY = TY + 2, FE = FX * FY;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* s_phi = reinterpret_cast<T*>(smem_raw);  // ring of 5 planes
  T* s_psi = s_phi + 5 * SL;                  // ring of 3 planes
  T* s_F = s_psi + 3 * SL;                    // ring of 3 planes x 3 components
  double* s_tab = reinterpret_cast<double*>(s_F + 9 * FE);  // log table (FP64)
  unsigned long long* s_bar = reinterpret_cast<unsigned long long*>(s_tab + PsiMath<T>::TAB);
  for (int q = threadIdx.x; q < PsiMath<T>::TAB; q += NT) s_tab[q] = g_log_table[q];
  if (PsiMath<T>::TAB) __syncthreads();
  const int n = a.c.n;
  const T eps = (T)a.c.eps, epsi = (T)a.c.epsi, enumv = (T)a.c.enumv, tiny = (T)a.c.tiny;
  const T dxi = (T)a.c.dxi, ddxi = (T)a.c.ddxi, dt = (T)a.c.dt, hdxi = (T)0.5 * dxi;
  const T gamma = (T)(1.0 * a.ctrl->gumax);  // multi/main.f90:362
  const T mu = (T)a.ctrl->mean[0], mv = (T)a.ctrl->mean[1], mw = (T)a.ctrl->mean[2];
  const int use_ident = a.c.tanh_identity;
  const T floor0 = a.c.phi_floor ? (T)0 : (T)-INFINITY;
  const T inv12e = (T)1 / ((T)1 + (T)2 * enumv);
  // psi where min(phi,1) is exactly 1 (drop interiors) or so small that both
  // val + enum == enum and 1 - val + enum == 1 - 0 + enum in floating point
  // (far field; the first implies the second, since it needs |val| below
  // half an ulp of enum, far under 2^-54): there the reference's expression
  // evaluates to psi1 / psi0 exactly, so those constants are computed once
  // and the log is skipped -- bitwise the same values.
  const T psi0 = eps * PsiMath<T>::log_ratio((T)0 + enumv, (T)1 - (T)0 + enumv, s_tab);
  const T psi1 = eps * PsiMath<T>::log_ratio((T)1 + enumv, (T)1 - (T)1 + enumv, s_tab);
  const int x0 = bx * TX, y0 = by * TY, k0 = bz * KZ;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  constexpr int RY = TY / PPT;  // row step between a thread's output rows
  const int i = x0 + tx;
  const int ip = (i + 1 == n) ? 0 : i + 1;
  const size_t nn = (size_t)n * n;
  // Each thread owns ring elements tid + r*NT of every plane (copy and psi)
  // and F elements tid + r*NT; their in-plane offsets are the same on every
  // plane, so they are computed once here.
  constexpr int NPE = (PE + NT - 1) / NT, NFE = (FE + NT - 1) / NT;
  int poff[NPE], fpe[NFE];
#pragma unroll
  for (int r = 0; r < NPE; ++r) {
    const int e = min(tid + r * NT, PE - 1);
    poff[r] = wrapi(x0 - 2 + e % LX, n) + n * wrapi(y0 - 2 + e / LX, n);
  }
#pragma unroll
  for (int r = 0; r < NFE; ++r) {
    const int e = min(tid + r * NT, FE - 1);
    fpe[r] = (e % FX + 1 + OFF) + (e / FX + 1) * EX;
  }
  // stored index of the thread's ring element r
  const auto pidx = [&](int r) {
    const int e = tid + r * NT;
    if constexpr (EX == LX && OFF == 0) return e;
    else return (e % LX + OFF) + (e / LX) * EX;
  };
  // Tiles whose staged phi box lies inside the grid load each plane with one
  // tensor-map box load; the edge tiles copy their elements with cp.async
  // and wrap.  Both fill the same stored cells.
  const bool tma = TMA && PG::interior(x0, y0, n);
  int sp = 3;              // ring slot of plane m at iteration m
  unsigned bar_phase = 0;  // bit s: parity of the next phase of slot s's barrier
  if (tma) {
    if (tid == 0) {
#pragma unroll
      for (int q = 0; q < 5; ++q) mbar_init(s_bar + q, 1);
      mbar_init_fence();
      if (gmaps) tensormap_acquire(phimap);
    }
    __syncthreads();
  }
  // Ring slots by role, rotated once per plane (no per-plane index
  // arithmetic): at iteration m the phi slots hold planes m-3 .. m+1 (m+1
  // still in flight), the psi slots m-2 .. m (m being written), and the F
  // slots m-3 .. m-1 (m-1 being written).
  T *Phm3 = s_phi, *Phm2 = s_phi + SL, *Phm1 = s_phi + 2 * SL, *Ph0 = s_phi + 3 * SL, *Php1 = s_phi + 4 * SL;
  T *PsW = s_psi, *Psm1 = s_psi + SL, *Psm2 = s_psi + 2 * SL;
  T *FW = s_F, *Fm2 = s_F + 3 * FE, *Fm3 = s_F + 6 * FE;
  int gij[PPT], gipj[PPT], gijp[PPT];
#pragma unroll
  for (int h = 0; h < PPT; ++h) {
    const int j = y0 + ty + h * RY, jp = (j + 1 == n) ? 0 : j + 1;
    gij[h] = i + n * j;
    gipj[h] = ip + n * j;
    gijp[h] = i + n * jp;
  }

  // phi plane m (2-cell ring) is copied into `dst` (ring slot `slot`) one
  // iteration ahead of its use.
  auto issue = [&](T* dst, int slot, int m) {
    if (tma) {
      if (tid == 0) {
        mbar_arrive_expect_tx(s_bar + slot, PG::tx_bytes());
        tma_load_2d(dst, phimap, x0 - PG::XS, wrapi(m, n) * n + y0 - 2, s_bar + slot);
      }
      return;
    }
    const T* src = a.phi_in + (size_t)wrapi(m, n) * nn;
#pragma unroll
    for (int r = 0; r < NPE; ++r) {
      const int e = tid + r * NT;
      if (r < NPE - 1 || e < PE) cp_async_elem(dst + pidx(r), src + poff[r]);
    }
    cp_async_commit();
  };
  issue(Ph0, sp, k0 - 2);
  for (int m = k0 - 2; m <= k0 + KZ + 1; ++m) {
    // plane m has landed: this thread's cp.async copies, or the slot's
    // barrier phase for the box load (a wait that gives up records a timeout
    // and carries on, so that no thread is left at a barrier)
    if (tma) {
      if (!mbar_wait(s_bar + sp, (bar_phase >> sp) & 1u, kWaitCycles)) atomicCAS(&a.ctrl->status, 0, kStatusTimeout);
      bar_phase ^= 1u << sp;
    } else {
      cp_async_wait<0>();
    }
    const int spn = sp == 4 ? 0 : sp + 1;  // slot of plane m+1
    // velocities of the output plane k = m-2, loaded now so that their latency
    // hides behind the psi and F work below
    T uc[PPT], uxp[PPT], vc[PPT], vyp[PPT], wc[PPT], wzp[PPT];
    if (m >= k0 + 2) {
      const size_t zo = nn * wrapi(m - 2, n), zop = nn * wrapi(m - 1, n);
#pragma unroll
      for (int h = 0; h < PPT; ++h) {
        uc[h] = a.u[zo + gij[h]];
        uxp[h] = a.u[zo + gipj[h]];
        vc[h] = a.v[zo + gij[h]];
        vyp[h] = a.v[zo + gijp[h]];
        wc[h] = a.w[zo + gij[h]];
        wzp[h] = a.w[zop + gij[h]];
      }
    }
    // (1) psi of plane m on the elements this thread copied.
#pragma unroll
    for (int r = 0; r < NPE; ++r) {
      const int e = tid + r * NT;
      if (r < NPE - 1 || e < PE) {
        const int ep = pidx(r);
        const T val = fmax(fmin(Ph0[ep], (T)1), floor0);
        PsW[ep] = (val + enumv == enumv) ? psi0
                 : ((val == (T)1) ? psi1 : eps * PsiMath<T>::log_ratio(val + enumv, (T)1 - val + enumv, s_tab));
      }
    }
    // psi of plane m is visible, and every thread is done with iteration m-1:
    // the phi slot plane m+1 reuses (plane m-4, read by the last output) is
    // free.  Two barriers per plane besides the F one, not three.
    __syncthreads();
    if (m + 1 <= k0 + KZ + 1) issue(Php1, spn, m + 1);
    else cp_async_commit();
    // (2) F on plane m-1 over the tile + 1 ring.
    if (m >= k0) {
      const T* Pc = Psm1;
      const T* Pm = Psm2;
      const T* Pp = PsW;
      const T* Phc = Phm1;
      T* F = FW;
#pragma unroll
      for (int r = 0; r < NFE; ++r) {
        const int e = tid + r * NT;
        if (r == NFE - 1 && e >= FE) break;
        const int pe = fpe[r];
        const T gxv = Pc[pe + 1] - Pc[pe - 1];
        const T gyv = Pc[pe + EX] - Pc[pe - EX];
        const T gzv = Pp[pe] - Pm[pe];
        if (gxv == (T)0 && gyv == (T)0 && gzv == (T)0) {  // uniform psi: n = 0 and F = 0 exactly
          F[e] = (T)0;
          F[FE + e] = (T)0;
          F[2 * FE + e] = (T)0;
          continue;
        }
        const T normod = inv_norm_plus(gxv * gxv + gyv * gyv + gzv * gzv, tiny);
        T t;
        if (use_ident) {
          // tanh(0.5*log(a/b)) = (a-b)/(a+b) with a = val+enum, b = 1-val+enum
          const T val = fmax(fmin(Phc[pe], (T)1), floor0);
          t = ((T)2 * val - (T)1) * inv12e;
        } else {
          t = tanh((T)0.5 * Pc[pe] * epsi);
        }
        const T g = (T)0.25 * ((T)1 - t * t);
        F[e] = g * (gxv * normod);
        F[FE + e] = g * (gyv * normod);
        F[2 * FE + e] = g * (gzv * normod);
      }
    }
    __syncthreads();
    // (3) output plane k = m-2.
    if (m >= k0 + 2) {
      const T* P0 = Phm2;
      const T* Pm1 = Phm3;
      const T* Pp1 = Phm1;
      const T* F0 = Fm2;
      const T* Fm = Fm3;
      const T* Fp = FW;
#pragma unroll
      for (int h = 0; h < PPT; ++h) {
        const int pe = (tx + 2 + OFF) + (ty + h * RY + 2) * EX;
        const int fe = (tx + 1) + (ty + h * RY + 1) * FX;
        const T c = P0[pe], pxp = P0[pe + 1], pxm = P0[pe - 1], pyp = P0[pe + EX], pym = P0[pe - EX];
        const T pzp = Pp1[pe], pzm = Pm1[pe];
        const size_t g = nn * wrapi(m - 2, n) + gij[h];
        const T uc_ = uc[h] - mu, uxp_ = uxp[h] - mu, vc_ = vc[h] - mv, vyp_ = vyp[h] - mv;
        const T wc_ = wc[h] - mw, wzp_ = wzp[h] - mw;
        // The factors 0.5 of the face averages and central differences are
        // folded into hdxi = 0.5*dxi: scaling by a power of 2 commutes with
        // rounding, so every term is bitwise the reference's (x*0.5*y - ..)*dxi.
        T r = -(uxp_ * (pxp + c) - uc_ * (c + pxm)) * hdxi - (vyp_ * (pyp + c) - vc_ * (c + pym)) * hdxi -
              (wzp_ * (pzp + c) - wc_ * (c + pzm)) * hdxi;
        r = r + gamma * (eps * (pxp - (T)2 * c + pxm) * ddxi + eps * (pyp - (T)2 * c + pym) * ddxi +
                         eps * (pzp - (T)2 * c + pzm) * ddxi);
        r = r - gamma * ((F0[fe + 1] - F0[fe - 1]) * hdxi + (F0[FE + fe + FX] - F0[FE + fe - FX]) * hdxi +
                         (Fp[2 * FE + fe] - Fm[2 * FE + fe]) * hdxi);
        a.phi_out[g] = c + dt * r;
      }
    }
    // rotate the rings for plane m+1: the slot of the oldest plane of each
    // ring takes the next plane
    T* t = Phm3;
    Phm3 = Phm2; Phm2 = Phm1; Phm1 = Ph0; Ph0 = Php1; Php1 = t;
    sp = spn;
    t = Psm2;
    Psm2 = Psm1; Psm1 = PsW; PsW = t;
    t = Fm3;
    Fm3 = Fm2; Fm2 = FW; FW = t;
  }
}

// ============================================================ momentum
// B1..B7 (multi/main.f90:513-682) fused: conservative convection, viscous
// term, ABC forcing, optional linear forcing A*u, surface tension
// f = 6 sigma chempot grad(phi) at cell centres interpolated to the faces,
// and the AB2 (Euler on the first step) predictor.  Writes ustar and the new
// rhs_o; reads the NEW phi (the reference computes B4 after A7).
// momentum tile height: 8 or 16 rows (a tuning choice per grid size)
template <class T, bool PF, int MTYv, bool TMA>
__device__ __forceinline__ void momentum_body(const StencilArgs<T>& a, int KZ, int bx, int by, int bz,
                                              const PlaneMaps* __restrict__ maps, bool gmaps) {
  if (a.ctrl->status) return;
  // MPT output rows per thread (rows ty + 8h): 256 threads for either tile
  constexpr int TY = MTYv, MPT = MTYv / 8, NT = TX * 8;
  typedef MomGeo<T, MTYv> G;
  constexpr int XS = G::XS, UX = G::UX, UE = G::UE, EX = G::EX, PE = G::PE;
  constexpr int QX = TX + 1, QY = TY + 1, QE = QX * QY;  // force over [-1,TX) x [-1,TY)
  // Ring of NS planes per field: planes m-2 .. m+PD at iteration m, the
  // last PD of them in flight.
  constexpr int NS = momentum_ring(MTYv), PD = NS - 3;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  T* s_u = reinterpret_cast<T*>(smem_raw);
  T* s_v = s_u + NS * G::USL;
  T* s_w = s_v + NS * G::USL;
  T* s_phi = s_w + NS * G::USL;  // PF only
  T* s_f = s_phi + NS * G::PSL;  // ring of 2 planes x 3 components (PF only)
  unsigned long long* s_bar = reinterpret_cast<unsigned long long*>(smem_raw + G::bar_offset(PF, NS));
  const int n = a.c.n;
  const T dxi = (T)a.c.dxi, ddxi = (T)a.c.ddxi, dt = (T)a.c.dt, mu_v = (T)a.c.mu, rhoi = (T)a.c.rhoi;
  const T eps = (T)a.c.eps, epsi = (T)a.c.epsi, sig6 = (T)(6.0 * a.c.sigma), lin = (T)a.c.lin_force;
  const T f1 = (T)a.c.f1, f2 = (T)a.c.f2, f3 = (T)a.c.f3;
  const T alpha = (T)a.ctrl->alpha, beta = (T)a.ctrl->beta;
  const T mu = (T)a.ctrl->mean[0], mv = (T)a.ctrl->mean[1], mw = (T)a.ctrl->mean[2];
  const int x0 = bx * TX, y0 = by * TY, k0 = bz * KZ;
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int i = x0 + tx;
  const size_t nn = (size_t)n * n;
  const T h = (T)0.5, q = (T)0.25;
  const T qdxi = q * dxi, hrhoi = h * rhoi;
  // Tiles whose staged boxes lie inside the grid (no periodic wrap) load
  // each plane with four tensor-map box loads issued by one thread; the
  // edge tiles copy the same boxes element-wise with cp.async and wrap.
  const bool tma = TMA && G::interior(x0, y0, n, PF);
  // Each thread owns elements tid + r*NT of the velocity, phi and force
  // planes; their in-plane offsets are the same on every plane.
  constexpr int NUE = (UE + NT - 1) / NT, NPE = (PE + NT - 1) / NT, NQE = (QE + NT - 1) / NT;
  int uoff[NUE], poff[NPE], qpe[NQE];
#pragma unroll
  for (int r = 0; r < NUE; ++r) {
    const int e = min(tid + r * NT, UE - 1);
    uoff[r] = wrapi(x0 - XS + e % UX, n) + n * wrapi(y0 - 1 + e / UX, n);
  }
#pragma unroll
  for (int r = 0; r < NPE; ++r) {
    const int e = min(tid + r * NT, PE - 1);
    poff[r] = PF ? wrapi(x0 - XS + e % EX, n) + n * wrapi(y0 - 2 + e / EX, n) : 0;
  }
#pragma unroll
  for (int r = 0; r < NQE; ++r) {
    const int e = min(tid + r * NT, QE - 1);
    qpe[r] = (e % QX + 1) + (e / QX + 1) * EX;
  }
  // sl[q] is the ring slot of plane m-2+q at iteration m; the roles rotate
  // once per plane.
  int sl[NS];
#pragma unroll
  for (int q2 = 0; q2 < NS; ++q2) sl[q2] = q2;
  unsigned bar_phase = 0;  // bit s: parity of the next phase of slot s's barrier
  if (tma) {
    if (tid == 0) {
#pragma unroll
      for (int q2 = 0; q2 < NS; ++q2) mbar_init(s_bar + q2, 1);
      mbar_init_fence();
      if (gmaps) {  // maps in the ensemble's slot table
        tensormap_acquire(&maps->u);
        tensormap_acquire(&maps->v);
        tensormap_acquire(&maps->w);
        if (PF) tensormap_acquire(&maps->phi);
      }
    }
    __syncthreads();
  }

  // Plane m of u, v, w (1-cell ring) and phi (2-cell ring) is copied into a
  // ring slot PD iterations ahead of its use, so the HBM latency of the
  // planes in flight overlaps the arithmetic of plane m-1.
  auto issue = [&](int slot, int m) {
    if (tma) {
      if (tid == 0) {
        const int yr = wrapi(m, n) * n;
        mbar_arrive_expect_tx(s_bar + slot, G::tx_bytes(PF));
        tma_load_2d(s_u + slot * G::USL, &maps->u, x0 - XS, yr + y0 - 1, s_bar + slot);
        tma_load_2d(s_v + slot * G::USL, &maps->v, x0 - XS, yr + y0 - 1, s_bar + slot);
        tma_load_2d(s_w + slot * G::USL, &maps->w, x0 - XS, yr + y0 - 1, s_bar + slot);
        if (PF) tma_load_2d(s_phi + slot * G::PSL, &maps->phi, x0 - XS, yr + y0 - 2, s_bar + slot);
      }
      return;
    }
    const size_t zoff = (size_t)wrapi(m, n) * nn;
    const T* su = a.u + zoff;
    const T* sv = a.v + zoff;
    const T* sw = a.w + zoff;
#pragma unroll
    for (int r = 0; r < NUE; ++r) {
      const int e = tid + r * NT;
      if (r < NUE - 1 || e < UE) {
        cp_async_elem(s_u + slot * G::USL + e, su + uoff[r]);
        cp_async_elem(s_v + slot * G::USL + e, sv + uoff[r]);
        cp_async_elem(s_w + slot * G::USL + e, sw + uoff[r]);
      }
    }
    if (PF) {
      const T* sp = a.phi_in + zoff;
#pragma unroll
      for (int r = 0; r < NPE; ++r) {
        const int e = tid + r * NT;
        if (r < NPE - 1 || e < PE) cp_async_elem(s_phi + slot * G::PSL + e, sp + poff[r]);
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int q2 = 0; q2 < PD; ++q2) issue(sl[2 + q2], k0 - 2 + q2);
  // registers carried from one output plane to the next (see below)
  T r_uc[MPT], r_uzp[MPT], r_uxp[MPT], r_vc[MPT], r_vzp[MPT], r_vyp[MPT], r_wc[MPT], r_wzp[MPT], r_wxmzp[MPT],
      r_wymzp[MPT];
  bool have_prev = false;
  for (int m = k0 - 2; m <= k0 + KZ; ++m) {
    // plane m has landed: this thread's cp.async copies, or the slot's
    // barrier phase for the box loads (a wait that gives up records a
    // timeout and carries on, so that no thread is left at a barrier)
    if (tma) {
      const int s = sl[2];
      if (!mbar_wait(s_bar + s, (bar_phase >> s) & 1u, kWaitCycles)) atomicCAS(&a.ctrl->status, 0, kStatusTimeout);
      bar_phase ^= 1u << s;
    } else {
      cp_async_wait<0>();
    }
    // rhs_o of the output plane k = m-1, loaded now so that its latency hides
    // behind the force computation below
    T ruo[MPT], rvo[MPT], rwo[MPT];
    if (m >= k0 + 1) {
#pragma unroll
      for (int hh = 0; hh < MPT; ++hh) {
        const size_t g = (size_t)i + (size_t)n * (y0 + ty + 8 * hh) + nn * wrapi(m - 1, n);
        ruo[hh] = a.ru[g];
        rvo[hh] = a.rv[g];
        rwo[hh] = a.rw[g];
      }
    }
    // plane m is visible, and every thread is done with iteration m-1, so the
    // slot plane m+PD reuses (plane m-3) is free: one barrier per plane fewer
    // than issuing the copy first (512^3: FP64 3.04 -> 2.98 ms, FP32 1.86 ->
    // 1.75 ms)
    __syncthreads();
    if (m + PD <= k0 + KZ) issue(sl[NS - 1], m + PD);
    else cp_async_commit();
    if (PF && m >= k0) {
      // B4: chempot, grad(phi), f at plane m-1 (multi/main.f90:617-623)
      const int fm = m - 1;
      // staged phi boxes start XS - 2 cells left of the ring
      const T* P0 = s_phi + sl[1] * G::PSL + (XS - 2);
      const T* Pm = s_phi + sl[0] * G::PSL + (XS - 2);
      const T* Pp = s_phi + sl[2] * G::PSL + (XS - 2);
      T* F = s_f + ((fm + 8) & 1) * 3 * QE;
#pragma unroll
      for (int r = 0; r < NQE; ++r) {
        const int e = tid + r * NT;
        if (r == NQE - 1 && e >= QE) break;
        const int pe = qpe[r];
        const T c = P0[pe], pxp = P0[pe + 1], pxm = P0[pe - 1], pyp = P0[pe + EX], pym = P0[pe - EX];
        const T pzp = Pp[pe], pzm = Pm[pe];
        const T chem = c * ((T)1 - c) * ((T)1 - (T)2 * c) * epsi -
                       eps * (pxp + pxm + pyp + pym + pzp + pzm - (T)6 * c) * ddxi;
        const T gx = h * (pxp - pxm) * dxi, gy = h * (pyp - pym) * dxi, gz = h * (pzp - pzm) * dxi;
        F[e] = sig6 * chem * gx;
        F[QE + e] = sig6 * chem * gy;
        F[2 * QE + e] = sig6 * chem * gz;
      }
    }
    if (PF) __syncthreads();
    if (m >= k0 + 1) {
      const int k = m - 1;
      // staged velocity boxes start XS - 1 cells left of the ring
      const T* U0 = s_u + sl[1] * G::USL + (XS - 1);
      const T* Um = s_u + sl[0] * G::USL + (XS - 1);
      const T* Up = s_u + sl[2] * G::USL + (XS - 1);
      const T* V0 = s_v + sl[1] * G::USL + (XS - 1);
      const T* Vm = s_v + sl[0] * G::USL + (XS - 1);
      const T* Vp = s_v + sl[2] * G::USL + (XS - 1);
      const T* W0 = s_w + sl[1] * G::USL + (XS - 1);
      const T* Wm = s_w + sl[0] * G::USL + (XS - 1);
      const T* Wp = s_w + sl[2] * G::USL + (XS - 1);
#pragma unroll
      for (int hh = 0; hh < MPT; ++hh) {
        const int j = y0 + ty + 8 * hh;
        const int e = (tx + 1) + (ty + 8 * hh + 1) * UX;
        // The pending mean removal is applied as values enter registers.  Values
        // of this thread's column at planes k-1 and k, and the x/y neighbours
        // the previous plane already loaded, come from the previous output
        // plane's registers (z-marching register blocking): 17 shared loads
        // per point instead of 27.
        T uc, uzm, uxpzm, vc, vzm, vypzm, wc, wzm, wxm, wym;
        if (have_prev) {
          uzm = r_uc[hh]; uc = r_uzp[hh]; uxpzm = r_uxp[hh];
          vzm = r_vc[hh]; vc = r_vzp[hh]; vypzm = r_vyp[hh];
          wzm = r_wc[hh]; wc = r_wzp[hh]; wxm = r_wxmzp[hh]; wym = r_wymzp[hh];
        } else {
          uc = U0[e] - mu; uzm = Um[e] - mu; uxpzm = Um[e + 1] - mu;
          vc = V0[e] - mv; vzm = Vm[e] - mv; vypzm = Vm[e + UX] - mv;
          wc = W0[e] - mw; wzm = Wm[e] - mw; wxm = W0[e - 1] - mw; wym = W0[e - UX] - mw;
        }
        const T uxp = U0[e + 1] - mu, uxm = U0[e - 1] - mu, uyp = U0[e + UX] - mu, uym = U0[e - UX] - mu;
        const T uzp = Up[e] - mu, uxpym = U0[e + 1 - UX] - mu;
        const T vxp = V0[e + 1] - mv, vxm = V0[e - 1] - mv, vyp = V0[e + UX] - mv, vym = V0[e - UX] - mv;
        const T vzp = Vp[e] - mv, vxmyp = V0[e - 1 + UX] - mv;
        const T wxp = W0[e + 1] - mw, wyp = W0[e + UX] - mw;
        const T wzp = Wp[e] - mw, wxmzp = Wp[e - 1] - mw, wymzp = Wp[e - UX] - mw;
        r_uc[hh] = uc; r_uzp[hh] = uzp; r_uxp[hh] = uxp;
        r_vc[hh] = vc; r_vzp[hh] = vzp; r_vyp[hh] = vyp;
        r_wc[hh] = wc; r_wzp[hh] = wzp; r_wxmzp[hh] = wxmzp; r_wymzp[hh] = wymzp;
        // B1 (multi/main.f90:527-549)
        T h11 = (uxp + uc) * (uxp + uc) - (uc + uxm) * (uc + uxm);
        T h12 = (uyp + uc) * (vyp + vxmyp) - (uc + uym) * (vc + vxm);
        T h13 = (uzp + uc) * (wzp + wxmzp) - (uc + uzm) * (wc + wxm);
        T h21 = (uxp + uxpym) * (vxp + vc) - (uc + uym) * (vc + vxm);
        T h22 = (vyp + vc) * (vyp + vc) - (vc + vym) * (vc + vym);
        T h23 = (wzp + wymzp) * (vzp + vc) - (wc + wym) * (vc + vzm);
        T h31 = (wxp + wc) * (uxp + uxpzm) - (wc + wxm) * (uc + uzm);
        T h32 = (vyp + vypzm) * (wyp + wc) - (vc + vzm) * (wc + wym);
        T h33 = (wzp + wc) * (wzp + wc) - (wc + wzm) * (wc + wzm);
        // (h * 0.25) * dxi == h * (0.25 * dxi) exactly: scaling by a power of 2
        h11 = h11 * qdxi; h12 = h12 * qdxi; h13 = h13 * qdxi;
        h21 = h21 * qdxi; h22 = h22 * qdxi; h23 = h23 * qdxi;
        h31 = h31 * qdxi; h32 = h32 * qdxi; h33 = h33 * qdxi;
        T ru = -(h11 + h12 + h13);
        T rv = -(h21 + h22 + h23);
        T rw = -(h31 + h32 + h33);
        // B2 (multi/main.f90:567-578)
        h11 = mu_v * (uxp - (T)2 * uc + uxm) * ddxi;
        h12 = mu_v * (uyp - (T)2 * uc + uym) * ddxi;
        h13 = mu_v * (uzp - (T)2 * uc + uzm) * ddxi;
        h21 = mu_v * (vxp - (T)2 * vc + vxm) * ddxi;
        h22 = mu_v * (vyp - (T)2 * vc + vym) * ddxi;
        h23 = mu_v * (vzp - (T)2 * vc + vzm) * ddxi;
        h31 = mu_v * (wxp - (T)2 * wc + wxm) * ddxi;
        h32 = mu_v * (wyp - (T)2 * wc + wym) * ddxi;
        h33 = mu_v * (wzp - (T)2 * wc + wzm) * ddxi;
        ru = ru + (h11 + h12 + h13) * rhoi;
        rv = rv + (h21 + h22 + h23) * rhoi;
        rw = rw + (h31 + h32 + h33) * rhoi;
        const int kz = wrapi(k, n);
        // B3 ABC forcing (multi/main.f90:591-593), global interior coordinates
        if (a.c.abc) {
          ru = ru + f3 * (T)a.fsin[kz] + f2 * (T)a.fcos[j];
          rv = rv + f1 * (T)a.fsin[i] + f3 * (T)a.fcos[kz];
          rw = rw + f2 * (T)a.fsin[j] + f1 * (T)a.fcos[i];
        }
        if (lin != (T)0) {  // linear forcing (extension)
          ru = ru + lin * uc;
          rv = rv + lin * vc;
          rw = rw + lin * wc;
        }
        if (PF) {  // B5 (multi/main.f90:652-654)
          const T* F0 = s_f + ((k + 8) & 1) * 3 * QE;
          const T* Fm = s_f + ((k + 7) & 1) * 3 * QE;
          const int qe = (tx + 1) + (ty + 8 * hh + 1) * QX;
          ru = ru + (F0[qe - 1] + F0[qe]) * hrhoi;  // == 0.5 * (..) * rhoi exactly
          rv = rv + (F0[QE + qe - QX] + F0[QE + qe]) * hrhoi;
          rw = rw + (Fm[2 * QE + qe] + F0[2 * QE + qe]) * hrhoi;
        }
        // B6, B7 (multi/main.f90:666-681)
        const size_t g = (size_t)i + (size_t)n * j + nn * kz;
        a.us[g] = uc + dt * (alpha * ru - beta * ruo[hh]);
        a.vs[g] = vc + dt * (alpha * rv - beta * rvo[hh]);
        a.ws[g] = wc + dt * (alpha * rw - beta * rwo[hh]);
        a.ru[g] = ru;
        a.rv[g] = rv;
        a.rw[g] = rw;
      }
      have_prev = true;
    }
    // rotate: the slot of plane m-2 takes plane m+PD+1 at the next iteration
    const int t = sl[0];
#pragma unroll
    for (int q2 = 0; q2 < NS - 1; ++q2) sl[q2] = sl[q2 + 1];
    sl[NS - 1] = t;
  }
}

// ============================================================ projection
// C2 + R1 (multi/main.f90:873-903): u = ustar - dt/rho*(p - p_m)*dxi, with the
// sums and maxima of the projected u, v, w reduced per CTA in FP64.
// z planes per projection CTA: 64 where n allows, else 32 or 16 (512^3:
// FP64 projection plus finalize 1.47 -> 1.41 ms against 16 planes, with a
// quarter of the partials to reduce; FP32 projection 1.85 -> 1.49 ms).  The
// FP64 loop takes it as a compile-time trip count (a run-time one measured
// 1.79 ms there).
__host__ __device__ constexpr int project_kz(int n) { return n % 64 == 0 ? 64 : (n % 32 == 0 ? 32 : 16); }

template <class T, int PKZ>
__device__ __forceinline__ void project_body(const StencilArgs<T>& a, int bx, int by, int bz, int gx, int gy) {
  if (a.ctrl->status) return;
  const int n = a.c.n;
  const T dtr = (T)a.c.dtr, dxi = (T)a.c.dxi;
  const int i = bx * TX + threadIdx.x % TX, j = by * TY + threadIdx.x / TX;
  const int k0 = bz * PKZ;
  const int im = i ? i - 1 : n - 1, jm = j ? j - 1 : n - 1;
  const size_t nn = (size_t)n * n;
  double su = 0, sv = 0, sw = 0;
  double xu = -INFINITY, xv = -INFINITY, xw = -INFINITY;
  T pprev = a.p[(size_t)i + (size_t)n * j + nn * wrapi(k0 - 1, n)];
#pragma unroll 4
  for (int k = k0; k < k0 + PKZ; ++k) {
    const size_t g = (size_t)i + (size_t)n * j + nn * k;
    const T pc = a.p[g];
    const T uo = a.us[g] - dtr * (pc - a.p[g - i + im]) * dxi;
    const T vo = a.vs[g] - dtr * (pc - a.p[g + (size_t)n * jm - (size_t)n * j]) * dxi;
    const T wo = a.ws[g] - dtr * (pc - pprev) * dxi;
    pprev = pc;
    a.uo[g] = uo;
    a.vo[g] = vo;
    a.wo[g] = wo;
    su += (double)uo;
    sv += (double)vo;
    sw += (double)wo;
    xu = fmax(xu, (double)uo);
    xv = fmax(xv, (double)vo);
    xw = fmax(xw, (double)wo);
    // NaN must not vanish in fmax: fold it into the sums too
    if (uo != uo || vo != vo || wo != wo) su = NAN;
  }
  // deterministic block reduction: xor-shuffle in warps, then warps in order
  double vals[6] = {su, sv, sw, xu, xv, xw};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < 3; ++t) vals[t] += __shfl_xor_sync(0xffffffffu, vals[t], o);
#pragma unroll
    for (int t = 3; t < 6; ++t) vals[t] = fmax(vals[t], __shfl_xor_sync(0xffffffffu, vals[t], o));
  }
  __shared__ double red[NT / 32][6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < 6; ++t) red[wid][t] = vals[t];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) r[t] = red[0][t];
    for (int w = 1; w < NT / 32; ++w) {
      for (int t = 0; t < 3; ++t) r[t] += red[w][t];
      for (int t = 3; t < 6; ++t) r[t] = fmax(r[t], red[w][t]);
    }
    const size_t b = (size_t)bx + (size_t)gx * (by + (size_t)gy * bz);
    for (int t = 0; t < 6; ++t) a.partials[b * 6 + t] = r[t];
  }
}

// ============================================================ projection (FP32 refine)
// FP32 refinement form of C2 + R1: the pressure is p = p0 + dp (first FP32
// solve plus the FP32 correction solve of the FP64 residual), the projection
// u = ustar - dt/rho*(p - p_m)*dxi is evaluated in FP64 and rounded to FP32
// only when stored, and the forward-difference divergence of the FP64
// projected field is reduced (max |div u|) before that rounding.
__device__ __forceinline__ void project_refine_body(const StencilArgs<float>& a, const float* __restrict__ dp, int bx,
                                                    int by, int bz, int gx, int gy) {
  if (a.ctrl->status) return;
  const int n = a.c.n;
  const double dtr = a.c.dtr, dxi = a.c.dxi;
  const int i = bx * TX + threadIdx.x % TX, j = by * TY + threadIdx.x / TX;
  const int pkz = project_kz(n), k0 = bz * pkz;
  const int im = i ? i - 1 : n - 1, jm = j ? j - 1 : n - 1;
  const int ip = (i + 1 == n) ? 0 : i + 1, jp = (j + 1 == n) ? 0 : j + 1;
  const size_t nn = (size_t)n * n;
  const float* p0 = a.p;
  auto P = [&](size_t g) { return (double)p0[g] + (double)dp[g]; };
  double su = 0, sv = 0, sw = 0, mdiv = 0;
  double xu = -INFINITY, xv = -INFINITY, xw = -INFINITY;
  const size_t col = (size_t)i + (size_t)n * j;
  double pm = P(col + nn * wrapi(k0 - 1, n));
  double pc = P(col + nn * k0);
  double wsc = (double)a.ws[col + nn * k0];
  for (int k = k0; k < k0 + pkz; ++k) {
    const size_t g = col + nn * k;
    const int kp = (k + 1 == n) ? 0 : k + 1;
    const size_t gzp = col + nn * kp;
    const double pn = P(gzp);
    const double wsn = (double)a.ws[gzp];
    const size_t gxm = g - i + im, gxp = g - i + ip;
    const size_t gym = g - (size_t)n * j + (size_t)n * jm, gyp = g - (size_t)n * j + (size_t)n * jp;
    const double uo = (double)a.us[g] - dtr * (pc - P(gxm)) * dxi;
    const double vo = (double)a.vs[g] - dtr * (pc - P(gym)) * dxi;
    const double wo = wsc - dtr * (pc - pm) * dxi;
    const double u1 = (double)a.us[gxp] - dtr * (P(gxp) - pc) * dxi;
    const double v1 = (double)a.vs[gyp] - dtr * (P(gyp) - pc) * dxi;
    const double w1 = wsn - dtr * (pn - pc) * dxi;
    const double div = ((u1 - uo) + (v1 - vo) + (w1 - wo)) * dxi;
    mdiv = fmax(mdiv, fabs(div));
    if (div != div) mdiv = NAN;
    a.uo[g] = (float)uo;
    a.vo[g] = (float)vo;
    a.wo[g] = (float)wo;
    su += uo;
    sv += vo;
    sw += wo;
    xu = fmax(xu, uo);
    xv = fmax(xv, vo);
    xw = fmax(xw, wo);
    if (uo != uo || vo != vo || wo != wo) su = NAN;
    pm = pc;
    pc = pn;
    wsc = wsn;
  }
  double vals[7] = {su, sv, sw, xu, xv, xw, mdiv};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < 3; ++t) vals[t] += __shfl_xor_sync(0xffffffffu, vals[t], o);
#pragma unroll
    for (int t = 3; t < 7; ++t) vals[t] = fmax(vals[t], __shfl_xor_sync(0xffffffffu, vals[t], o));
  }
  __shared__ double red[NT / 32][7];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int t = 0; t < 7; ++t) red[wid][t] = vals[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    double r[7];
    for (int t = 0; t < 7; ++t) r[t] = red[0][t];
    for (int w = 1; w < NT / 32; ++w) {
      for (int t = 0; t < 3; ++t) r[t] += red[w][t];
      for (int t = 3; t < 7; ++t) r[t] = fmax(r[t], red[w][t]);
    }
    const size_t b = (size_t)bx + (size_t)gx * (by + (size_t)gy * bz);
    for (int t = 0; t < 7; ++t) a.partials[b * 7 + t] = r[t];
  }
}

// ============================================================ divergence check (FP32 refine)
// On request, the max |div u| of the FP32 refinement form's FP64 projection
// u = ustar - dt/rho*(p - p_m)*dxi with p = p0 + dp, from the stored ustar,
// p0 and dp: the arithmetic of project_refine_body's divergence, so it
// measures the field the step projected before rounding it to FP32.  Maxima
// are order-independent: CTAs combine theirs with an integer atomicMax on the
// bit patterns of the (non-negative, or NaN) values.
__global__ void __launch_bounds__(NT) refine_div_kernel(StencilArgs<float> a, const float* __restrict__ dp,
                                                        unsigned long long* __restrict__ out) {
  const int n = a.c.n;
  const double dtr = a.c.dtr, dxi = a.c.dxi;
  const int i = blockIdx.x * TX + threadIdx.x % TX, j = blockIdx.y * TY + threadIdx.x / TX;
  const int pkz = project_kz(n), k0 = blockIdx.z * pkz;
  const int im = i ? i - 1 : n - 1, jm = j ? j - 1 : n - 1;
  const int ip = (i + 1 == n) ? 0 : i + 1, jp = (j + 1 == n) ? 0 : j + 1;
  const size_t nn = (size_t)n * n;
  const float* p0 = a.p;
  auto P = [&](size_t g) { return (double)p0[g] + (double)dp[g]; };
  double mdiv = 0;
  const size_t col = (size_t)i + (size_t)n * j;
  double pm = P(col + nn * wrapi(k0 - 1, n));
  double pc = P(col + nn * k0);
  double wsc = (double)a.ws[col + nn * k0];
  for (int k = k0; k < k0 + pkz; ++k) {
    const size_t g = col + nn * k;
    const size_t gzp = col + nn * ((k + 1 == n) ? 0 : k + 1);
    const double pn = P(gzp);
    const double wsn = (double)a.ws[gzp];
    const size_t gxm = g - i + im, gxp = g - i + ip;
    const size_t gym = g - (size_t)n * j + (size_t)n * jm, gyp = g - (size_t)n * j + (size_t)n * jp;
    const double uo = (double)a.us[g] - dtr * (pc - P(gxm)) * dxi;
    const double vo = (double)a.vs[g] - dtr * (pc - P(gym)) * dxi;
    const double wo = wsc - dtr * (pc - pm) * dxi;
    const double u1 = (double)a.us[gxp] - dtr * (P(gxp) - pc) * dxi;
    const double v1 = (double)a.vs[gyp] - dtr * (P(gyp) - pc) * dxi;
    const double w1 = wsn - dtr * (pn - pc) * dxi;
    const double div = ((u1 - uo) + (v1 - vo) + (w1 - wo)) * dxi;
    mdiv = fmax(mdiv, fabs(div));
    if (div != div) mdiv = NAN;
    pm = pc;
    pc = pn;
    wsc = wsn;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, mdiv, o);
    mdiv = (x != x) ? x : fmax(mdiv, x);
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(fabs(mdiv)));
}

cudaError_t launch_refine_divergence(const StencilArgs<float>& a, const float* dp, double* out, cudaStream_t st) {
  const int n = a.c.n;
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
  if (e) return e;
  dim3 grid(n / TX, n / TY, n / project_kz(n));
  refine_div_kernel<<<grid, NT, 0, st>>>(a, dp, reinterpret_cast<unsigned long long*>(out));
  return cudaGetLastError();
}

// ============================================================ finalize
// M1, C3, R2 and the CFL guard (multi/main.f90:906-946), one CTA:
// means = sum/nx/ny/nz, removed lazily (stored in ctrl->mean and subtracted by
// every reader of u, v, w); gumax = max(max(u)-um, max(v)-vm, max(w)-wm), which
// equals the reference's max of the mean-removed fields because rounding is
// monotonic; then gamma, CFL, AB2 switch and the sticky error status.
constexpr int FNT = 1024;

// Partials hold `stride` values per CTA: sums of u, v, w, maxima of u, v, w,
// and (stride 7, FP32 refine form) the max |div u| of the FP64 projection.
__device__ __forceinline__ void finalize_body(const double* __restrict__ partials, int nparts, int stride, Ctrl* ctrl,
                                              const StepConst& c) {
  if (ctrl->status) return;
  double v[7] = {0, 0, 0, -INFINITY, -INFINITY, -INFINITY, 0};
  for (int b = threadIdx.x; b < nparts; b += FNT) {
    for (int t = 0; t < 3; ++t) v[t] += partials[(size_t)b * stride + t];
    for (int t = 3; t < stride; ++t) v[t] = fmax(v[t], partials[(size_t)b * stride + t]);
  }
  __shared__ double red[FNT / 32][7];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    for (int t = 0; t < 3; ++t) v[t] += __shfl_xor_sync(0xffffffffu, v[t], o);
    for (int t = 3; t < 7; ++t) v[t] = fmax(v[t], __shfl_xor_sync(0xffffffffu, v[t], o));
  }
  if ((threadIdx.x & 31) == 0)
    for (int t = 0; t < 7; ++t) red[threadIdx.x >> 5][t] = v[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < FNT / 32; ++w) {
      for (int t = 0; t < 3; ++t) red[0][t] += red[w][t];
      for (int t = 3; t < 7; ++t) red[0][t] = fmax(red[0][t], red[w][t]);
    }
  }
  if (threadIdx.x == 0) {
    const double nd = (double)c.n;
    const double um = red[0][0] / nd / nd / nd;
    const double vm = red[0][1] / nd / nd / nd;
    const double wm = red[0][2] / nd / nd / nd;
    const double uc = red[0][3] - um, vc = red[0][4] - vm, wc = red[0][5] - wm;
    const double umax = fmax(wc, fmax(uc, vc));
    const double cou = umax * c.dt * c.dxi;
    ctrl->mean[0] = um;
    ctrl->mean[1] = vm;
    ctrl->mean[2] = wm;
    ctrl->last_mean[0] = um;
    ctrl->last_mean[1] = vm;
    ctrl->last_mean[2] = wm;
    ctrl->gumax = umax;
    ctrl->cfl = cou;
    ctrl->alpha = 1.5;
    ctrl->beta = 0.5;
    ctrl->max_div = (stride > 6) ? red[0][6] : -1.0;
    ctrl->nstep += 1;
    const double s = red[0][0] + red[0][1] + red[0][2];
    if (!isfinite(s) || !isfinite(umax)) ctrl->status = 5;  // MHIT_ERR_NONFINITE
    else if (cou > ctrl->cfl_limit) ctrl->status = 4;      // MHIT_ERR_CFL
  }
}

// ============================================================ entry points
// Single simulation: block coordinates are the grid's.
template <class T>
__global__ void __launch_bounds__(PNT, phase_min_blocks<T>())
    phase_kernel(StencilArgs<T> a, int KZ, const __grid_constant__ CUtensorMap phimap) {
  phase_body<T, true>(a, KZ, blockIdx.x, blockIdx.y, blockIdx.z, &phimap, false);
}
template <class T, bool PF, int MTYv>
__global__ void __launch_bounds__(TX * 8, momentum_min_blocks<T>(PF, MTYv))
    momentum_kernel(StencilArgs<T> a, int KZ, const __grid_constant__ PlaneMaps maps) {
  momentum_body<T, PF, MTYv, true>(a, KZ, blockIdx.x, blockIdx.y, blockIdx.z, &maps, false);
}
template <class T, int PKZ>
__global__ void __launch_bounds__(NT, 4) project_kernel(StencilArgs<T> a) {
  project_body<T, PKZ>(a, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
}
__global__ void __launch_bounds__(NT) project_refine_kernel(StencilArgs<float> a, const float* __restrict__ dp) {
  project_refine_body(a, dp, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y);
}
__global__ void __launch_bounds__(FNT) finalize_kernel(const double* __restrict__ partials, int nparts, int stride,
                                                       Ctrl* ctrl, StepConst c) {
  finalize_body(partials, nparts, stride, ctrl, c);
}

// Batched over the slots of a served ensemble: grid z (x for finalize)
// covers the slots; each slot runs exactly the arithmetic of a single
// simulation, so a result is the same alone and in any mix.
template <class T>
__global__ void __launch_bounds__(PNT, phase_min_blocks<T>()) phase_kernel_b(const SlotArgs<T>* __restrict__ slots, int KZ,
                                                                            int zch) {
  const int sl = blockIdx.z / zch;
  if (!slots[sl].active) return;
  StencilArgs<T> a = slots[sl].st;
  const int par = (int)(a.ctrl->nstep & 1);
  a.phi_in = slots[sl].phi[par];
  a.phi_out = slots[sl].phi[par ^ 1];
  phase_body<T, true>(a, KZ, blockIdx.x, blockIdx.y, blockIdx.z - sl * zch, &slots[sl].maps.phase_phi[par], true);
}
template <class T, bool PF, int MTYv>
__global__ void __launch_bounds__(TX * 8, momentum_min_blocks<T>(PF, MTYv)) momentum_kernel_b(const SlotArgs<T>* __restrict__ slots, int KZ,
                                                                         int zch) {
  const int sl = blockIdx.z / zch;
  if (!slots[sl].active) return;
  StencilArgs<T> a = slots[sl].st;
  const int par = (int)((a.ctrl->nstep + 1) & 1);
  if (PF) a.phi_in = slots[sl].phi[par];  // the updated phi
  momentum_body<T, PF, MTYv, true>(a, KZ, blockIdx.x, blockIdx.y, blockIdx.z - sl * zch,
                                   &slots[sl].maps.mom[MTYv == 16 ? 1 : 0][par], true);
}
template <class T, int PKZ>
__global__ void __launch_bounds__(NT, 4) project_kernel_b(const SlotArgs<T>* __restrict__ slots, int zch) {
  const int sl = blockIdx.z / zch;
  if (!slots[sl].active) return;
  project_body<T, PKZ>(slots[sl].st, blockIdx.x, blockIdx.y, blockIdx.z - sl * zch, gridDim.x, gridDim.y);
}
__global__ void __launch_bounds__(NT) project_refine_kernel_b(const SlotArgs<float>* __restrict__ slots, int zch) {
  const int sl = blockIdx.z / zch;
  if (!slots[sl].active) return;
  project_refine_body(slots[sl].st, slots[sl].dp, blockIdx.x, blockIdx.y, blockIdx.z - sl * zch, gridDim.x,
                      gridDim.y);
}
template <class T>
__global__ void __launch_bounds__(FNT) finalize_kernel_b(const SlotArgs<T>* __restrict__ slots, int nparts, int stride) {
  const int sl = blockIdx.x;
  if (!slots[sl].active) return;
  finalize_body(slots[sl].st.partials, nparts, stride, slots[sl].st.ctrl, slots[sl].st.c);
}

// Self-check of the bounded slot-barrier wait the staged-plane kernels use:
// one warp arms a barrier; if `arrive`, a thread arrives on it, otherwise
// nothing does and the wait gives up after `limit` cycles.  Writes 0 or the
// timeout status; the kernel returns either way.
__global__ void wait_check_kernel(int arrive, long long limit, int* out) {
  __shared__ unsigned long long bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
  const bool ok = mbar_wait(&bar, 0, limit);
  __syncwarp();
  if (threadIdx.x == 0) *out = ok ? 0 : kStatusTimeout;
}

// u -= mean in place, then mean = 0 (materialises the lazy mean removal).
template <class T>
__global__ void materialize_kernel(T* u, T* v, T* w, size_t count, Ctrl* ctrl) {
  const T mu = (T)ctrl->mean[0], mv = (T)ctrl->mean[1], mw = (T)ctrl->mean[2];
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
    u[g] = u[g] - mu;
    v[g] = v[g] - mv;
    w[g] = w[g] - mw;
  }
}

__global__ void clear_mean_kernel(Ctrl* ctrl) {
  ctrl->mean[0] = 0;
  ctrl->mean[1] = 0;
  ctrl->mean[2] = 0;
}

// ============================================================ launchers
template <class T> static size_t phase_smem() {
  return sizeof(T) * (size_t)(8 * PhaseGeo<T>::PSL + 9 * (TX + 2) * (PTY + 2)) +
         sizeof(double) * (PsiMath<T>::TAB + 5);
}
template <class T> static size_t momentum_smem(bool pf, int mty) {
  const int ns = momentum_ring(mty);
  const size_t b = mty == 8 ? MomGeo<T, 8>::bar_offset(pf, ns) : MomGeo<T, 16>::bar_offset(pf, ns);
  return b + sizeof(unsigned long long) * ns;
}

// cuTensorMapEncodeTiled from the driver, resolved once through the runtime
// (no link-time dependency on the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

cudaError_t encode_tensor_map(CUtensorMap* m, int rank, const void* base, const uint64_t* dims,
                              const uint64_t* strides, const uint32_t* box, int elem_bytes) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return cudaErrorNotSupported;
  if (rank < 1 || rank > 3) return cudaErrorInvalidValue;
  cuuint64_t d[3], sb[2];
  cuuint32_t bx[3], estr[3] = {1, 1, 1};
  for (int i = 0; i < rank; ++i) {
    d[i] = dims[i];
    bx[i] = box[i];
    if (i + 1 < rank) sb[i] = strides[i];
  }
  const CUresult r = fn(m, elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void*>(base), d, sb, bx, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// 2D map of an n^3 field as n columns by n*n rows, box bw x bh.
template <class T> static cudaError_t plane_map(CUtensorMap* m, const T* base, int n, int bw, int bh) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return cudaErrorNotSupported;
  const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n * n};
  const cuuint64_t strides[1] = {(cuuint64_t)n * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<T*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <class T, int TYv> static cudaError_t momentum_maps(PlaneMaps* pm, const StencilArgs<T>& a, bool pf) {
  typedef MomGeo<T, TYv> G;
  const int n = a.c.n;
  cudaError_t e;
  if ((e = plane_map(&pm->u, a.u, n, G::UX, G::UY))) return e;
  if ((e = plane_map(&pm->v, a.v, n, G::UX, G::UY))) return e;
  if ((e = plane_map(&pm->w, a.w, n, G::UX, G::UY))) return e;
  if (pf && (e = plane_map(&pm->phi, a.phi_in, n, G::EX, G::EY))) return e;
  return cudaSuccess;
}

// A served-ensemble slot's tensor maps: the momentum boxes for both tile
// heights and both phi parities, the phase kernel's phi box per parity, and
// the column passes' spectrum views.
template <class T> cudaError_t encode_slot_maps(SlotArgs<T>* s, int n, bool pf) {
  cudaError_t e;
  StencilArgs<T> a = s->st;
  a.c.n = n;
  for (int par = 0; par < 2; ++par) {
    a.phi_in = pf ? s->phi[par] : nullptr;
    if ((e = momentum_maps<T, 8>(&s->maps.mom[0][par], a, pf))) return e;
    if ((e = momentum_maps<T, 16>(&s->maps.mom[1][par], a, pf))) return e;
    if (pf && (e = plane_map(&s->maps.phase_phi[par], s->phi[par], n, PhaseGeo<T>::EX, PTY + 4))) return e;
  }
  return encode_column_maps<T>(&s->maps, s->po.spec, n);
}
template cudaError_t encode_slot_maps<double>(SlotArgs<double>*, int, bool);
template cudaError_t encode_slot_maps<float>(SlotArgs<float>*, int, bool);

int stencil_size_ok(int n) {
  return n >= 32 && n % TX == 0 && n % TY == 0 && n % PTY == 0 && n % project_kz(n) == 0 && n % pick_kz(n) == 0;
}

int project_partials(int n) { return (n / TX) * (n / TY) * (n / project_kz(n)); }

template <class T> static cudaError_t prep_t() {
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(phase_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)phase_smem<T>())))
    return e;
  const void* mk[8] = {(const void*)momentum_kernel<T, true, 8>, (const void*)momentum_kernel<T, false, 8>,
                       (const void*)momentum_kernel<T, true, 16>, (const void*)momentum_kernel<T, false, 16>,
                       (const void*)momentum_kernel_b<T, true, 8>, (const void*)momentum_kernel_b<T, false, 8>,
                       (const void*)momentum_kernel_b<T, true, 16>, (const void*)momentum_kernel_b<T, false, 16>};
  for (int q = 0; q < 8; ++q) {
    const bool pf = (q % 2) == 0;
    const int mty = ((q / 2) % 2) ? 16 : 8;
    if ((e = cudaFuncSetAttribute(mk[q], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)momentum_smem<T>(pf, mty))))
      return e;
  }
  if ((e = cudaFuncSetAttribute(phase_kernel_b<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)phase_smem<T>())))
    return e;
  return cudaSuccess;
}

cudaError_t prepare_stencils() {
  cudaError_t e = upload_log_table();
  if (e) return e;
  e = prep_t<double>();
  if (e) return e;
  return prep_t<float>();
}

template <class T> cudaError_t launch_phase(const StencilArgs<T>& a, cudaStream_t st, int kz) {
  const int n = a.c.n;
  if (kz <= 0) kz = pick_kz(n);
  dim3 grid(n / TX, n / PTY, n / kz);
  CUtensorMap pm;
  cudaError_t e = plane_map(&pm, a.phi_in, n, PhaseGeo<T>::EX, PTY + 4);
  if (e) return e;
  phase_kernel<T><<<grid, PNT, phase_smem<T>(), st>>>(a, kz, pm);
  return cudaGetLastError();
}

template <class T> cudaError_t launch_momentum(const StencilArgs<T>& a, bool pf, cudaStream_t st, int kz, int mty) {
  const int n = a.c.n;
  if (kz <= 0) kz = pick_kz(n);
  if (mty != 8) mty = 16;
  dim3 grid(n / TX, n / mty, n / kz);
  const size_t sm = momentum_smem<T>(pf, mty);
  PlaneMaps pm;
  memset(&pm, 0, sizeof(pm));
  cudaError_t e = mty == 8 ? momentum_maps<T, 8>(&pm, a, pf) : momentum_maps<T, 16>(&pm, a, pf);
  if (e) return e;
  if (mty == 8) {
    if (pf) momentum_kernel<T, true, 8><<<grid, TX * 8, sm, st>>>(a, kz, pm);
    else momentum_kernel<T, false, 8><<<grid, TX * 8, sm, st>>>(a, kz, pm);
  } else {
    if (pf) momentum_kernel<T, true, 16><<<grid, TX * 8, sm, st>>>(a, kz, pm);
    else momentum_kernel<T, false, 16><<<grid, TX * 8, sm, st>>>(a, kz, pm);
  }
  return cudaGetLastError();
}

template <class T> cudaError_t launch_project(const StencilArgs<T>& a, cudaStream_t st) {
  const int n = a.c.n;
  dim3 grid(n / TX, n / TY, n / project_kz(n));
  switch (project_kz(n)) {
    case 64: project_kernel<T, 64><<<grid, NT, 0, st>>>(a); break;
    case 32: project_kernel<T, 32><<<grid, NT, 0, st>>>(a); break;
    default: project_kernel<T, 16><<<grid, NT, 0, st>>>(a); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_project_refine(const StencilArgs<float>& a, const float* dp, cudaStream_t st) {
  const int n = a.c.n;
  dim3 grid(n / TX, n / TY, n / project_kz(n));
  project_refine_kernel<<<grid, NT, 0, st>>>(a, dp);
  return cudaGetLastError();
}

int project_refine_partials(int n) { return project_partials(n); }

cudaError_t launch_finalize(const double* partials, int nparts, int stride, Ctrl* ctrl, StepConst c,
                            cudaStream_t st) {
  finalize_kernel<<<1, FNT, 0, st>>>(partials, nparts, stride, ctrl, c);
  return cudaGetLastError();
}

template <class T> cudaError_t launch_materialize(T* u, T* v, T* w, int n, Ctrl* ctrl, cudaStream_t st) {
  const size_t count = (size_t)n * n * n;
  materialize_kernel<T><<<1184, 256, 0, st>>>(u, v, w, count, ctrl);
  clear_mean_kernel<<<1, 1, 0, st>>>(ctrl);
  return cudaGetLastError();
}

int stencil_kz_ok(int n, int kz) { return kz >= 2 && kz <= n && n % kz == 0; }

cudaError_t launch_wait_check(int arrive, long long limit_cycles, int* out_dev, cudaStream_t st) {
  wait_check_kernel<<<1, 32, 0, st>>>(arrive, limit_cycles, out_dev);
  return cudaGetLastError();
}

template <class T>
cudaError_t launch_phase_batched(const SlotArgs<T>* slots, int nslots, int n, int kz, cudaStream_t st) {
  dim3 grid(n / TX, n / PTY, (n / kz) * nslots);
  phase_kernel_b<T><<<grid, PNT, phase_smem<T>(), st>>>(slots, kz, n / kz);
  return cudaGetLastError();
}
template <class T>
cudaError_t launch_momentum_batched(const SlotArgs<T>* slots, int nslots, int n, int kz, bool pf, cudaStream_t st,
                                   int mty) {
  if (mty != 8) mty = 16;
  dim3 grid(n / TX, n / mty, (n / kz) * nslots);
  const size_t sm = momentum_smem<T>(pf, mty);
  if (mty == 8) {
    if (pf) momentum_kernel_b<T, true, 8><<<grid, TX * 8, sm, st>>>(slots, kz, n / kz);
    else momentum_kernel_b<T, false, 8><<<grid, TX * 8, sm, st>>>(slots, kz, n / kz);
  } else {
    if (pf) momentum_kernel_b<T, true, 16><<<grid, TX * 8, sm, st>>>(slots, kz, n / kz);
    else momentum_kernel_b<T, false, 16><<<grid, TX * 8, sm, st>>>(slots, kz, n / kz);
  }
  return cudaGetLastError();
}
template <class T>
cudaError_t launch_project_batched(const SlotArgs<T>* slots, int nslots, int n, cudaStream_t st) {
  dim3 grid(n / TX, n / TY, (n / project_kz(n)) * nslots);
  if constexpr (sizeof(T) == 8) {
    switch (project_kz(n)) {
      case 64: project_kernel_b<T, 64><<<grid, NT, 0, st>>>(slots, n / project_kz(n)); break;
      case 32: project_kernel_b<T, 32><<<grid, NT, 0, st>>>(slots, n / project_kz(n)); break;
      default: project_kernel_b<T, 16><<<grid, NT, 0, st>>>(slots, n / project_kz(n)); break;
    }
  } else
    project_refine_kernel_b<<<grid, NT, 0, st>>>(slots, n / project_kz(n));
  return cudaGetLastError();
}
template cudaError_t launch_project_batched<double>(const SlotArgs<double>*, int, int, cudaStream_t);
template cudaError_t launch_project_batched<float>(const SlotArgs<float>*, int, int, cudaStream_t);
cudaError_t launch_finalize_batched(const SlotArgs<double>* slots, int nslots, int n, cudaStream_t st) {
  finalize_kernel_b<double><<<nslots, FNT, 0, st>>>(slots, step_partials_fp64(n), 6);
  return cudaGetLastError();
}
cudaError_t launch_finalize_batched_f32(const SlotArgs<float>* slots, int nslots, int n, cudaStream_t st) {
  if (fused_projection(n))  // fused x inverse + projection: 6 values per CTA, no divergence
    finalize_kernel_b<float><<<nslots, FNT, 0, st>>>(slots, xinv_project_partials(n), 6);
  else
    finalize_kernel_b<float><<<nslots, FNT, 0, st>>>(slots, project_partials(n), 7);
  return cudaGetLastError();
}
template cudaError_t launch_phase_batched<double>(const SlotArgs<double>*, int, int, int, cudaStream_t);
template cudaError_t launch_phase_batched<float>(const SlotArgs<float>*, int, int, int, cudaStream_t);
template cudaError_t launch_momentum_batched<double>(const SlotArgs<double>*, int, int, int, bool, cudaStream_t, int);
template cudaError_t launch_momentum_batched<float>(const SlotArgs<float>*, int, int, int, bool, cudaStream_t, int);

template cudaError_t launch_phase<double>(const StencilArgs<double>&, cudaStream_t, int);
template cudaError_t launch_phase<float>(const StencilArgs<float>&, cudaStream_t, int);
template cudaError_t launch_momentum<double>(const StencilArgs<double>&, bool, cudaStream_t, int, int);
template cudaError_t launch_momentum<float>(const StencilArgs<float>&, bool, cudaStream_t, int, int);
template cudaError_t launch_project<double>(const StencilArgs<double>&, cudaStream_t);
template cudaError_t launch_project<float>(const StencilArgs<float>&, cudaStream_t);
template cudaError_t launch_materialize<double>(double*, double*, double*, int, Ctrl*, cudaStream_t);
template cudaError_t launch_materialize<float>(float*, float*, float*, int, Ctrl*, cudaStream_t);

}  // namespace mhit
