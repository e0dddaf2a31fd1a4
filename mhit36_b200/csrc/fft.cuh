// FFT building blocks of libmhit: radix-2/3/4/8 butterflies and the
// register-resident line transform (reg_fft_stages) that every x, y and z
// pass of the Poisson solve uses.
//
// The transform is the Stockham autosort formulation (natural-order output):
// for each stage with radix R and span Ns,
//   v[r] = x[j + r*N/R] * w_N^(DIR * r*(j mod Ns)*N/(Ns*R)),  v = DFT_R(v),
//   x'[(j/Ns)*Ns*R + (j mod Ns) + r*Ns] = v[r].
// DIR = -1 is the forward transform e^{-2 pi i jk/N} (cuFFT's
// CUFFT_FORWARD, used by the reference at multi/main.f90:750-761), DIR = +1
// the unnormalised inverse (multi/main.f90:802-812).  Twiddles come from a
// table tw[m] = e^{-2 pi i m/N} computed on the host in long double.
#pragma once
#include "common.cuh"

namespace mhit {

template <int R, int DIR, class C> struct DFT;

template <int DIR, class C> struct DFT<2, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <int DIR, class C> __device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = cmul_i<DIR>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <int DIR, class C> struct DFT<4, DIR, C> {
  static __device__ __forceinline__ void run(C* v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }
};

template <int DIR, class C> struct DFT<8, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    typedef decltype(v[0].x) T;
    const T h = (T)0.70710678118654752440084436210484903928;
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    // w8^1 = h(1 + DIR i), w8^2 = DIR i, w8^3 = h(-1 + DIR i)
    C t1, t3;
    t1.x = h * (o1.x - (T)DIR * o1.y);
    t1.y = h * (o1.y + (T)DIR * o1.x);
    C t2 = cmul_i<DIR>(o2);
    t3.x = h * (-o3.x - (T)DIR * o3.y);
    t3.y = h * (-o3.y + (T)DIR * o3.x);
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1);
    v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2);
    v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3);
    v[7] = csub(e3, t3);
  }
};

template <int DIR, class C> struct DFT<3, DIR, C> {
  static __device__ __forceinline__ void run(C* v) {
    typedef decltype(v[0].x) T;
    const T s3 = (T)0.86602540378443864676372317075293618347;  // sqrt(3)/2
    C a = v[0], b = v[1], c = v[2];
    C t1 = cadd(b, c);
    C t2;
    t2.x = a.x - (T)0.5 * t1.x;
    t2.y = a.y - (T)0.5 * t1.y;
    C d = cmul_i<DIR>(cscale(csub(b, c), s3));
    v[0] = cadd(a, t1);
    v[1] = cadd(t2, d);
    v[2] = csub(t2, d);
  }
};

// ---------------------------------------------------------------- register-resident lines
// A line is spread over TPC = N/E threads, each holding E of its elements in
// registers, v[m] = x[t + TPC*m] for thread t of the line: E = 8 for
// power-of-two N, E = 12 for N = 3*2^k (96, 192, 384, 768).  Every stage's
// radix R divides E (8, 4 or 2 for E = 8; 4, 2, 3 for E = 12, in that
// order), and its butterflies run on registers -- butterfly b of the thread
// is j = t + TPC*b with inputs v[b + (E/R)*r], which are x[j + r*N/R], the
// Stockham map of fft_stage -- and the data crosses shared memory only
// between stages: a stage writes its outputs at their Stockham positions and
// the next stage reads the canonical v[m] back.  The last stage's outputs are
// the canonical positions themselves (NS*R = N makes them x[j + r*N/R]), so
// they stay in registers.
//
// Exchange buffer: `at(n)` is the shared-memory slot of element n of the
// thread's line.  The exchanges write either consecutive elements or
// elements R apart (d = Rj + r over consecutive j), and both must be free of
// bank conflicts for the phase a warp's access is split into (8 lanes for
// 16-byte elements, 16 for 8-byte ones).  Two index maps do that:
//   * reg_pad: one pad element after every 8 (n + n/8).  Lines are
//     interleaved for column slabs (element n of line c at pad(n)*CC + c)
//     and follow one another for FP64 x lines (c*reg_rows(N) + pad(n)).
//   * reg_swz: an XOR swizzle within aligned groups of 16, n ^ ((n/8) & 15),
//     for FP32 x lines (c*N + swz(n)).  With 8-byte elements a phase reads
//     16 consecutive elements, which the pad map splits unevenly over the
//     banks; the swizzle keeps them distinct (512^3: FP32 x inverse
//     0.28 -> 0.25 ms), while for FP64 its extra index arithmetic costs more
//     than it saves.
__host__ __device__ constexpr int reg_rows(int N) { return N + N / 8; }
__device__ __forceinline__ int reg_pad(int n) { return n + (n >> 3); }
__device__ __forceinline__ int reg_swz(int n) { return n ^ ((n >> 3) & 15); }
// Elements per thread of a register-resident line of length N.
__host__ __device__ constexpr int reg_elems(int N) { return (N & (N - 1)) == 0 ? 8 : 12; }
constexpr int pick_radix_reg(int rem, int E) {
  return (rem % 8 == 0 && E % 8 == 0) ? 8
         : (rem % 4 == 0 && E % 4 == 0) ? 4
         : (rem % 2 == 0 && E % 2 == 0) ? 2
         : (rem % 3 == 0 && E % 3 == 0) ? 3 : rem;
}

template <int N, int NS, int DIR, class C, int E, class At>
__device__ __forceinline__ void reg_fft_stages(C (&v)[E], C* s, const C* __restrict__ tw, int t, const At& at) {
  if constexpr (NS < N) {
    constexpr int R = pick_radix_reg(N / NS, E);
    static_assert(E % R == 0 && (N / NS) % R == 0, "register-resident lines: the radix must divide E");
    constexpr int B = E / R, TPC = N / E, TSTRIDE = N / (NS * R);
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int j = t + TPC * b;
      const int jm = j % NS;
      C u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        C a = v[b + B * r];
        if (NS > 1 && r > 0) {
          const C w = tw[r * jm * TSTRIDE];
          a = (DIR < 0) ? cmul(a, w) : cmulc(a, w);
        }
        u[r] = a;
      }
      DFT<R, DIR, C>::run(u);
#pragma unroll
      for (int r = 0; r < R; ++r) v[b + B * r] = u[r];
    }
    if constexpr (NS * R < N) {
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int j = t + TPC * b;
        const int d0 = (j / NS) * NS * R + j % NS;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          s[at(d0 + r * NS)] = v[b + B * r];
        }
      }
      __syncthreads();
#pragma unroll
      for (int m = 0; m < E; ++m) v[m] = s[at(t + TPC * m)];
      __syncthreads();
      reg_fft_stages<N, NS * R, DIR, C, E>(v, s, tw, t, at);
    }
  }
}

}  // namespace mhit
