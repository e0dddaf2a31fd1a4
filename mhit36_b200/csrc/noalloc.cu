// Allocation-free Poisson solve: mhit_poisson_noalloc (include/mhit.h).
//
// Some callers cannot let a library call cudaMalloc / cudaFree.  Typical
// cases: an application whose device memory is entirely owned by its own
// allocator (a caching allocator that has already reserved the pool, so a
// cudaMalloc from us would fail or fragment it), and latency-critical loops
// that cannot afford the device-wide synchronisation cudaFree implies.  For
// them this entry point runs the same Poisson kernels as mhit_poisson_device
// without a handle: the caller passes device input and output, and the
// solve's scratch -- the half spectrum and the twiddle / k^2 tables -- lives
// in the fixed file-scope device arrays below, sized for grids up to
// MHIT_NOALLOC_MAX_N^3.  Every GPU that loads the library holds these arrays
// (18.9 MB) until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// arrays' device addresses with cudaGetSymbolAddress (their names in host code
// are only host-side stand-ins) and caches them; that first call should come
// before any stream capture.  Every call shares the same arrays and leaves its
// contents behind, so calls that overlap on the GPU (different streams, or
// different host threads) race; serialise them.  Nothing in the scratch has to
// start at zero: every element a solve reads is written earlier in the same
// call (columns beyond kx = n/2 are transformed independently and zeroed by the
// k^2 division before anything reads them).
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>

#include "internal.h"
#include "mhit.h"

namespace {

constexpr int kMaxN = MHIT_NOALLOC_MAX_N;
constexpr size_t kPitchMax = (kMaxN / 2 + 1 + 7) / 8 * 8;  // spectrum row pitch for n = kMaxN
constexpr size_t kSpecElems = (size_t)kMaxN * kMaxN * kPitchMax;

static __device__ __align__(256) double2 g_noalloc_spec[kSpecElems];
static __device__ __align__(256) double2 g_noalloc_tw[kMaxN];
static __device__ __align__(256) double g_noalloc_k2[kMaxN];

constexpr int kMaxDevices = 64;
struct Addrs {
  bool ready = false;
  double2* spec = nullptr;
  double2* tw = nullptr;
  double* k2 = nullptr;
};
Addrs g_addrs[kMaxDevices];
std::mutex g_mutex;

int setup_device(int dev, Addrs* out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  Addrs& a = g_addrs[dev];
  if (!a.ready) {
    if (cudaGetSymbolAddress((void**)&a.spec, g_noalloc_spec) != cudaSuccess) return MHIT_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&a.tw, g_noalloc_tw) != cudaSuccess) return MHIT_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&a.k2, g_noalloc_k2) != cudaSuccess) return MHIT_ERR_CUDA;
    a.ready = true;
  }
  *out = a;
  return MHIT_OK;
}

bool built_size(int n) {
  bool ok = false;
#define MHIT_CASE(NN) ok |= (n == NN);
  MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
  return ok;
}

}  // namespace

extern "C" int mhit_poisson_noalloc(const double* rhs_dev, double* p_dev, int n, int k2_mode, int grid_mode,
                                    void* stream) {
  if (!rhs_dev || !p_dev || n < 2) return MHIT_ERR_INVALID;
  if (n > kMaxN) return MHIT_ERR_SCRATCH_LIMIT;
  if (!built_size(n)) return MHIT_ERR_UNSUPPORTED;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MHIT_ERR_CUDA;
  Addrs a;
  int rc = setup_device(dev, &a);
  if (rc) return rc;
  if (mhit::spectrum_pitch(n, 0) > kPitchMax) return MHIT_ERR_SCRATCH_LIMIT;
  if (mhit::prepare_poisson(n) != cudaSuccess) return MHIT_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // Tables on the host stack, as mhit_create builds them (same values, so the
  // result equals mhit_poisson_device's bit for bit).
  double2 tw[kMaxN];
  double k2[kMaxN];
  const double twopi = 8.0 * atan(1.0);
  const double lx = twopi;
  const double dx = (grid_mode == MHIT_GRID_CONSISTENT) ? lx / n : lx / (n - 1);
  const double ddxi = 1.0 / dx / dx;
  const double pi = 4.0 * atan(1.0);
  for (int m = 0; m < n; ++m) {
    long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
    tw[m].x = (double)cosl(ang);
    tw[m].y = -(double)sinl(ang);
    if (k2_mode == MHIT_K2_FD) {
      const double s = sin(pi * m / n);
      k2[m] = (4.0 * ddxi) * (s * s);
    } else {
      const double kk = (m < n / 2 ? (double)m : (double)(m - n)) * (twopi / lx);
      k2[m] = kk * kk;
    }
  }
  // Pageable-source copies return once the source has been staged, so the
  // stack arrays may go out of scope afterwards.
  if (cudaMemcpyAsync(a.tw, tw, n * sizeof(double2), cudaMemcpyHostToDevice, st) != cudaSuccess) return MHIT_ERR_CUDA;
  if (cudaMemcpyAsync(a.k2, k2, n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) return MHIT_ERR_CUDA;

  mhit::PoissonArgs<double> pa;
  pa.rhs = rhs_dev;
  pa.spec = a.spec;
  pa.p = p_dev;
  pa.tw = a.tw;
  pa.k2tab = a.k2;
  pa.ctrl = nullptr;
  if (mhit::launch_poisson<double>(n, pa, st) != cudaSuccess) return MHIT_ERR_CUDA;
  return MHIT_OK;
}
