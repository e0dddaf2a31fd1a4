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
// are only host-side stand-ins), fills the twiddle tables of every built size
// up to the maximum and the k^2 tables of every (size, k2_mode, grid_mode)
// with one synchronous copy, and opts those sizes' kernels into their shared
// memory.  That first call should come before any stream capture.  After it,
// a call only launches the solve's kernels on the caller's stream: nothing is
// copied from the host.
//
// Every call shares the same spectrum array and leaves its contents behind,
// so calls that overlap on the GPU (different streams, or different host
// threads) race; serialise them.  Nothing in the spectrum has to start at
// zero: every element a solve reads is written earlier in the same call
// (columns beyond kx = n/2 are transformed independently and zeroed by the
// k^2 division before anything reads them).
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include <vector>

#include "internal.h"
#include "mhit.h"

namespace {

constexpr int kMaxN = MHIT_NOALLOC_MAX_N;
constexpr size_t kPitchMax = (kMaxN / 2 + 1 + 7) / 8 * 8;  // spectrum row pitch for n = kMaxN
constexpr size_t kSpecElems = (size_t)kMaxN * kMaxN * kPitchMax;

// Built sizes up to kMaxN, and the offset of each size's tables.
constexpr int kSizeSlots = 16;
struct SizeTable {
  int count = 0;
  int n[kSizeSlots] = {};
  int off[kSizeSlots] = {};
  int total = 0;
};
constexpr SizeTable make_sizes() {
  SizeTable t;
#define MHIT_CASE(NN)            \
  if (NN <= kMaxN) {             \
    t.n[t.count] = NN;           \
    t.off[t.count] = t.total;    \
    t.total += NN;               \
    ++t.count;                   \
  }
  MHIT_FOR_SIZES(MHIT_CASE)
#undef MHIT_CASE
  return t;
}
constexpr SizeTable kSizes = make_sizes();
static_assert(kSizes.count > 0 && kSizes.count <= kSizeSlots, "size table");
// k^2 tables: one per (k2_mode, grid_mode) for every size
constexpr int kModes = 4;

static __device__ __align__(256) double2 g_noalloc_spec[kSpecElems];
static __device__ __align__(256) double2 g_noalloc_tw[kSizes.total];
static __device__ __align__(256) double g_noalloc_k2[kModes * kSizes.total];

constexpr int kMaxDevices = 64;
struct Addrs {
  bool ready = false;
  double2* spec = nullptr;
  double2* tw = nullptr;
  double* k2 = nullptr;
};
Addrs g_addrs[kMaxDevices];
std::mutex g_mutex;

int size_slot(int n) {
  for (int q = 0; q < kSizes.count; ++q)
    if (kSizes.n[q] == n) return q;
  return -1;
}

int mode_index(int k2_mode, int grid_mode) {
  return (k2_mode == MHIT_K2_FD ? 2 : 0) + (grid_mode == MHIT_GRID_CONSISTENT ? 1 : 0);
}

// The tables mhit_create builds for a handle, for every size and mode (the
// same values, so a solve here equals mhit_poisson_device's bit for bit).
void host_tables(std::vector<double2>& tw, std::vector<double>& k2) {
  tw.assign(kSizes.total, double2{0, 0});
  k2.assign((size_t)kModes * kSizes.total, 0.0);
  const double twopi = 8.0 * atan(1.0);
  const double lx = twopi;
  const double pi = 4.0 * atan(1.0);
  for (int q = 0; q < kSizes.count; ++q) {
    const int n = kSizes.n[q], off = kSizes.off[q];
    for (int m = 0; m < n; ++m) {
      long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
      tw[off + m].x = (double)cosl(ang);
      tw[off + m].y = -(double)sinl(ang);
    }
    for (int k2_mode = 0; k2_mode < 2; ++k2_mode)
      for (int grid_mode = 0; grid_mode < 2; ++grid_mode) {
        double* t = k2.data() + (size_t)mode_index(k2_mode, grid_mode) * kSizes.total + off;
        const double dx = (grid_mode == MHIT_GRID_CONSISTENT) ? lx / n : lx / (n - 1);
        const double ddxi = 1.0 / dx / dx;
        for (int m = 0; m < n; ++m) {
          if (k2_mode == MHIT_K2_FD) {
            const double s = sin(pi * m / n);
            t[m] = (4.0 * ddxi) * (s * s);
          } else {
            const double kk = (m < n / 2 ? (double)m : (double)(m - n)) * (twopi / lx);
            t[m] = kk * kk;
          }
        }
      }
  }
}

int setup_device(int dev, Addrs* out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  Addrs& a = g_addrs[dev];
  if (!a.ready) {
    Addrs t;
    if (cudaGetSymbolAddress((void**)&t.spec, g_noalloc_spec) != cudaSuccess) return MHIT_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&t.tw, g_noalloc_tw) != cudaSuccess) return MHIT_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&t.k2, g_noalloc_k2) != cudaSuccess) return MHIT_ERR_CUDA;
    std::vector<double2> tw;
    std::vector<double> k2;
    host_tables(tw, k2);
    if (cudaMemcpy(t.tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
      return MHIT_ERR_CUDA;
    if (cudaMemcpy(t.k2, k2.data(), k2.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      return MHIT_ERR_CUDA;
    for (int q = 0; q < kSizes.count; ++q)
      if (mhit::prepare_poisson(kSizes.n[q]) != cudaSuccess) return MHIT_ERR_CUDA;
    t.ready = true;
    a = t;
  }
  *out = a;
  return MHIT_OK;
}

}  // namespace

extern "C" int mhit_poisson_noalloc(const double* rhs_dev, double* p_dev, int n, int k2_mode, int grid_mode,
                                    void* stream) {
  if (!rhs_dev || !p_dev || n < 2) return MHIT_ERR_INVALID;
  if (n > kMaxN) return MHIT_ERR_SCRATCH_LIMIT;
  const int slot = size_slot(n);
  if (slot < 0) return MHIT_ERR_UNSUPPORTED;
  if (mhit::spectrum_pitch(n, 0) > kPitchMax) return MHIT_ERR_SCRATCH_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return MHIT_ERR_CUDA;
  Addrs a;
  int rc = setup_device(dev, &a);
  if (rc) return rc;
  mhit::PoissonArgs<double> pa;
  pa.rhs = rhs_dev;
  pa.spec = a.spec;
  pa.p = p_dev;
  pa.tw = a.tw + kSizes.off[slot];
  pa.k2tab = a.k2 + (size_t)mode_index(k2_mode, grid_mode) * kSizes.total + kSizes.off[slot];
  pa.ctrl = nullptr;
  if (mhit::launch_poisson<double>(n, pa, static_cast<cudaStream_t>(stream)) != cudaSuccess) return MHIT_ERR_CUDA;
  return MHIT_OK;
}
