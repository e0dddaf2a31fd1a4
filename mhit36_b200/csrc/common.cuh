// Shared device-side definitions for libmhit (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mhit {

// Device-resident control block.  Every kernel of a step reads it instead of
// taking step-dependent scalars as launch arguments, so one captured CUDA graph
// replays every step.
struct Ctrl {
  double mean[3];       // mean still to be removed from the stored u, v, w
  double gumax;         // signed Umax of the last step; gamma = 1.0*gumax
  double alpha, beta;   // AB2 weights of the next step (1, 0 before step 1)
  double cfl;           // gumax*dt*dxi of the last step
  double cfl_limit;     // step error above this (7 in the reference)
  double last_mean[3];  // means removed by the last step
  double max_div;       // max |div u| of the FP64 projection (FP32 refine form)
  long long nstep;      // steps taken
  int status;           // sticky MHIT_* error; kernels return early when set
  int pad_;
};

// Scalars fixed for the life of a handle, passed by value.
struct StepConst {
  int n;
  int abc;            // ABC forcing active
  int tanh_identity;  // tanh(psi/2eps) from phi directly
  int phi_floor;      // psi from max(min(phi,1),0) instead of min(phi,1)
  double dt, mu, rho, rhoi, dxi, ddxi, eps, epsi, enumv, tiny, sigma, lin_force;
  double f1, f2, f3;
  double cdiv;        // rho*dxi/dt   (multi/main.f90:723)
  double dtr;         // dt/rho       (multi/main.f90:881)
};

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ size_t gidx(int i, int j, int k, int n) {
  return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * (size_t)k);
}

// ---- asynchronous global -> shared copies (sm_80+ cp.async) ----
// One element per call (4 or 8 bytes); a thread's copies land in issue
// order groups: commit after a batch, wait until at most N groups are pending.
template <class T> __device__ __forceinline__ void cp_async_elem(T* smem_dst, const T* gmem_src) {
  static_assert(sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) == 16, "cp.async element size");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(T) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem_src), "n"(sizeof(T)) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- tensor-memory-accelerator tile loads completed on an mbarrier ----
// One thread arms a ring slot's barrier with the bytes it expects and issues
// the 2D box loads (cp.async.bulk.tensor, this GPU's own global memory, no
// multicast); every consumer waits on the slot's phase.  The box start's
// x coordinate times the element size must be a multiple of 16 bytes.
// SM clock cycles a wait on a ring slot's barrier lasts before it gives up
// (about 2 s at the B200's clocks; a staged plane lands within microseconds),
// and the sticky status it records.
constexpr long long kWaitCycles = 4000000000LL;
constexpr int kStatusTimeout = 10;  // MHIT_ERR_TIMEOUT
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
// make initialised barriers visible to the async proxy (then __syncthreads)
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(b)) : "memory");
}
// Wait for the phase with the given parity to complete, giving up once
// `limit_cycles` SM clock cycles have passed (a poll may suspend the thread
// for a short hardware time limit).  Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity, long long limit_cycles) {
  const unsigned a = smem_addr(b);
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit_cycles) return false;
  }
}
// Tensor maps in global memory written by a kernel (generic proxy): the
// writer releases them to the tensor-map proxy, the thread that issues
// box loads with one acquires it first.
__device__ __forceinline__ void tensormap_release() {
  asm volatile("fence.proxy.tensormap::generic.release.gpu;\n" ::: "memory");
}
__device__ __forceinline__ void tensormap_acquire(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
}
// 2D box at (x, y) of the tensor `map` into shared memory at `dst` (16-byte
// aligned; the box is stored densely, row pitch = box width).
__device__ __forceinline__ void tma_load_2d(void* dst, const void* map, int x, int y, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// 3D box at (x, y, z) of the tensor `map` into shared memory at `dst`.
__device__ __forceinline__ void tma_load_3d(void* dst, const void* map, int x, int y, int z, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// ---- complex helpers (double2 / float2) ----
template <class T> struct C2;
template <> struct C2<double> { typedef double2 t; };
template <> struct C2<float> { typedef float2 t; };

template <class C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <class C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <class C> __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
template <class C, class T> __device__ __forceinline__ C cscale(C a, T s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
// multiply by (DIR * i)
template <int DIR, class C> __device__ __forceinline__ C cmul_i(C a) {
  C r;
  if (DIR > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

}  // namespace mhit
