// Drop count and size distribution of the phase field on the GPU.
//
// Restates the serial post-processor post/DropCountSize: binarise phi >= 0.5
// (get_interface.f90:12-22), find 26-connected components with periodic wrap
// (the recursive flood fill of flood_fill.f90:1-127, which overflows the stack
// for large drops), number the drops in the order the Fortran scan meets
// their first cell (get_interface.f90:28-47), and give each drop's equivalent
// diameter deq = dx*(6 V/pi)^(1/3) with V its cell count (calculate_deq.f90:29-33).
//
// GPU algorithm: lock-free union-find over the 13 forward neighbours of every
// foreground cell; roots only ever decrease (atomicMin), so each component's
// root ends as its smallest linear index -- the cell the reference's scan
// reaches first -- and sorting the roots reproduces the reference's order.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "internal.h"

namespace mhit {

template <class T>
__global__ void ccl_init_kernel(const T* __restrict__ phi, int* __restrict__ lab, int* __restrict__ cnt, size_t count) {
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
    lab[g] = (phi[g] >= (T)0.5) ? (int)g : -1;
    cnt[g] = 0;
  }
}

// Root of x.  Labels only decrease and L[x] <= x, so the chain strictly
// decreases and ends within x steps; the loop bound only makes that explicit.
__device__ __forceinline__ int ccl_find(const int* L, int x) {
  int p = L[x];
  for (int it = 0; p != x && it < (1 << 30); ++it) {
    x = p;
    p = L[x];
  }
  return x;
}

__device__ __forceinline__ void ccl_unite(int* L, int a, int b, int* err) {
  for (int it = 0; it < (1 << 24); ++it) {
    a = ccl_find(L, a);
    b = ccl_find(L, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&L[b], a);
    if (old == b) return;
    b = old;
  }
  atomicExch(err, 1);  // bounded retry loop gave up (never expected)
}

__global__ void ccl_merge_kernel(int* __restrict__ L, int n, int* err) {
  const size_t count = (size_t)n * n * n, nn = (size_t)n * n;
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
    if (L[g] < 0) continue;
    const int i = (int)(g % n), j = (int)((g / n) % n), k = (int)(g / nn);
    // the 13 forward neighbours: dk > 0, or dk == 0 and dj > 0, or dk == dj == 0 and di > 0
    for (int dk = 0; dk <= 1; ++dk)
      for (int dj = -1; dj <= 1; ++dj)
        for (int di = -1; di <= 1; ++di) {
          if (dk == 0 && (dj < 0 || (dj == 0 && di <= 0))) continue;
          const int ii = wrapi(i + di, n), jj = wrapi(j + dj, n), kk = wrapi(k + dk, n);
          const size_t nb = (size_t)ii + (size_t)n * jj + nn * kk;
          if (L[nb] >= 0) ccl_unite(L, (int)g, (int)nb, err);
        }
  }
}

__global__ void ccl_count_kernel(int* __restrict__ L, int* __restrict__ cnt, size_t count) {
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
    if (L[g] < 0) continue;
    const int r = ccl_find(L, (int)g);
    atomicAdd(&cnt[r], 1);
  }
}

__global__ void ccl_roots_kernel(const int* __restrict__ L, const int* __restrict__ cnt, size_t count,
                                 int2* __restrict__ out, int cap, int* __restrict__ nout) {
  for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
    if (L[g] == (int)g) {
      const int slot = atomicAdd(nout, 1);
      if (slot < cap) out[slot] = make_int2((int)g, cnt[g]);
    }
  }
}

template <class T>
cudaError_t launch_dropcount(const T* phi, int n, int* lab, int* cnt, int2* roots, int cap, int* d_counter,
                             cudaStream_t st) {
  const size_t count = (size_t)n * n * n;
  const int grid = 148 * 8, block = 256;
  ccl_init_kernel<T><<<grid, block, 0, st>>>(phi, lab, cnt, count);
  cudaError_t e = cudaMemsetAsync(d_counter, 0, 2 * sizeof(int), st);  // [0] roots, [1] error flag
  if (e) return e;
  ccl_merge_kernel<<<grid, block, 0, st>>>(lab, n, d_counter + 1);
  ccl_count_kernel<<<grid, block, 0, st>>>(lab, cnt, count);
  ccl_roots_kernel<<<grid, block, 0, st>>>(lab, cnt, count, roots, cap, d_counter);
  return cudaGetLastError();
}

template cudaError_t launch_dropcount<double>(const double*, int, int*, int*, int2*, int, int*, cudaStream_t);
template cudaError_t launch_dropcount<float>(const float*, int, int*, int*, int2*, int, int*, cudaStream_t);

}  // namespace mhit
