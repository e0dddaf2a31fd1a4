// On-GPU FP64 diagnostics of the resident state.
//
// The reference has no in-solver energy or dissipation output; its
// dissipation comes from the serial post-processor post/compute_diss
// (main.f90:72-117): eps = 2 nu <S_ij S_ij> with centred differences and
// periodic wrap on the stored (staggered) fields, dx = 2 pi/(nx-1) where pi is
// the default-real literal 3.14159265358979 of post/compute_diss/module.f90:5
// (so rounded to float32).  This kernel computes the same sum on the GPU, plus
// the kinetic energy 0.5<u^2+v^2+w^2>, the max |div u| of the projection's
// forward-difference divergence, and the phi volume sum and bounds.
#include <cuda_runtime.h>
#include <math.h>
#include "common.cuh"
#include "internal.h"

namespace mhit {

constexpr int DTX = 32, DTY = 8, DNT = DTX * DTY, DKZ = 16;
constexpr int NSTAT = 8;  // sum(u^2+v^2+w^2), sum(SijSij), max|div|, sum phi, min phi, max phi, sum u, pad

template <class T>
__global__ void __launch_bounds__(DNT) stats_kernel(const T* __restrict__ u, const T* __restrict__ v,
                                                    const T* __restrict__ w, const T* __restrict__ phi,
                                                    const Ctrl* __restrict__ ctrl, int n, double dxi_c,
                                                    double dxi_d, double* __restrict__ partials) {
  const double mu = ctrl->mean[0], mv = ctrl->mean[1], mw = ctrl->mean[2];
  const int i = blockIdx.x * DTX + threadIdx.x % DTX, j = blockIdx.y * DTY + threadIdx.x / DTX;
  const int ip = (i + 1 == n) ? 0 : i + 1, im = i ? i - 1 : n - 1;
  const int jp = (j + 1 == n) ? 0 : j + 1, jm = j ? j - 1 : n - 1;
  const size_t nn = (size_t)n * n;
  double s[NSTAT] = {0, 0, 0, 0, INFINITY, -INFINITY, 0, 0};
  for (int k = blockIdx.z * DKZ; k < (blockIdx.z + 1) * DKZ; ++k) {
    const int kp = (k + 1 == n) ? 0 : k + 1, km = k ? k - 1 : n - 1;
    auto U = [&](int a, int b, int c) { return (double)u[(size_t)a + (size_t)n * b + nn * c] - mu; };
    auto V = [&](int a, int b, int c) { return (double)v[(size_t)a + (size_t)n * b + nn * c] - mv; };
    auto W = [&](int a, int b, int c) { return (double)w[(size_t)a + (size_t)n * b + nn * c] - mw; };
    const double uc = U(i, j, k), vc = V(i, j, k), wc = W(i, j, k);
    s[0] += uc * uc + vc * vc + wc * wc;
    s[6] += uc;
    // compute_diss (post/compute_diss/main.f90:87-111)
    const double h = 0.5 * dxi_d;
    const double dudx = (U(ip, j, k) - U(im, j, k)) * h, dudy = (U(i, jp, k) - U(i, jm, k)) * h,
                 dudz = (U(i, j, kp) - U(i, j, km)) * h;
    const double dvdx = (V(ip, j, k) - V(im, j, k)) * h, dvdy = (V(i, jp, k) - V(i, jm, k)) * h,
                 dvdz = (V(i, j, kp) - V(i, j, km)) * h;
    const double dwdx = (W(ip, j, k) - W(im, j, k)) * h, dwdy = (W(i, jp, k) - W(i, jm, k)) * h,
                 dwdz = (W(i, j, kp) - W(i, j, km)) * h;
    const double S12 = 0.5 * (dudy + dvdx), S13 = 0.5 * (dudz + dwdx), S23 = 0.5 * (dvdz + dwdy);
    s[1] += dudx * dudx + dvdy * dvdy + dwdz * dwdz + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23);
    // forward-difference divergence of the projection (multi/main.f90:723-725)
    const double div = ((U(ip, j, k) - uc) + (V(i, jp, k) - vc) + (W(i, j, kp) - wc)) * dxi_c;
    s[2] = fmax(s[2], fabs(div));
    if (div != div) s[2] = NAN;
    if (phi) {
      const double f = (double)phi[(size_t)i + (size_t)n * j + nn * k];
      s[3] += f;
      s[4] = fmin(s[4], f);
      s[5] = fmax(s[5], f);
    }
  }
  __shared__ double red[DNT / 32][NSTAT];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    for (int t = 0; t < NSTAT; ++t) {
      const double x = __shfl_xor_sync(0xffffffffu, s[t], o);
      if (t == 2 || t == 5) s[t] = fmax(s[t], x);
      else if (t == 4) s[t] = fmin(s[t], x);
      else s[t] += x;
    }
  }
  if ((threadIdx.x & 31) == 0)
    for (int t = 0; t < NSTAT; ++t) red[threadIdx.x >> 5][t] = s[t];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int wdx = 1; wdx < DNT / 32; ++wdx)
      for (int t = 0; t < NSTAT; ++t) {
        const double x = red[wdx][t];
        if (t == 2 || t == 5) red[0][t] = fmax(red[0][t], x);
        else if (t == 4) red[0][t] = fmin(red[0][t], x);
        else red[0][t] += x;
      }
    const size_t b = (size_t)blockIdx.x + (size_t)gridDim.x * (blockIdx.y + (size_t)gridDim.y * blockIdx.z);
    for (int t = 0; t < NSTAT; ++t) partials[b * NSTAT + t] = red[0][t];
  }
}

__global__ void stats_final_kernel(const double* __restrict__ partials, int nparts, double* __restrict__ out) {
  __shared__ double red[256][NSTAT];
  double s[NSTAT] = {0, 0, 0, 0, INFINITY, -INFINITY, 0, 0};
  for (int b = threadIdx.x; b < nparts; b += 256)
    for (int t = 0; t < NSTAT; ++t) {
      const double x = partials[(size_t)b * NSTAT + t];
      if (t == 2 || t == 5) s[t] = fmax(s[t], x);
      else if (t == 4) s[t] = fmin(s[t], x);
      else s[t] += x;
    }
  for (int t = 0; t < NSTAT; ++t) red[threadIdx.x][t] = s[t];
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int t = 0; t < NSTAT; ++t) {
        const double x = red[threadIdx.x + st][t];
        double& y = red[threadIdx.x][t];
        if (t == 2 || t == 5) y = fmax(y, x);
        else if (t == 4) y = fmin(y, x);
        else y += x;
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int t = 0; t < NSTAT; ++t) out[t] = red[0][t];
}

int stats_partials(int n) { return (n / DTX) * (n / DTY) * (n / DKZ); }

template <class T>
cudaError_t launch_stats(const T* u, const T* v, const T* w, const T* phi, const Ctrl* ctrl, int n, double dxi_c,
                         double dxi_d, double* partials, double* out, cudaStream_t st) {
  dim3 grid(n / DTX, n / DTY, n / DKZ);
  stats_kernel<T><<<grid, DNT, 0, st>>>(u, v, w, phi, ctrl, n, dxi_c, dxi_d, partials);
  stats_final_kernel<<<1, 256, 0, st>>>(partials, stats_partials(n), out);
  return cudaGetLastError();
}

template cudaError_t launch_stats<double>(const double*, const double*, const double*, const double*, const Ctrl*,
                                          int, double, double, double*, double*, cudaStream_t);
template cudaError_t launch_stats<float>(const float*, const float*, const float*, const float*, const Ctrl*, int,
                                         double, double, double*, double*, cudaStream_t);

}  // namespace mhit
