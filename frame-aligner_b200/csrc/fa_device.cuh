// fa_device.cuh -- device helpers shared by several translation units.
#pragma once

#include "fa_kernels.cuh"

namespace fa {

// f = sum over tiles (thread-strided runs, then a fixed tree); g[c] = sum over the tiles listed in
// ctrl_tiles[c], in tile order.
__device__ __forceinline__ void reduce_partials(const RefDev& R, const double* __restrict__ parts, double* f_out, double* g_out) {
  __shared__ double sf[kSolveThreads];
  double acc = 0.0;
  for (int t = threadIdx.x; t < R.n_tiles; t += blockDim.x) acc += parts[(long long)t * kPartialDoubles];
  sf[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sf[threadIdx.x] += sf[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *f_out = sf[0];
  const int nd = R.n_dim;
  for (int i = threadIdx.x; i < R.P; i += blockDim.x) {
    const int c = i / nd, k = i % nd;
    const int2 tr = R.ctrl_tiles[c];
    double a = 0.0;
    for (int t = tr.x; t < tr.y; t++) {
      const double* pt = parts + (long long)t * kPartialDoubles;
      const int s = c - (int)pt[1];
      if (s >= 0 && s < 3) a += pt[2 + s * 3 + k];
    }
    g_out[i] = a;
  }
  __syncthreads();
}

}  // namespace fa
