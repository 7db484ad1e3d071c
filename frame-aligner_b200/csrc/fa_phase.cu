// fa_phase.cu -- the hand-written parts of the rigid-start phase correlation
// (FrameAligner/VolumePhaseCorrelator.cpp:57-139); the FFTs themselves are cuFFT D2Z / Z2D.
//
//   phase_window_kernel     in[i] * window[i] -> double           (VolumePhaseCorrelator.cpp:62-63)
//   phase_normalise_kernel  X * conj(R) / (|X * conj(R)| + DBL_MIN) (VolumePhaseCorrelator.cpp:70-75)
//   phase_argmax_*          first index of the maximum            (VolumePhaseCorrelator.cpp:81-90)
#include <float.h>

#include "fa_kernels.cuh"

namespace fa {

__global__ void phase_window_kernel(const float* __restrict__ in, const double* __restrict__ w,
                                    double* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __dmul_rn((double)in[i], w[i]);
}

cudaError_t launch_phase_window(const float* in, const double* window, double* out, long long n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  phase_window_kernel<<<blocks, 256, 0, s>>>(in, window, out, n);
  return cudaGetLastError();
}

__global__ void phase_conj_kernel(const double2* __restrict__ in, double2* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double2 v = in[i];
    out[i] = make_double2(v.x, -v.y);
  }
}

cudaError_t launch_phase_conj(const double2* in, double2* out, long long n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  phase_conj_kernel<<<blocks, 256, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

// Cross-power spectrum in place: z = X * Rc (Rc = conj(F(reference)), stored), z / (|z| + DBL_MIN).
// Products and sums are rounded separately (no FMA), like the reference's SSE3 build.
__global__ void phase_normalise_kernel(double2* __restrict__ spec, const double2* __restrict__ rc, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 a = spec[i], b = rc[i];
    const double re = __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
    const double im = __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x));
    const double nrm = __dadd_rn(hypot(re, im), DBL_MIN);
    spec[i] = make_double2(__ddiv_rn(re, nrm), __ddiv_rn(im, nrm));
  }
}

cudaError_t launch_phase_normalise(double2* spec, const double2* ref_conj, long long n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  phase_normalise_kernel<<<blocks, 256, 0, s>>>(spec, ref_conj, n);
  return cudaGetLastError();
}

// (value, index) with "greater value, then smaller index" ordering; NaN never wins, as the
// reference's strict `in[i] > pk` starting from -DBL_MAX.
__device__ __forceinline__ void better(double& v, long long& i, double v2, long long i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

__global__ void __launch_bounds__(256) phase_argmax_blocks(const double* __restrict__ surf, long long n,
                                                           double* __restrict__ bval, long long* __restrict__ bidx) {
  double v = -DBL_MAX;
  long long idx = 0x7fffffffffffffffLL;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    better(v, idx, surf[i], i);
  __shared__ double sv[256];
  __shared__ long long si[256];
  sv[threadIdx.x] = v;
  si[threadIdx.x] = idx;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      double v2 = sv[threadIdx.x + w];
      long long i2 = si[threadIdx.x + w];
      double vv = sv[threadIdx.x];
      long long ii = si[threadIdx.x];
      better(vv, ii, v2, i2);
      sv[threadIdx.x] = vv;
      si[threadIdx.x] = ii;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bval[blockIdx.x] = sv[0];
    bidx[blockIdx.x] = si[0];
  }
}

__global__ void __launch_bounds__(256) phase_argmax_final(const double* __restrict__ bval,
                                                          const long long* __restrict__ bidx, int nb,
                                                          long long* __restrict__ out) {
  double v = -DBL_MAX;
  long long idx = 0x7fffffffffffffffLL;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) better(v, idx, bval[i], bidx[i]);
  __shared__ double sv[256];
  __shared__ long long si[256];
  sv[threadIdx.x] = v;
  si[threadIdx.x] = idx;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      double vv = sv[threadIdx.x];
      long long ii = si[threadIdx.x];
      better(vv, ii, sv[threadIdx.x + w], si[threadIdx.x + w]);
      sv[threadIdx.x] = vv;
      si[threadIdx.x] = ii;
    }
    __syncthreads();
  }
  // every element NaN (or -inf): the reference keeps idx = 0
  if (threadIdx.x == 0) *out = (si[0] == 0x7fffffffffffffffLL) ? 0 : si[0];
}

cudaError_t launch_phase_argmax(const double* surf, long long n, double* block_val, long long* block_idx,
                                int n_blocks, long long* out_idx, cudaStream_t s) {
  phase_argmax_blocks<<<n_blocks, 256, 0, s>>>(surf, n, block_val, block_idx);
  phase_argmax_final<<<1, 256, 0, s>>>(block_val, block_idx, n_blocks, out_idx);
  return cudaGetLastError();
}

}  // namespace fa
