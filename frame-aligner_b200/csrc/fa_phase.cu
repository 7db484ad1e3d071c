// fa_phase.cu -- the hand-written parts of the rigid-start phase correlation
// (FrameAligner/VolumePhaseCorrelator.cpp:57-139); the FFTs themselves are cuFFT D2Z / Z2D.
//
//   phase_window_kernel     in[i] * window[i] -> double           (VolumePhaseCorrelator.cpp:62-63)
//   phase_normalise_kernel  X * conj(R) / (|X * conj(R)| + DBL_MIN) (VolumePhaseCorrelator.cpp:70-75)
//   phase_argmax_*          first index of the maximum            (VolumePhaseCorrelator.cpp:81-90)
#include <float.h>

#include "fa_kernels.cuh"

namespace fa {

// Windowed FP64 input of a batch of frames: out[b][i] = double(vol_b[i]) * ((1 * wy[y]) * wx[x]) --
// the reference's window (1 along z) formed as in VolumePhaseCorrelator.cpp:141-153, applied as at
// :62-63. vol_b is dense FP32 or uint16 (in_kind is an fa_dtype); the correlator sees the raw frames,
// without the +1 offset.
__global__ void phase_window_kernel(const void* const* __restrict__ vols, int in_kind, const double* __restrict__ wy,
                                    const double* __restrict__ wx, int ny, int nx, int n_rows,
                                    double* __restrict__ out) {
  const int b = blockIdx.y;
  const void* vol = vols[b];
  const long long n_el = (long long)n_rows * nx;
  double* o = out + (long long)b * n_el;
  for (int row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const double wrow = __dmul_rn(1.0, wy[row % ny]);
    const long long base = (long long)row * nx;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const long long i = base + x;
      const float v = in_kind == FA_U16 ? (float)static_cast<const unsigned short*>(vol)[i]
                                        : static_cast<const float*>(vol)[i];
      o[i] = __dmul_rn((double)v, __dmul_rn(wrow, wx[x]));
    }
  }
}

cudaError_t launch_phase_window(const void* const* vols, int in_kind, const double* wy, const double* wx, int ny,
                                int nx, long long n_el, int batch, double* out, cudaStream_t s) {
  const int n_rows = (int)(n_el / nx);
  int blocks = n_rows;
  const int cap = (148 * 16 + batch - 1) / batch;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  phase_window_kernel<<<dim3(blocks, batch), 256, 0, s>>>(vols, in_kind, wy, wx, ny, nx, n_rows, out);
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

// Cross-power spectrum in place for a batch: z = X_b * Rc (Rc = conj(F(reference)), stored),
// z / (|z| + DBL_MIN) (VolumePhaseCorrelator.cpp:70-75). Products and sums are rounded separately
// (no FMA), like the reference's SSE3 build.
__global__ void phase_normalise_kernel(double2* __restrict__ spec, const double2* __restrict__ rc, long long n) {
  double2* sp = spec + (long long)blockIdx.y * n;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x) {
    const double2 a = sp[j], b = rc[j];
    const double re = __dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y));
    const double im = __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x));
    const double nrm = __dadd_rn(hypot(re, im), DBL_MIN);
    sp[j] = make_double2(__ddiv_rn(re, nrm), __ddiv_rn(im, nrm));
  }
}

cudaError_t launch_phase_normalise(double2* spec, const double2* ref_conj, long long n, int batch, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  const int cap = (148 * 16 + batch - 1) / batch;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  phase_normalise_kernel<<<dim3(blocks, batch), 256, 0, s>>>(spec, ref_conj, n);
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

// First maximum of each frame's surface: grid (blocks per frame, frames); then one block per frame.
__global__ void __launch_bounds__(256) phase_argmax_blocks(const double* __restrict__ surf, long long n,
                                                           double* __restrict__ bval, long long* __restrict__ bidx) {
  const double* sf = surf + (long long)blockIdx.y * n;
  double v = -DBL_MAX;
  long long idx = 0x7fffffffffffffffLL;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    better(v, idx, sf[i], i);
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
  if (threadIdx.x == 0) {
    bval[(long long)blockIdx.y * gridDim.x + blockIdx.x] = sv[0];
    bidx[(long long)blockIdx.y * gridDim.x + blockIdx.x] = si[0];
  }
}

__global__ void __launch_bounds__(256) phase_argmax_final(const double* __restrict__ bval,
                                                          const long long* __restrict__ bidx, int nb,
                                                          long long* __restrict__ out) {
  const double* bv = bval + (long long)blockIdx.x * nb;
  const long long* bi = bidx + (long long)blockIdx.x * nb;
  double v = -DBL_MAX;
  long long idx = 0x7fffffffffffffffLL;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) better(v, idx, bv[i], bi[i]);
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
  if (threadIdx.x == 0) out[blockIdx.x] = (si[0] == 0x7fffffffffffffffLL) ? 0 : si[0];
}

cudaError_t launch_phase_argmax_final(const double* block_val, const long long* block_idx, int nb, int batch,
                                      long long* out_idx, cudaStream_t s) {
  phase_argmax_final<<<batch, 256, 0, s>>>(block_val, block_idx, nb, out_idx);
  return cudaGetLastError();
}

cudaError_t launch_phase_argmax(const double* surf, long long n, int batch, double* block_val, long long* block_idx,
                                int blocks_per_frame, long long* out_idx, cudaStream_t s) {
  phase_argmax_blocks<<<dim3(blocks_per_frame, batch), 256, 0, s>>>(surf, n, block_val, block_idx);
  phase_argmax_final<<<batch, 256, 0, s>>>(block_val, block_idx, blocks_per_frame, out_idx);
  return cudaGetLastError();
}

}  // namespace fa
