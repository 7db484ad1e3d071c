// fa_output.cu -- what FrameWarpAligner produces for a frame once its D is known
// (FrameAligner/FrameWarpAligner.cpp:221-247, 317-346), on the device:
//
//   splat_kernel      AbstractFrameWarper::warpImage (FrameWarper.cpp:71-136): the forward,
//                     intensity-preserving splat of a frame and its coverage
//   metric kernels    correlation() (Cv3dUtils.cpp:57-81) of the warped and of the unaligned frame
//                     against the reference over coverage > 0, and the coverage fraction
//   to_u16_kernel     reshapeForOutput's convertTo(CV_16U) of the realigned images
//
// The splat recomputes the reference's warpPoint exactly: the interval index and the float Df of
// precomputeInterp (FrameWarper.cpp:252-263) from the processed scan durations in FP64, then
// d = Df D[i+1] + (1 - Df) D[i] and the trilinear splat weights in FP64 as the reference does.
// The reference accumulates each target voxel in float in scan order; here contributions arrive by
// float atomic adds in arbitrary order, so sums agree to float rounding (a few ulp), not bit for
// bit. Metric sums are FP64 in a fixed order (per-thread strides, then a tree per block, then the
// blocks in order), so they are deterministic.
#include <cmath>
#include <cstring>
#include <fstream>

#include "fa_runtime.h"

using fa::Job;
using fa::RefDev;
using namespace fa_rt;

namespace fa {
namespace {

// Processed scan durations (AbstractFrameWarper::processScanParameters).
struct ScanD {
  double pd, ild, ifd, stack;
};

constexpr int kMetricBlocks = 296;
constexpr int kMetricThreads = 256;
constexpr int kMetricTerms = 8;  // count, sum w, sum r, sum ww, sum rr, sum f, sum ff, spare

// Di and Df of the voxel stored at (x, y, z) (the scan visits it at x, or nx-1-x on odd lines of a
// bidirectional scan).
__device__ __forceinline__ void exact_interval(const RefDev& R, const ScanD& sc, int x, int y, int z, int* i,
                                               double* f) {
  const bool flip = R.bidir && (y & 1);
  const int xs = flip ? R.nx - 1 - x : x;
  const double t = __dadd_rn(__dadd_rn(__dmul_rn((double)z, sc.ifd), __dmul_rn((double)y, sc.ild)),
                             __dmul_rn((double)xs, sc.pd));
  const double q = __dmul_rn(__ddiv_rn(t, sc.stack), (double)(R.nD - 1));
  const double fl = floor(q);
  *i = (int)fl;
  *f = (double)(float)__dsub_rn(q, fl);  // Df is stored as float
}

__device__ __forceinline__ float load_raw(const void* p, int kind, long long i) {
  return kind == FA_U16 ? (float)static_cast<const unsigned short*>(p)[i] : static_cast<const float*>(p)[i];
}

template <int NDIM>
__global__ void __launch_bounds__(256) splat_kernel(const RefDev* __restrict__ Rp, ScanD sc,
                                                    const void* __restrict__ img, int img_kind,
                                                    const double* __restrict__ D, float* __restrict__ wimg,
                                                    float* __restrict__ cov) {
  const RefDev& R = *Rp;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < R.N;
       p += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(p % nx);
    const long long r = p / nx;
    const int y = (int)(r % ny);
    const int z = (int)(r / ny);
    int i;
    double f;
    exact_interval(R, sc, x, y, z, &i, &f);
    const double g = __dsub_rn(1.0, f);
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; c++) d[c] = __dadd_rn(__dmul_rn(f, D[3 * (i + 1) + c]), __dmul_rn(g, D[3 * i + c]));
    if (NDIM == 2) d[2] = 0.0;  // single plane: the z component is ignored, every target is in plane 0
    const double lx = __dsub_rn((double)x, d[0]), ly = __dsub_rn((double)y, d[1]), lz = __dsub_rn((double)z, d[2]);
    const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
    const int x0 = (int)flx, y0 = (int)fly, z0 = (int)flz;
    const double fx = __dsub_rn(lx, (double)x0), fy = __dsub_rn(ly, (double)y0), fz = __dsub_rn(lz, (double)z0);
    const int x1 = x0 < nx - 1 ? x0 + 1 : x0, y1 = y0 < ny - 1 ? y0 + 1 : y0, z1 = z0 < nz - 1 ? z0 + 1 : z0;
    bool valid = x0 >= 0 && y0 >= 0 && x0 <= nx - 1 && y0 <= ny - 1;  // isValidPoint (FrameWarper.h:9-21)
    if (nz > 1) valid = valid && z0 >= 0 && z0 <= nz - 1;
    if (!valid) continue;
    const double v = (double)load_raw(img, img_kind, p);
    const double ax = __dsub_rn(1.0, fx), ay = __dsub_rn(1.0, fy), az = __dsub_rn(1.0, fz);
    // (weight y) * (weight x) * (weight z), in the reference's order; zero weights add nothing
    const double wy[2] = {ay, fy}, wx[2] = {ax, fx}, wz[2] = {az, fz};
    const int ty[2] = {y0, y1}, tx[2] = {x0, x1}, tz[2] = {z0, z1};
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
      for (int b = 0; b < 2; b++)
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const double w = __dmul_rn(__dmul_rn(wy[b], wx[c]), wz[a]);
          if (w == 0.0) continue;
          const long long t = ((long long)tz[a] * ny + ty[b]) * nx + tx[c];
          if (wimg != nullptr) atomicAdd(wimg + t, (float)__dmul_rn(w, v));
          atomicAdd(cov + t, (float)w);
        }
  }
}

__device__ __forceinline__ void block_sum(double* v, int n, double* smem) {
  // smem: kMetricThreads * n doubles; thread 0 ends with the sums, in a fixed tree order
  for (int k = 0; k < n; k++) smem[k * kMetricThreads + threadIdx.x] = v[k];
  __syncthreads();
  for (int w = kMetricThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int k = 0; k < n; k++) smem[k * kMetricThreads + threadIdx.x] += smem[k * kMetricThreads + threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < n; k++) v[k] = smem[k * kMetricThreads];
}

// Pass 1 over coverage > 0: count and the sums / sums of squares of the warped frame w, the
// reference r and the unaligned frame f (raw + 1). parts: kMetricBlocks x kMetricTerms.
__global__ void __launch_bounds__(kMetricThreads) metric_sums_kernel(const float* __restrict__ cov,
                                                                     const float* __restrict__ warped,
                                                                     const float* __restrict__ ref,
                                                                     const void* __restrict__ raw, int raw_kind,
                                                                     long long n, double* __restrict__ parts) {
  __shared__ double smem[kMetricThreads * 7];
  double a[7] = {0, 0, 0, 0, 0, 0, 0};
  for (long long i = blockIdx.x * (long long)kMetricThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMetricThreads) {
    if (!(cov[i] > 0.0f)) continue;
    const double w = warped[i], r = ref[i], f = (double)(load_raw(raw, raw_kind, i) + 1.0f);
    a[0] += 1.0;
    a[1] += w;
    a[2] += r;
    a[3] += w * w;
    a[4] += r * r;
    a[5] += f;
    a[6] += f * f;
  }
  block_sum(a, 7, smem);
  if (threadIdx.x == 0)
    for (int k = 0; k < 7; k++) parts[blockIdx.x * kMetricTerms + k] = a[k];
}

// Pass 2: sum (w - mean w)(r - mean r) and sum (f - mean f)(r - mean r); means from pass 1's
// totals in tot[0..7).
__global__ void __launch_bounds__(kMetricThreads) metric_cov_kernel(const float* __restrict__ cov,
                                                                    const float* __restrict__ warped,
                                                                    const float* __restrict__ ref,
                                                                    const void* __restrict__ raw, int raw_kind,
                                                                    long long n, const double* __restrict__ tot,
                                                                    double* __restrict__ parts) {
  __shared__ double smem[kMetricThreads * 2];
  const double cnt = tot[0];
  const double mw = tot[1] / cnt, mr = tot[2] / cnt, mf = tot[5] / cnt;
  double a[2] = {0, 0};
  for (long long i = blockIdx.x * (long long)kMetricThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kMetricThreads) {
    if (!(cov[i] > 0.0f)) continue;
    const double dr = (double)ref[i] - mr;
    a[0] += ((double)warped[i] - mw) * dr;
    a[1] += ((double)(load_raw(raw, raw_kind, i) + 1.0f) - mf) * dr;
  }
  block_sum(a, 2, smem);
  if (threadIdx.x == 0) {
    parts[blockIdx.x * kMetricTerms + 0] = a[0];
    parts[blockIdx.x * kMetricTerms + 1] = a[1];
  }
}

// Sums kMetricBlocks partial rows in block order into out[0..n).
__global__ void metric_total_kernel(const double* __restrict__ parts, int n, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= n) return;
  double s = 0;
  for (int b = 0; b < kMetricBlocks; b++) s += parts[b * kMetricTerms + k];
  out[k] = s;
}

// convertTo(CV_16U): round half to even, saturate to [0, 65535], NaN -> 0; num / den when den is set.
__global__ void to_u16_kernel(const float* __restrict__ num, const float* __restrict__ den, long long n,
                              unsigned short* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float v = den != nullptr ? __fdiv_rn(num[i], den[i]) : num[i];
    int r = v == v ? __float2int_rn(v) : 0;
    r = r < 0 ? 0 : (r > 65535 ? 65535 : r);
    out[i] = (unsigned short)r;
  }
}

// FrameWarpAligner::shiftPixel (FrameWarpAligner.cpp:253-266) for n points: warpPoint
// (FrameWarper.cpp:397-419) is called with the coordinates converted to int (truncation), and points
// outside the volume are not moved.
__global__ void shift_points_kernel(const RefDev* __restrict__ Rp, ScanD sc, const double* __restrict__ D, long long n,
                                    double* __restrict__ px, double* __restrict__ py, double* __restrict__ pz) {
  const RefDev& R = *Rp;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double x = px[k], y = py[k], z = pz[k];
    // int conversion of coordinates that fit in an int; others are outside the volume anyway
    const bool fits = fabs(x) < 2147483647.0 && fabs(y) < 2147483647.0 && fabs(z) < 2147483647.0;
    if (!fits) continue;
    const int xi = (int)x, yi = (int)y, zi = (int)z;
    if (xi < 0 || xi >= R.nx || yi < 0 || yi >= R.ny || zi < 0 || zi >= R.nz) continue;
    int i;
    double f;
    exact_interval(R, sc, xi, yi, zi, &i, &f);
    const double g = __dsub_rn(1.0, f);
    const int nd = R.n_dim;
    double d[3];
#pragma unroll
    for (int c = 0; c < 3; c++)
      d[c] = c < nd ? __dadd_rn(__dmul_rn(f, D[3 * (i + 1) + c]), __dmul_rn(g, D[3 * i + c])) : 0.0;
    px[k] = __dsub_rn(x, d[0]);
    py[k] = __dsub_rn(y, d[1]);
    pz[k] = __dsub_rn(z, d[2]);
  }
}

}  // namespace

cudaError_t launch_shift_points(const RefDev* ref_dev, const double* scan4, const double* D_dev, long long n, double* x,
                                double* y, double* z, cudaStream_t s) {
  const ScanD sc{scan4[0], scan4[1], scan4[2], scan4[3]};
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  shift_points_kernel<<<(int)(blocks < 1 ? 1 : blocks), 256, 0, s>>>(ref_dev, sc, D_dev, n, x, y, z);
  return cudaGetLastError();
}

cudaError_t launch_splat(const RefDev* ref_dev, const RefDev& R, const double* scan4, const void* img, int img_kind,
                         const double* D_dev, float* wimg, float* cov, cudaStream_t s) {
  const ScanD sc{scan4[0], scan4[1], scan4[2], scan4[3]};
  const long long N = R.N;
  cudaError_t e = cudaSuccess;
  if (wimg) e = cudaMemsetAsync(wimg, 0, (size_t)N * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(cov, 0, (size_t)N * sizeof(float), s);
  if (e != cudaSuccess) return e;
  long long blocks = (N + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (R.n_dim == 3)
    splat_kernel<3><<<(int)blocks, 256, 0, s>>>(ref_dev, sc, img, img_kind, D_dev, wimg, cov);
  else
    splat_kernel<2><<<(int)blocks, 256, 0, s>>>(ref_dev, sc, img, img_kind, D_dev, wimg, cov);
  return cudaGetLastError();
}

// totals[0..7): count, sums of pass 1; totals[8..10): the two covariance sums.
cudaError_t launch_metrics(const float* cov, const float* warped, const float* ref, const void* raw, int raw_kind,
                           long long n, double* parts, double* totals, cudaStream_t s) {
  metric_sums_kernel<<<kMetricBlocks, kMetricThreads, 0, s>>>(cov, warped, ref, raw, raw_kind, n, parts);
  metric_total_kernel<<<1, 32, 0, s>>>(parts, 7, totals);
  metric_cov_kernel<<<kMetricBlocks, kMetricThreads, 0, s>>>(cov, warped, ref, raw, raw_kind, n, totals, parts);
  metric_total_kernel<<<1, 32, 0, s>>>(parts, 2, totals + 8);
  return cudaGetLastError();
}

cudaError_t launch_to_u16(const float* num, const float* den, long long n, unsigned short* out, cudaStream_t s) {
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  to_u16_kernel<<<(int)(blocks < 1 ? 1 : blocks), 256, 0, s>>>(num, den, n, out);
  return cudaGetLastError();
}

}  // namespace fa

// ================================================================== host side =====================

namespace {

void scan4_of(const fa_reference* R, double* scan4) {
  const fa_scan_params p = process_scan(R->scan, R->nz, R->nD);
  scan4[0] = p.pixel_duration;
  scan4[1] = p.interline_duration;
  scan4[2] = p.interframe_duration;
  scan4[3] = p.stack_duration;
}

// correlation() (Cv3dUtils.cpp:57-81) from the metric totals: population standard deviations,
// covariance as the masked mean of the centred product.
double correlation_from(const double* t, int which) {
  const double cnt = t[0];
  if (cnt == 0) return 0.0;
  const double sa = which == 0 ? t[1] : t[5], saa = which == 0 ? t[3] : t[6];
  const double ma = sa / cnt, mb = t[2] / cnt;
  const double va = saa / cnt - ma * ma, vb = t[4] / cnt - mb * mb;
  const double sda = std::sqrt(va > 0 ? va : 0), sdb = std::sqrt(vb > 0 ? vb : 0);
  const double cv = t[8 + which] / cnt;
  return cv / (sda * sdb);
}

fa_status results_reserve(fa_aligner* A, fa_dtype dtype) {
  if (A->res_slot) return FA_OK;
  fa_reference* R = A->ref;
  const size_t N = (size_t)R->N;
  FA_TRY(frame_alloc(R, fa::kFrameF32, &A->res_slot));
  FA_TRY(dalloc(A->ctx, N * sizeof(float), &A->res_raw, A->res_allocs));  // room for FA_F32 or FA_U16
  FA_TRY(dalloc_t(A->ctx, N, &A->res_wimg, A->res_allocs));
  FA_TRY(dalloc_t(A->ctx, N, &A->res_cov, A->res_allocs));
  FA_TRY(dalloc_t(A->ctx, N, &A->res_warp, A->res_allocs));
  FA_TRY(dalloc_t(A->ctx, N, &A->res_u16, A->res_allocs));
  FA_TRY(dalloc_t(A->ctx, (size_t)R->nD * 3, &A->res_D, A->res_allocs));
  FA_TRY(dalloc_t(A->ctx, (size_t)296 * 8 + 16, &A->res_parts, A->res_allocs));
  (void)dtype;
  return FA_OK;
}

}  // namespace

namespace fa_rt {

void aligner_release_results(fa_aligner* A) {
  if (A->res_slot) fa_deregister_frame(A->res_slot);
  A->res_slot = nullptr;
  dfree_all(A->ctx, A->res_allocs);
  A->res_raw = nullptr;
  A->res_wimg = A->res_cov = A->res_warp = nullptr;
  A->res_u16 = nullptr;
  A->res_D = A->res_parts = nullptr;
}

}  // namespace fa_rt

extern "C" fa_status fa_warp_image(fa_reference* R, const float* frame, const double* D, float* wimg,
                                   float* coverage) {
  if (!R || !frame || !D || !coverage) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (!finite_all(D, (size_t)R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  FA_CU(cudaSetDevice(R->ctx->device));
  const size_t N = (size_t)R->N;
  std::vector<Alloc> tmp;
  float *img, *w, *c;
  double* Dd;
  auto done = [&](fa_status st) {
    std::string keep = g_err;
    cudaStreamSynchronize(R->stream);
    dfree_all(R->ctx, tmp);
    g_err = keep;
    return st;
  };
  fa_status st;
  if ((st = dalloc_t(R->ctx, N, &img, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, N, &w, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, N, &c, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, (size_t)R->nD * 3, &Dd, tmp)) != FA_OK) return done(st);
  double scan4[4];
  scan4_of(R, scan4);
  cudaStream_t s = R->stream;
  cudaError_t e = cudaMemcpyAsync(img, frame, N * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Dd, D, (size_t)R->nD * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = fa::launch_splat(R->dev, R->host, scan4, img, FA_F32, Dd, wimg ? w : nullptr, c, s);
  g_launches += 1;
  if (e == cudaSuccess && wimg) e = cudaMemcpyAsync(wimg, w, N * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(coverage, c, N * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("warp image: ") + cudaGetErrorString(e)));
  return done(FA_OK);
}

extern "C" fa_status fa_aligner_results(fa_aligner* A, const void* const* frames, fa_dtype dtype, int n,
                                        const double* D, fa_frame_result* results, uint16_t* const* realigned,
                                        uint16_t* const* realigned_preserving, float* const* mask) {
  if (!A) return fail(FA_ERR_BAD_ARG, "NULL aligner");
  std::lock_guard<std::mutex> lk(A->mu);
  if (!A->ref) return fail(FA_ERR_STATE, "Reference imaging not yet set");
  if (!frames || n <= 0 || !D) return fail(FA_ERR_BAD_ARG, "bad arguments");
  if (dtype != FA_F32 && dtype != FA_U16) return fail(FA_ERR_BAD_ARG, "frames must be FA_F32 or FA_U16");
  fa_reference* R = A->ref;
  if (!finite_all(D, (size_t)n * R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  FA_CU(cudaSetDevice(A->ctx->device));
  FA_TRY(results_reserve(A, dtype));
  const long long N = R->N;
  double scan4[4];
  scan4_of(R, scan4);
  fa_frame* F = A->res_slot;
  cudaStream_t s = F->stream;
  std::vector<float4> hdp((size_t)R->nD * fa::kDParamF4);
  double totals[16];
  for (int k = 0; k < n; k++) {
    if (!frames[k]) return fail(FA_ERR_BAD_ARG, "NULL frame pointer");
    const double* Dk = D + (size_t)k * R->nD * 3;
    make_dparams(Dk, R->nD, R->n_dim, hdp.data());
    FA_CU(cudaMemcpyAsync(A->res_raw, frames[k], (size_t)N * dtype_size(dtype), cudaMemcpyHostToDevice, s));
    FA_CU(cudaMemcpyAsync(A->res_D, Dk, (size_t)R->nD * 3 * sizeof(double), cudaMemcpyHostToDevice, s));
    FA_CU(cudaMemcpyAsync(F->job.dparams, hdp.data(), hdp.size() * sizeof(float4), cudaMemcpyHostToDevice, s));
    // getMask / getWarpedFrame: splat of the raw frame (FrameWarpAligner.cpp:317-326, 340-346)
    const bool want_wimg = realigned_preserving && realigned_preserving[k];
    FA_CU(fa::launch_splat(R->dev, R->host, scan4, A->res_raw, dtype, A->res_D, want_wimg ? A->res_wimg : nullptr,
                           A->res_cov, s));
    // warped_smoothed: warpImageInterpolated of the (smoothed) frame + 1, invalid value 0 (:223);
    // the unaligned correlation uses the same frame
    const void* fsm = A->res_raw;
    fa_dtype fsm_type = dtype;
    if (A->prm.smoothing > 0) {
      FA_TRY(aligner_smooth(A, A->res_raw, dtype, s));
      fsm = A->smooth_out;
      fsm_type = FA_F32;
    }
    FA_CU(fa::launch_to_slot(fsm, fsm_type, F->data, fa::kFrameF32, R->nz, R->ny, R->nx, F->job.fpitch, F->job.fplane,
                             true, s));
    FA_CU(fa::launch_warp(R->dev, R->host, F->data, F->job.fplane, F->job.fpitch, fa::kFrameF32, F->job.dparams,
                          0.0f, A->res_warp, s));
    FA_CU(fa::launch_metrics(A->res_cov, A->res_warp, R->host.ref32, fsm, fsm_type, N, A->res_parts,
                             A->res_parts + 296 * 8, s));
    g_launches += 7;
    if (results) FA_CU(cudaMemcpyAsync(totals, A->res_parts + 296 * 8, 16 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (mask && mask[k])
      FA_CU(cudaMemcpyAsync(mask[k], A->res_cov, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (want_wimg) {
      FA_CU(fa::launch_to_u16(A->res_wimg, A->res_cov, N, A->res_u16, s));
      FA_CU(cudaMemcpyAsync(realigned_preserving[k], A->res_u16, (size_t)N * 2, cudaMemcpyDeviceToHost, s));
      g_launches += 1;
    }
    if (realigned && realigned[k]) {
      // getInterpolatedWarpedFrame: warpImageInterpolated of the raw frame (:328-338); the buffers
      // reused here are read by earlier work on the same stream first
      FA_CU(fa::launch_to_slot(A->res_raw, dtype, F->data, fa::kFrameF32, R->nz, R->ny, R->nx, F->job.fpitch,
                               F->job.fplane, false, s));
      FA_CU(fa::launch_warp(R->dev, R->host, F->data, F->job.fplane, F->job.fpitch, fa::kFrameF32, F->job.dparams,
                            0.0f, A->res_warp, s));
      FA_CU(fa::launch_to_u16(A->res_warp, nullptr, N, A->res_u16, s));
      FA_CU(cudaMemcpyAsync(realigned[k], A->res_u16, (size_t)N * 2, cudaMemcpyDeviceToHost, s));
      g_launches += 3;
    }
    FA_CU(cudaStreamSynchronize(s));
    if (results) {
      fa_frame_result& r = results[k];
      r.correlation = correlation_from(totals, 0);
      r.unaligned_correlation = correlation_from(totals, 1);
      r.coverage = totals[0] / (double)N;
      r.use_frame = (r.correlation >= A->prm.correlation_threshold && r.coverage >= A->prm.coverage_threshold) ? 1 : 0;
    }
  }
  return FA_OK;
}

extern "C" fa_status fa_shift_pixels(fa_reference* R, const double* D, long long n, double* x, double* y, double* z) {
  if (!R || !D || n < 0 || (n > 0 && (!x || !y || !z))) return fail(FA_ERR_BAD_ARG, "bad arguments");
  if (n == 0) return FA_OK;
  if (!finite_all(D, (size_t)R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  FA_CU(cudaSetDevice(R->ctx->device));
  std::vector<Alloc> tmp;
  double *dx, *dy, *dz, *Dd;
  auto done = [&](fa_status st) {
    std::string keep = g_err;
    cudaStreamSynchronize(R->stream);
    dfree_all(R->ctx, tmp);
    g_err = keep;
    return st;
  };
  fa_status st;
  if ((st = dalloc_t(R->ctx, (size_t)n, &dx, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, (size_t)n, &dy, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, (size_t)n, &dz, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(R->ctx, (size_t)R->nD * 3, &Dd, tmp)) != FA_OK) return done(st);
  double scan4[4];
  scan4_of(R, scan4);
  cudaStream_t s = R->stream;
  const size_t b = (size_t)n * sizeof(double);
  cudaError_t e = cudaMemcpyAsync(dx, x, b, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dy, y, b, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dz, z, b, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Dd, D, (size_t)R->nD * 3 * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = fa::launch_shift_points(R->dev, scan4, Dd, n, dx, dy, dz, s);
  g_launches += 1;
  if (e == cudaSuccess) e = cudaMemcpyAsync(x, dx, b, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(y, dy, b, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(z, dz, b, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("shift pixels: ") + cudaGetErrorString(e)));
  return done(FA_OK);
}

extern "C" fa_status fa_write_realignment_info(const char* filename, const fa_scan_params* image_params, int n_frames,
                                               int nD, const double* D, const fa_frame_result* results) {
  if (!filename || !image_params || n_frames < 0 || nD < 1 || (n_frames > 0 && (!D || !results)))
    return fail(FA_ERR_BAD_ARG, "bad arguments");
  if (n_frames == 0) return FA_OK;  // the reference writes nothing without frames
  std::ofstream os(filename);
  if (!os) return fail(FA_ERR_BAD_ARG, std::string("cannot open ") + filename);
  // FrameWarpAligner::writeRealignmentInfo (FrameWarpAligner.cpp:288-314), default stream formatting
  os << "Realignment Information Version, 2\n";
  os << "Line Duration," << image_params->line_duration << "\n";
  os << "Interline Duration," << image_params->interline_duration << "\n";
  os << "Frame Duration," << image_params->frame_duration << "\n";
  os << "Interframe Duration," << image_params->interframe_duration << "\n";
  os << "Lines," << image_params->n_y << "\n";
  os << "Frames Per Stack," << image_params->n_z << "\n";
  os << "Frame, UnalignedCorrelation, Correlation, Coverage";
  for (int j = 0; j < nD; j++) os << ", dx_" << j << ", dy_" << j << ", dz_" << j;
  os << "\n";
  for (int i = 0; i < n_frames; i++) {
    os << i << "," << results[i].unaligned_correlation << "," << results[i].correlation << ", " << results[i].coverage;
    for (int j = 0; j < nD; j++) {
      const double* d = D + ((size_t)i * nD + j) * 3;
      os << ", " << d[0] << ", " << d[1] << ", " << d[2];
    }
    os << "\n";
  }
  if (!os) return fail(FA_ERR_CUDA, "write failed");
  return FA_OK;
}
