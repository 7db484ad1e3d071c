// fa_noalloc.cu -- fa_get_error_jacobian_static: the fused error + J^T e evaluation of one frame
// with all of its scratch in a fixed, file-scope device array, so that the call itself allocates no
// device or pinned memory.
//
// Why: some callers cannot call cudaMalloc at the time they evaluate a frame -- for example a host
// application that has reserved the whole device memory pool for its own allocator before loading
// this library, or a real-time acquisition loop that must not pay for (or risk failing) an
// allocation between frames. They register the reference once (that call allocates) and keep their
// frames in memory they own; this entry point then needs nothing else.
//
// The array below (kStaticScratchBytes) holds the job descriptor, the control-point parameters, the
// per-tile partial sums and the reduced result. Every GPU that loads the library holds it until the
// process exits. Its address is looked up once per device with cudaGetSymbolAddress on the first
// call made with that device current; make that first call before any stream capture.
#include <cstdio>
#include <mutex>

#include "fa_kernels.cuh"

namespace {

constexpr size_t kStaticScratchBytes = size_t(2) << 20;  // 2 MiB

// Host code never dereferences this name: it is a host-side stand-in for the device array. The
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace

// Internal accessors into fa_api.cu (the reference layout is private to the runtime).
namespace fa {
fa_status static_eval_prepare(const fa_reference* ref, const double* D, const RefDev** dev, const RefDev** host, int* nD,
                              int* n_dim, bool* mixed, int* device);
fa_status static_eval_fail(fa_status s, const char* msg);
void static_eval_dparams(const double* D, int nD, int n_dim, float4* out);
void static_eval_count_launches(int n);
}  // namespace fa

extern "C" fa_status fa_get_error_jacobian_static(const fa_reference* ref, const void* frame_device, fa_dtype dtype,
                                                  const double* D, double* f, double* jac) {
  const fa::RefDev* dev = nullptr;
  const fa::RefDev* host = nullptr;
  int nD = 0, n_dim = 0;
  bool mixed = false;
  int device = 0;
  if (!ref || !frame_device || !D || !f || !jac) return fa::static_eval_fail(FA_ERR_BAD_ARG, "NULL argument");
  fa_status st = fa::static_eval_prepare(ref, D, &dev, &host, &nD, &n_dim, &mixed, &device);
  if (st != FA_OK) return st;
  if (dtype != (mixed ? FA_F16 : FA_F32))
    return fa::static_eval_fail(FA_ERR_BAD_ARG, mixed ? "a mixed-precision reference needs FA_F16 frames"
                                                      : "an FP32 reference needs FA_F32 frames");
  // Layout inside the array: Job | dparams (nD*3 float4) | result (1+P doubles) | tile partials.
  const int P = nD * n_dim;
  const size_t off_dp = align256(sizeof(fa::Job));
  const size_t off_res = off_dp + align256((size_t)nD * fa::kDParamF4 * sizeof(float4));
  const size_t off_parts = off_res + align256((size_t)(1 + P) * sizeof(double));
  const size_t need = off_parts + (size_t)host->n_tiles * fa::kPartialDoubles * sizeof(double);
  if (need > kStaticScratchBytes) {
    char m[160];
    std::snprintf(m, sizeof(m), "volume needs %zu bytes of static scratch (%d tiles); the maximum is %zu bytes", need,
                  host->n_tiles, kStaticScratchBytes);
    return fa::static_eval_fail(FA_ERR_BAD_ARG, m);
  }
  if (device < 0 || device >= kMaxDevices) return fa::static_eval_fail(FA_ERR_BAD_ARG, "device ordinal out of range");
  // The work runs with the reference's device current; the caller's current device is restored on
  // every return.
  int caller_device = -1;
  if (cudaGetDevice(&caller_device) != cudaSuccess) return fa::static_eval_fail(FA_ERR_CUDA, "cudaGetDevice failed");
  struct RestoreDevice {
    int d;
    ~RestoreDevice() { cudaSetDevice(d); }
  } restore{caller_device};
  if (cudaSetDevice(device) != cudaSuccess) return fa::static_eval_fail(FA_ERR_CUDA, "cudaSetDevice failed");
  char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[device]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
      if (e != cudaSuccess) {
        char m[160];
        std::snprintf(m, sizeof(m), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return fa::static_eval_fail(FA_ERR_CUDA, m);
      }
      g_addr[device] = p;
    }
    base = static_cast<char*>(g_addr[device]);
  }
  fa::Job job{};
  job.ref = dev;
  job.frame = frame_device;
  job.fplane = (long long)host->nx * host->ny;  // the caller's dense frame, no halo
  job.fpitch = host->nx;
  job.fpad = 0;
  job.dparams = reinterpret_cast<float4*>(base + off_dp);
  job.result = reinterpret_cast<double*>(base + off_res);
  job.partials = reinterpret_cast<double*>(base + off_parts);
  job.state = nullptr;
  // Every scratch word the kernels read is written earlier in this call (the job, the parameters,
  // each tile's partials, the result), so nothing needs clearing between calls. Host staging uses a
  // fixed stack buffer: the successful path allocates neither device nor host memory.
  cudaError_t e = cudaMemcpy(base, &job, sizeof(job), cudaMemcpyHostToDevice);
  constexpr int kChunk = 64;
  float4 dp[kChunk * fa::kDParamF4];
  double D_chunk[(kChunk + 1) * 3];
  for (int k0 = 0; k0 < nD && e == cudaSuccess; k0 += kChunk) {
    const int k1 = (k0 + kChunk < nD) ? k0 + kChunk : nD;
    // control points [k0, k1] (one past the chunk: the parameters hold D[k+1] - D[k])
    const int kk = (k1 < nD) ? k1 + 1 : k1;
    for (int k = k0; k < kk; k++)
      for (int c = 0; c < 3; c++) D_chunk[(k - k0) * 3 + c] = D[k * 3 + c];
    float4 tmp[(kChunk + 1) * fa::kDParamF4];
    fa::static_eval_dparams(D_chunk, kk - k0, n_dim, tmp);
    for (int i = 0; i < (k1 - k0) * fa::kDParamF4; i++) dp[i] = tmp[i];
    e = cudaMemcpy(job.dparams + (size_t)k0 * fa::kDParamF4, dp, (size_t)(k1 - k0) * fa::kDParamF4 * sizeof(float4),
                   cudaMemcpyHostToDevice);
  }
  const fa::Job* jd = reinterpret_cast<const fa::Job*>(base);
  // The four-voxels-per-lane kernel needs rows of a multiple of 4 voxels and a 16-byte aligned frame;
  // it runs with the register budget the reference's tile shape was tuned for.
  const bool vec4 = host->nx % 4 == 0 && (reinterpret_cast<uintptr_t>(frame_device) & 15u) == 0;
  if (e == cudaSuccess)
    e = fa::launch_eval(jd, 1, host->n_tiles, n_dim, dtype == FA_F16 ? fa::kFrameF16 : fa::kFrameF32, mixed, 0, vec4,
                        host->tune_mb_small);
  if (e == cudaSuccess) e = fa::launch_reduce(jd, *host, 0);
  if (e == cudaSuccess) e = cudaMemcpy(f, job.result, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(jac, job.result + 1, (size_t)P * sizeof(double), cudaMemcpyDeviceToHost);
  fa::static_eval_count_launches(2);
  if (e != cudaSuccess) {
    char m[160];
    std::snprintf(m, sizeof(m), "static evaluation: %s", cudaGetErrorString(e));
    return fa::static_eval_fail(FA_ERR_CUDA, m);
  }
  return FA_OK;
}
