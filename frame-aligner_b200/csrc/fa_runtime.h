// fa_runtime.h -- host runtime state shared by the C ABI translation units (fa_api.cu, fa_server.cu):
// the opaque handle types of include/fa_b200.h, device allocation under the context budget, error
// reporting, and the helpers the serving loop reuses from the single-aligner path.
#pragma once

#include <cufft.h>

#include <atomic>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "fa_kernels.cuh"

namespace fa_rt {

// Last error message of the calling thread (fa_last_error) and the count of this library's kernel
// launches (fa_kernel_launches).
extern thread_local std::string g_err;
extern std::atomic<long long> g_launches;

// Records msg as the calling thread's last error and returns s.
fa_status fail(fa_status s, const std::string& msg);

#define FA_CU(call)                                                                                       \
  do {                                                                                                    \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess) return fa_rt::fail(FA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define FA_TRY(call)            \
  do {                          \
    fa_status s_ = (call);      \
    if (s_ != FA_OK) return s_; \
  } while (0)

struct Alloc {
  void* p;
  size_t n;
};

// Exact scan geometry, computed on the host in double with the reference's expressions
// (FrameWarper.cpp:252-283), without per-voxel tables.
struct Geometry {
  int nz, ny, nx, nD, n_rows;
  long long N;
  std::vector<long long> scan_begin;  // first scan index of interval k (k = 0..nD-2)
  std::vector<int> begin, end;        // storage D_range
  std::vector<fa::RowDesc> rows;
  float dq;
  long long lmin;
  int tile_rows, n_tiles;
  std::vector<int> tile_c0;
  std::vector<int2> ctrl_tiles;
};

}  // namespace fa_rt

struct fa_context {
  int device = 0;
  int autotune = 0;
  size_t budget = 0;
  std::atomic<size_t> used{0};
  std::mutex mu;
};

struct fa_reference {
  fa_context* ctx = nullptr;
  int nz = 0, ny = 0, nx = 0, nD = 0, n_dim = 0, P = 0;
  long long N = 0;
  fa_precision prec = FA_PREC_F32;
  fa_scan_params scan{};
  fa_rt::Geometry G;
  int* tile_c0_dev = nullptr;
  int2* ctrl_dev = nullptr;
  std::vector<double> hd, hl;  // host copies of the Hessian blocks (diagonal, sub-diagonal)
  fa::RefDev host{};
  fa::RefDev* dev = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<fa_rt::Alloc> allocs;
  std::atomic<int> n_frames{0};
};

struct fa_frame {
  fa_reference* ref = nullptr;
  void* data = nullptr;
  int kind = fa::kFrameF32;
  cudaStream_t stream = nullptr;
  fa::Job job{};
  fa::Job* job_dev = nullptr;
  fa::FrameState* state = nullptr;
  double* h_result = nullptr;  // pinned: [f, g(P)]
  float4* h_dparams = nullptr;  // pinned: nD * 3
  double* h_x = nullptr;        // pinned: P
  fa::FrameState* h_state = nullptr;  // pinned
  float* warp_out = nullptr;
  std::vector<double> lastD;
  std::vector<double> last_g;
  double last_f = 0;
  bool have_last = false;
  std::mutex mu;
  std::vector<fa_rt::Alloc> allocs;
};

struct fa_correlator {
  fa_context* ctx = nullptr;
  int nz = 0, ny = 0, nx = 0;
  long long n_el = 0, n_complex = 0;
  int cap = 0;                          // most frames per batched FFT (a power of two)
  // D2Z / Z2D plans per batch size (powers of two up to cap), made on first use; they share one work
  // area (they run one after another on the correlator's stream)
  std::map<int, std::pair<cufftHandle, cufftHandle>> plans;
  void* work = nullptr;
  size_t work_bytes = 0;
  std::vector<fa_rt::Alloc> work_allocs;
  // fused kx-plane passes (fa_plane_corr.cu) when the dimensions allow them; cuFFT otherwise
  bool planes = false;
  fa::PlaneDims pd{};
  double2* tw_x = nullptr;              // W_nx^m, m < nx
  double2* tw_y = nullptr;              // W_ny^m, m < ny
  double2* tw_z = nullptr;              // W_nz^m, m < nz (split (z, y) pass only)
  cudaStream_t stream = nullptr;
  double* wy = nullptr;                 // square-root Hann window along y
  double* wx = nullptr;                 // ... and along x (1 along z)
  double* real = nullptr;               // cap * n_el (cuFFT path only)
  double2* spec = nullptr;              // cap * n_complex
  double2* ref_conj = nullptr;          // n_complex (planes [kx][z][y] when `planes`, else cuFFT's order)
  double2* ref_conj_rows = nullptr;     // cuFFT's order, made when a plane-path correlator falls back
  float* vol = nullptr;                 // one host-uploaded volume
  const void** d_ptrs = nullptr;        // device array of input pointers, then (from ptr_cap) slot pointers
  const void** h_ptrs = nullptr;        // pinned staging of the same
  int ptr_cap = 0;
  double* bval = nullptr;
  long long* bidx = nullptr;
  long long* d_idx = nullptr;           // one peak index per frame (ptr_cap)
  long long* h_idx = nullptr;
  int n_blocks = 0;                     // argmax blocks per frame (cuFFT path)
  std::mutex mu;
  std::vector<fa_rt::Alloc> allocs;
  std::vector<fa_rt::Alloc> ptr_allocs;
};

namespace fa_rt {

// Device buffers, a pinned active count and the instantiated graph of a batched solve, kept
// between calls on the same frames (in the same order) with the same solve geometry.
struct BatchCache {
  std::vector<Alloc> allocs;
  fa::Job* jobs_dev = nullptr;
  int* d_active = nullptr;  // [0] active frames, [1] rounds of the device-side loop
  int* d_list = nullptr;
  int* d_prefix = nullptr;
  int* h_rounds = nullptr;  // pinned: rounds the last solve ran
  int per_round = 0;        // kernel launches per round
  int cap = 0;
  cudaGraphExec_t exec = nullptr;
  std::vector<fa_frame*> frames;  // the frames the graph was captured for
  long long key[7] = {0, 0, 0, 0, 0, 0, 0};
};
// Frees the cache's buffers and graph (after the caller's streams are idle).
void batch_cache_release(fa_context* ctx, BatchCache* c);

}  // namespace fa_rt

struct fa_aligner {
  fa_context* ctx = nullptr;
  fa_aligner_params prm{};
  fa_reference* ref = nullptr;
  fa_correlator* corr = nullptr;
  int nz = 0, ny = 0, nx = 0, nD = 0;
  int dz = 0, dy = 0, dx = 0;  // downsampled dims
  cudaStream_t stream = nullptr;
  std::vector<fa_frame*> slots;
  int slot_kind = -1;
  void* staging = nullptr;     // raw frames copied from the host when they need a conversion pass
  size_t staging_bytes = 0;
  float* vols = nullptr;       // downsampled frames for the correlator (spatial_binning > 1)
  size_t vols_count = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev_corr = nullptr;
  double last_ms = 0;
  double last_corr_ms = 0;  // of last_ms: until the last frame's conversion and phase correlation
  // host frames: uploads on their own stream, one event per chunk of frames
  cudaStream_t copy_stream = nullptr;
  std::vector<cudaEvent_t> copy_ev;
  std::vector<cudaEvent_t> group_ev;  // peaks of a group of frames read back
  std::deque<fa_rt::BatchCache> batch_cache;  // the batched solve's buffers and graph per solve group
  // smoothStack (smoothing > 0): Gaussian weights along x and y, and two frame-sized work buffers
  // used one frame at a time in stream order
  float* smooth_kx = nullptr;
  float* smooth_ky = nullptr;
  int smooth_nkx = 0, smooth_nky = 0;
  float* smooth_tmp = nullptr;
  float* smooth_out = nullptr;
  std::vector<fa_rt::Alloc> smooth_allocs;
  // per-frame outputs and metrics (fa_aligner_results): an FP32 frame slot and work buffers
  fa_frame* res_slot = nullptr;
  void* res_raw = nullptr;
  float* res_wimg = nullptr;
  float* res_cov = nullptr;
  float* res_warp = nullptr;
  unsigned short* res_u16 = nullptr;
  double* res_D = nullptr;
  double* res_parts = nullptr;
  std::vector<fa_rt::Alloc> res_allocs;
  std::vector<fa_rt::Alloc> allocs;   // staging / vols
  std::vector<fa_rt::Alloc> ref_allocs;
  std::mutex mu;
};

namespace fa_rt {

// cudaMalloc of bytes charged to the context's budget; the block is recorded in owner.
fa_status dalloc(fa_context* ctx, size_t bytes, void** out, std::vector<Alloc>& owner);
template <typename T>
fa_status dalloc_t(fa_context* ctx, size_t count, T** out, std::vector<Alloc>& owner) {
  void* p = nullptr;
  FA_TRY(dalloc(ctx, count * sizeof(T), &p, owner));
  *out = static_cast<T*>(p);
  return FA_OK;
}
// Frees every block in owner and returns its bytes to the budget.
void dfree_all(fa_context* ctx, std::vector<Alloc>& owner);

size_t dtype_size(fa_dtype t);
// ImageScanParameters after AbstractFrameWarper::processScanParameters.
fa_scan_params process_scan(const fa_scan_params& in, int nz, int nD);
// Control-point parameters of the fused pass (3 float4 per control point) from D (nD x 3 doubles).
void make_dparams(const double* D, int nD, int n_dim, float4* out);
bool finite_all(const double* v, size_t n);
// Frees the buffers of fa_aligner_results (with the aligner's reference).
void aligner_release_results(fa_aligner* A);
// cv::GaussianBlur's float kernel for sigma (the size rule and weights of smoothStack's blur); empty
// when it would exceed 257 taps.
std::vector<float> gaussian_kernel(double sigma);
// smoothStack of one dense raw frame (device) into A->smooth_out on stream s (no-op without smoothing).
fa_status aligner_smooth(fa_aligner* A, const void* raw, fa_dtype dtype, cudaStream_t s);
// Frame slot (zero-halo storage of the given FrameKind + solve buffers + stream) for reference R.
fa_status frame_alloc(fa_reference* R, int kind, fa_frame** out);
// Slot storage the aligner uses for frames of dtype (raw uint16 counts + 1, FP16 or FP32 values + 1).
int slot_kind_for(const fa_aligner* A, fa_dtype dtype);
// The correlator's D2Z / Z2D plans for a batch size (made and cached on first use).
fa_status correlator_plans(fa_correlator* C, int batch, cufftHandle* fwd, cufftHandle* inv);
// Window, forward DFT, normalisation, inverse DFT and argmax for n device volumes; peak indices to
// C->d_idx[first .. first + n). surface (n * n_el doubles, optional) receives the correlation
// surfaces; planes selects the fused kx-plane passes (when C->planes) or cuFFT. Calls with
// first > 0 use pointer and result slots reserved before (correlator_reserve(C, first + n)), so
// that consecutive calls queue on the stream without waiting for one another.
// With `slots` (n interior pointers of frame slots of `slot_kind` with the given pitch and plane),
// the plane path also writes each frame + 1 into its slot as it reads it (*slots_written = true);
// on the cuFFT path it does not, and the caller converts the frames itself.
fa_status correlator_enqueue(fa_correlator* C, const void* const* vols, int in_kind, int n,
                             double* surface = nullptr, bool planes = true, int first = 0,
                             void* const* slots = nullptr, int slot_kind = 0, int slot_pitch = 0,
                             long long slot_plane = 0, bool* slots_written = nullptr);
// Pointer staging and peak slots for n volumes (grows with a stream synchronisation).
fa_status correlator_reserve(fa_correlator* C, int n);
// Peak index -> signed integer shift (x, y, z).
void unravel_shift(const fa_correlator* C, long long idx, double* shift);

}  // namespace fa_rt
