// fa_kernels.cuh -- kernel launch declarations (implemented in fa_kernels.cu, fa_solve.cu).
#pragma once

#include <vector>

#include "fa_internal.h"

namespace fa {

constexpr int kEvalThreads = 256;
constexpr int kEvalWarps = kEvalThreads / 32;
constexpr int kSolveThreads = 128;

// Exact float Sobel3d (Sobel3d.cpp:60-85) of an FP32 volume.
cudaError_t launch_sobel(const float* m, int nz, int ny, int nx, float* gx, float* gy, float* gz,
                         cudaStream_t s);

// Per-tile Hessian partials (exact Df per voxel, FP32 products, FP64 sums) and their reduction
// into Hd / Hl. scan4 = {pixel, interline, interframe, stack} durations after processing.
cudaError_t launch_hessian(const RefDev* ref_dev, const RefDev& ref_host, const double* scan4, double* tile_parts,
                           double* Hd, double* Hl, cudaStream_t s);

// FP32 -> BF16 copy.
cudaError_t launch_to_bf16(const float* in, __nv_bfloat16* out, long long n, cudaStream_t s);
// FP32 reference and gradient planes -> the interleaved BF16 groups of RefDev::q16 (ceil(n / 4) * 16
// values; entries past the volume are zero).
cudaError_t launch_to_quad16(const float* ref, const float* gx, const float* gy, const float* gz, long long n,
                             __nv_bfloat16* q16, cudaStream_t s);
// Any input dtype -> FP32 or FP16 frame storage.
cudaError_t launch_convert(const void* in, fa_dtype in_type, void* out, fa_dtype out_type, long long n,
                           cudaStream_t s);

// Dense frame (any dtype) -> a frame slot's interior (pitch / plane stride), optionally with +1.
cudaError_t launch_to_slot(const void* in, fa_dtype in_type, void* out, int out_kind, int nz, int ny, int nx,
                           int fpitch, long long fplane, bool add_one, cudaStream_t s);

// Raw frame -> storage with the +1 offset; raw -> downsampled float (block sums).
cudaError_t launch_offset_convert(const void* in, fa_dtype in_type, void* out, fa_dtype out_type, long long n,
                                  cudaStream_t s);
cudaError_t launch_downsample(const void* in, fa_dtype in_type, int nz, int ny, int nx, int b, float* out,
                              cudaStream_t s);

// smoothStack: per-plane Gaussian of a dense frame (kx: nkx weights along x, ky: nky along y; tmp and
// out: nz*ny*nx floats).
cudaError_t launch_smooth(const void* in, fa_dtype in_type, int nz, int ny, int nx, const float* kx, int nkx,
                          const float* ky, int nky, float* tmp, float* out, cudaStream_t s);

// Fused warp + error + J^T e over all tiles of n_jobs frames (grid.y = job). frame_kind is a
// FrameKind, ref_bf16 selects the BF16 reference/gradient copies, rows_multiple_of_4 the
// four-voxels-per-lane kernel (every job's nx % 4 == 0).
cudaError_t launch_eval(const Job* jobs_dev, int n_jobs, int max_tiles, int n_dim, int frame_kind, bool ref_bf16,
                        cudaStream_t s, bool rows_multiple_of_4, int mb = 2);

// Persistent fused pass over the compacted active list: grid CTAs walk the (active[a], tile) items,
// item = tile_prefix[a] + tile for a < *n_active, so frames of different sizes share one launch
// (rows must be multiples of 4). most_items bounds the grid.
cudaError_t launch_eval4_active(const Job* jobs_dev, const int* active, const int* n_active, const int* tile_prefix,
                                long long most_items, int n_dim, int frame_kind, bool ref_bf16, int mb, int grid,
                                cudaStream_t s);

// Thread-local (spill) bytes of that kernel's instantiation for a register budget of mb CTAs per SM.
size_t eval4_active_local_bytes(int n_dim, int frame_kind, bool ref_bf16, int mb);

// Rebuilds the active list of a job table (frames not done, ascending index), the exclusive prefix
// sum of their tile counts (tile_prefix[*n_active] = items of the next fused pass), and, when busy is
// non-null, appends frames that are done and still busy to done_list[*n_done...] and clears busy.
cudaError_t launch_compact(const Job* jobs_dev, int n_jobs, int* active, int* n_active, int* tile_prefix, int* busy,
                           int* done_list, int* n_done, cudaStream_t s);

// Initialises the solve state of n frames (zero start, optional rigid and warm starts) and marks them busy.
// Loop control inside a while-conditional graph body: ++*rounds, and the body repeats while
// *n_active > 0 and *rounds < max_rounds.
cudaError_t launch_loop_control(cudaGraphConditionalHandle h, const int* n_active, int* rounds, int max_rounds,
                                cudaStream_t s);
// Zero / paired start of n jobs from phase-correlation peak indices in device memory (correlator
// dims cnz x cny x cnx, x and y scaled by the binning).
cudaError_t launch_activate_peaks(const Job* jobs_dev, int n, const long long* peaks, int cnx, int cny, int cnz,
                                  int binning, int max_iter, bool pair, cudaStream_t s);
cudaError_t launch_activate(const Job* jobs_dev, const Activation* recs, int n, int* busy, cudaStream_t s);

// Reduces one job's tile partials into result = [f, g(P)] (deterministic order).
cudaError_t launch_reduce(const Job* job_dev, const RefDev& ref_host, cudaStream_t s);

// Warped image (CpuFrameWarper::warpImageInterpolated semantics) for one frame.
cudaError_t launch_warp(const RefDev* ref_dev, const RefDev& ref_host, const void* frame, long long fplane, int fpitch,
                        int frame_kind,
                        const float4* dparams, float invalid_value, float* out, cudaStream_t s);

// One trust-region step for each job (grid = n_jobs): reduce partials, advance the state machine,
// solve the next subproblem, write the next trial point's dparams. With an active list, block b
// serves jobs[active[b]] for b < *n_active. max_nD / n_dim size the shared-memory staging (frames
// above about 200 KB work in global memory).
cudaError_t launch_solve(const Job* jobs_dev, int n_jobs, int max_nD, int n_dim, cudaStream_t s,
                         const int* active = nullptr, const int* n_active = nullptr);

// Test hook: the device trust-region subproblem on given dense H (P x P) and g.
// The band Cholesky factor of H (lambda = 0) into L0 (nD * nd rows of 2 * nd) and inv0 (nD * nd); *ok
// = 0 when H is not positive definite. One thread: the same arithmetic as the solver's factorisations.
cudaError_t launch_chol0(const double* Hd, const double* Hl, int nD, int nd, double* L0, double* inv0, int* ok,
                         cudaStream_t s);
cudaError_t launch_test_subproblem(const double* Hd, const double* Hl, int nD, int nd, double hinf, double mindiag,
                                   const double* g, double radius, double* p_out, int* boundary_out, double* work,
                                   cudaStream_t s);

// Outputs after the solve (fa_output.cu). scan4 = processed {pixel, interline, interframe, stack}.
// Forward splat of a dense raw frame (FA_F32 / FA_U16) by D (device, nD x 3): coverage always, the
// intensity-preserving image when wimg is set (both zeroed first).
cudaError_t launch_splat(const RefDev* ref_dev, const RefDev& ref_host, const double* scan4, const void* img,
                         int img_kind, const double* D_dev, float* wimg, float* cov, cudaStream_t s);
// Masked sums for the correlations of the warped frame and of the unaligned frame (raw + 1) against
// the reference over cov > 0: totals[0..7) = count, sum w, sum r, sum ww, sum rr, sum f, sum ff;
// totals[8..10) = the centred cross sums. parts: 296 x 8 doubles of scratch.
cudaError_t launch_metrics(const float* cov, const float* warped, const float* ref, const void* raw, int raw_kind,
                           long long n, double* parts, double* totals, cudaStream_t s);
// FrameWarpAligner::shiftPixel for n points (device arrays, in place).
cudaError_t launch_shift_points(const RefDev* ref_dev, const double* scan4, const double* D_dev, long long n, double* x,
                                double* y, double* z, cudaStream_t s);
// convertTo(CV_16U) of num (or num / den).
cudaError_t launch_to_u16(const float* num, const float* den, long long n, unsigned short* out, cudaStream_t s);

// Phase correlation kernels (fa_phase.cu), each over a batch of frames.
cudaError_t launch_phase_window(const void* const* vols, int in_kind, const double* wy, const double* wx, int ny,
                                int nx, long long n_el, int batch, double* out, cudaStream_t s);
cudaError_t launch_phase_normalise(double2* spec, const double2* ref_conj, long long n, int batch, cudaStream_t s);
cudaError_t launch_phase_argmax(const double* surf, long long n, int batch, double* block_val, long long* block_idx,
                                int blocks_per_frame, long long* out_idx, cudaStream_t s);
cudaError_t launch_phase_conj(const double2* in, double2* out, long long n, cudaStream_t s);
// Second argmax stage alone: the first maximum of nb (value, index) pairs per frame.
cudaError_t launch_phase_argmax_final(const double* block_val, const long long* block_idx, int nb, int batch,
                                      long long* out_idx, cudaStream_t s);

// Phase correlation as three fused passes over kx planes (fa_plane_corr.cu), for power-of-two
// volumes with nz <= 16, 8 <= ny <= 2048, 16 <= nx <= 4096 and nz * ny <= 8192 (plane_dims is false
// otherwise). Half-spectra are stored as planes spec[kx][z][y], kx = 0..nx/2.
struct PlaneDims {
  int nz, ny, nx, rows;      // rows = nz * ny
  int log2M, log2ny, log2G;  // M = nx / 2; G rows per row CTA
  int PP;                    // planes per plane CTA (one-kernel (z, y) pass); 0 when split
  int n_twx, tw_x_post;      // x twiddles: stage table of the nx/2-point DFT, then W_nx^k (k <= nx/2)
  int n_twy;                 // y twiddles: stage table of the ny-point DFT
  long long n_complex, n_el;
  // Split (z, y) pass, for planes too large for one CTA (nz * ny > 8192 or nz > 16): a y-line pass,
  // a z-column pass with the cross-power, and an inverse y-line pass.
  bool split;
  int log2nz;
  int LY;                    // y lines per CTA of the y-line passes
  int log2YB;                // y columns per CTA of the z-column pass
  int n_twz;                 // z twiddles: stage table of the nz-point DFT
};
bool plane_dims(int nz, int ny, int nx, PlaneDims* d);
// The twiddle tables the passes read (tw_x: d.n_twx entries, tw_y: d.n_twy, tw_z: d.n_twz when the
// pass is split, else empty), computed in long double.
void plane_twiddles(const PlaneDims& d, std::vector<double2>* tw_x, std::vector<double2>* tw_y,
                    std::vector<double2>* tw_z);
// CTAs (argmax partials) per frame of the last pass.
int plane_blocks_per_frame(const PlaneDims& d);
// Frame slots the first pass may fill while it reads the frames: frame i's value + 1 (the slot
// conversion, stored as `kind`: raw uint16 saturated, FP16 or FP32) at ptrs[i] + z * plane +
// y * pitch + x (16-byte aligned rows).
struct SlotOut {
  const void* const* ptrs;  // device array, one interior pointer per frame of the batch (writable slots)
  int kind;           // FrameKind
  int pitch;
  long long plane;
};
// Window + real DFT along x of each frame (dense FP32 or uint16, in_kind an fa_dtype) into spec
// (batch * n_complex); with `slot` (optional) also the frames' slots.
cudaError_t launch_plane_rows_fwd(const PlaneDims& d, const void* const* vols, int in_kind, int batch,
                                  const double* wy, const double* wx, const double2* tw_x, double2* spec,
                                  cudaStream_t s, const SlotOut* slot = nullptr);
// Per plane: forward DFT over (z, y), then either out = conj (reference) or, in place,
// out = inverse DFT of the normalised cross-power spectrum with ref_conj.
cudaError_t launch_plane_yz(const PlaneDims& d, const double2* in, double2* out, const double2* ref_conj,
                            const double2* tw_y, int batch, bool reference, cudaStream_t s);
// The same for split dimensions (d.split), in place in spec: forward DFT of every y line, then per
// z column the forward z DFT and either conj (reference: written to ref_conj instead) or the
// normalised cross-power with ref_conj and the inverse z DFT, then the inverse DFT of every y line
// (not for the reference).
cudaError_t launch_plane_yz_split(const PlaneDims& d, double2* spec, double2* ref_conj, const double2* tw_y,
                                  const double2* tw_z, int batch, bool reference, cudaStream_t s);
// One frame's half-spectrum from planes spec[kx][z][y] to cuFFT's order [z][y][kx].
cudaError_t launch_plane_to_rows(const PlaneDims& d, const double2* in, double2* out, cudaStream_t s);
// Inverse real DFT along x and the per-CTA first maximum (bval / bidx: batch * plane_blocks_per_frame);
// surface (batch * n_el doubles) receives the real surface when not null.
cudaError_t launch_plane_rows_inv_argmax(const PlaneDims& d, const double2* spec, int batch, const double2* tw_x,
                                         double* bval, long long* bidx, double* surface, cudaStream_t s);

}  // namespace fa
