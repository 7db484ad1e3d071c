/*
 * fa_b200.h -- C ABI of the B200 (sm_100a) frame-aligner warper library.
 *
 * This library replaces the GPU warper of flimfit/frame-aligner (class GpuFrameWarper,
 * FrameAligner/GpuFrameWarper.h:31-72) behind the warper interface AbstractFrameWarper
 * (FrameAligner/FrameWarper.h:95-143). Every entry point is plain C: pointers, sizes, status codes.
 * Paths in the citations are relative to the reference project's root.
 *
 * Conventions
 *  - Volumes are {nz, ny, nx} row-major, x fastest (FrameAligner/Cv3dUtils.cpp:6-8: Z=0, Y=1, X=2).
 *  - A displacement set D is nD control points of 3 doubles (x, y, z), the memory layout of
 *    std::vector<cv::Point3d>. For single-plane data (nz == 1, n_dim == 2) the z component is
 *    ignored.
 *  - Parameter vectors (Jacobians, Hessians) use OptimisationModel's order
 *    [D0.x, D0.y, (D0.z), D1.x, ...] (FrameAligner/OptimisationModel.cpp:14-27), P = nD * n_dim.
 *  - Pointers named host_* or documented as host memory are ordinary (pageable or pinned) host
 *    memory; pointers documented as device memory must be CUDA device allocations on the
 *    context's device.
 *  - Every function returns fa_status. The library never resets the device; on FA_ERR_CUDA the
 *    context stays usable unless the CUDA error was sticky. fa_last_error() describes the last
 *    failure on the calling thread.
 */
#ifndef FA_B200_H
#define FA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FA_OK = 0,
  FA_ERR_BAD_ARG = 1,      /* invalid argument (the reference would throw or has undefined behaviour) */
  FA_ERR_OOM = 2,          /* device memory or the context's memory budget is exhausted */
  FA_ERR_CUDA = 3,         /* a CUDA runtime / cuFFT call failed */
  FA_ERR_TIMEOUT = 4,      /* a bounded wait ran out */
  FA_ERR_UNSUPPORTED = 5,  /* valid for the reference but outside what this library implements */
  FA_ERR_NOT_FOUND = 6,    /* unknown handle / request id */
  FA_ERR_STATE = 7,        /* call out of order (e.g. no reference set) */
  FA_ERR_BUSY = 8          /* no free slot; retry later */
} fa_status;

typedef enum { FA_F32 = 0, FA_F16 = 1, FA_BF16 = 2, FA_U16 = 3 } fa_dtype;

/* Fields of ImageScanParameters (FrameAligner/ImageScanParameters.h:22-31), after construction. */
typedef struct {
  double line_duration;
  double interline_duration;
  double pixel_duration;
  double frame_duration;
  double interframe_duration;
  double stack_duration;
  int n_x, n_y, n_z;
  int bidirectional;
} fa_scan_params;

typedef struct fa_context fa_context;
typedef struct fa_reference fa_reference;
typedef struct fa_frame fa_frame;
typedef struct fa_correlator fa_correlator;

typedef struct {
  int device;            /* CUDA device ordinal */
  size_t memory_budget;  /* bytes of device memory the context may hold; 0 = 90% of free memory */
  int autotune;          /* 1: fa_set_reference times the fused pass's tile shapes on the device and keeps
                            the fastest (cached per volume shape for the process); 0: fixed defaults */
} fa_config;

/* Storage precision of a reference's device copies (the FP32 copy always exists: the Gauss-Newton
   Hessian and the plain path use it). */
typedef enum {
  FA_PREC_F32 = 0,   /* plain path: FP32 reference, gradient and frames */
  FA_PREC_MIXED = 1  /* BF16 reference + gradient, FP16 frames, FP32 accumulation, FP64 solve */
} fa_precision;

/* ---------------------------------------------------------------- context --------------------- */

/* GpuFrameWarper::getGpuSupportInformation (FrameAligner/GpuFrameWarper.cpp:16-44): *supported = 1
   when a compute-capability 10.x device is visible; message receives a short reason otherwise. */
fa_status fa_gpu_support(int* supported, char* message, size_t message_len);
fa_status fa_create(const fa_config* cfg, fa_context** out);
fa_status fa_destroy(fa_context* ctx);
/* Message of the last failure on this thread (static storage, valid until the next call). */
const char* fa_last_error(void);
const char* fa_status_string(fa_status s);

/* ImageScanParameters::ImageScanParameters (FrameAligner/ImageScanParameters.h:7-20). The
   reference constructor leaves `bidirectional` uninitialised; here it is an argument. */
fa_status fa_scan_params_init(double line_duration, double interline_duration, double interframe_duration, int n_x,
                              int n_y, int n_z, int bidirectional, fa_scan_params* out);

/* ---------------------------------------------------------------- reference ------------------- */

/* AbstractFrameWarper::setReference (FrameAligner/FrameWarper.cpp:186-205) followed by
   GpuFrameWarper::setupReferenceInformation (FrameAligner/GpuFrameWarper.cpp:75-152):
   interval tables, Sobel gradient, steepest-descent weights and the constant block-tridiagonal
   Hessian H = J^T J, all on the device. `reference` is host memory (nz*ny*nx floats, the smoothed
   reference with FrameWarpAligner's +1 offset already applied). Errors: FA_ERR_BAD_ARG for
   nx < 2, ny < 2, nD < 2 or a scan that does not reach interval nD-2 (the reference throws
   "Something went wrong", FrameWarper.cpp:280-281); FA_ERR_UNSUPPORTED when a control interval is
   skipped, shorter than one image row, or (bidirectional) not increasing in storage order. */
fa_status fa_set_reference(fa_context* ctx, const float* reference, int nz, int ny, int nx, int nD,
                           const fa_scan_params* scan, fa_precision precision, fa_reference** out);
/* Same, with the reference already in device memory (FP32). */
fa_status fa_set_reference_device(fa_context* ctx, const float* reference_device, int nz, int ny, int nx, int nD,
                                  const fa_scan_params* scan, fa_precision precision, fa_reference** out);
fa_status fa_reference_destroy(fa_reference* ref);
/* n_dim (2 or 3, FrameWarper.cpp:198) and the parameter count P = nD * n_dim. */
fa_status fa_reference_info(const fa_reference* ref, int* n_dim, int* n_params);
/* Tile shape of the fused pass (voxels per tile, CTAs per SM its register budget targets), as chosen
   by the autotuner or set by fa_reference_retune. No counterpart in the reference. */
fa_status fa_reference_tuning(const fa_reference* ref, int* tile_voxels, int* ctas_per_sm);
/* Forces a tile shape (tile_voxels rounded down to whole image rows and capped by the shortest
   control interval; ctas_per_sm in 2..4). Only while no frame of the reference is registered. */
fa_status fa_reference_retune(fa_reference* ref, int tile_voxels, int ctas_per_sm);
/* The member H read by OptimisationModel (OptimisationModel.cpp:61): dense P x P, row-major,
   host memory. */
fa_status fa_get_hessian(const fa_reference* ref, double* H);
/* The Sobel3d gradient images (Sobel3d.cpp:60-85), host memory, nz*ny*nx floats each; gz may be
   NULL. */
fa_status fa_get_gradient(const fa_reference* ref, float* gx, float* gy, float* gz);
/* D_range (FrameWarper.cpp:239-293): 2*nD ints {begin, end}; the unused last entry is {0, 0}. */
fa_status fa_get_ranges(const fa_reference* ref, int* ranges);

/* ---------------------------------------------------------------- frames ---------------------- */

/* GpuFrameWarper::registerFrame (FrameAligner/GpuFrameWarper.cpp:46-64): copies one frame
   (host memory, nz*ny*nx elements of `dtype`, FrameWarpAligner's +1 offset already applied) into
   device memory in the reference's storage precision. Frames are independent: each owns its
   stream and scratch, so different frames may be used from different threads concurrently. */
fa_status fa_register_frame(fa_reference* ref, const void* data, fa_dtype dtype, fa_frame** out);
/* Same, source in device memory. */
fa_status fa_register_frame_device(fa_reference* ref, const void* data_device, fa_dtype dtype, fa_frame** out);
/* Replaces a registered frame's pixels (host memory) without reallocating. */
fa_status fa_update_frame(fa_frame* frame, const void* data, fa_dtype dtype);
/* GpuFrameWarper::deregisterFrame (FrameAligner/GpuFrameWarper.cpp:66-73). */
fa_status fa_deregister_frame(fa_frame* frame);

/* ---------------------------------------------------------------- evaluation ------------------ */

/* CpuFrameWarper::getError / GpuFrameWarper::getError (FrameWarper.cpp:169-176,
   GpuFrameWarper.cpp:182-190): the sum of squared errors over voxels whose interpolated value is
   positive. One fused pass also forms J^T e, which fa_get_jacobian returns for the same D. */
fa_status fa_get_error(fa_frame* frame, const double* D, double* f);
/* AbstractFrameWarper::computeJacobian / GpuFrameWarper::getJacobian (FrameWarper.cpp:147-167,
   GpuFrameWarper.cpp:192-235): g = J^T e (P doubles, host memory). Reuses the pass of the last
   fa_get_error on this frame when D is identical; otherwise runs one. */
fa_status fa_get_jacobian(fa_frame* frame, const double* D, double* jac);
/* CpuFrameWarper::warpImageInterpolated (FrameWarper.cpp:31-69): trilinear (bilinear for a single
   plane) zero-padded resampling at x + d(x); exact zeros become invalid_value. out: host memory,
   nz*ny*nx floats. */
fa_status fa_warp(fa_frame* frame, const double* D, float invalid_value, float* out);

/* AbstractFrameWarper::warpImage (FrameAligner/FrameWarper.cpp:71-136): the forward,
   intensity-preserving splat of a frame (host, nz*ny*nx floats) by D into wimg (may be NULL) and the
   sum of splat weights per voxel into coverage; host outputs. Sums agree with the reference to float
   rounding (contributions are added in arbitrary order). */
fa_status fa_warp_image(fa_reference* ref, const float* frame, const double* D, float* wimg, float* coverage);

/* ---------------------------------------------------------------- alignment ------------------- */

typedef struct {
  int iterations;        /* trust-region iterations (subproblem solves) */
  int evaluations;       /* fused error+gradient passes, starting points included */
  int accepted;          /* accepted steps */
  int status;            /* 0 = converged by the stop rule, 1 = hit max_iterations */
  double f_final;        /* sum of squared errors at the returned D */
  double radius_final;
} fa_align_stats;

/* The solve of FrameWarpAligner::addFrame (FrameAligner/FrameWarpAligner.cpp:194-219) on the
   device: starting points {0, rigid_shift} (first minimum wins), then the trust region
   (radius 40, stop when |delta f| < 1e-8) with the constant Hessian. rigid_shift: 3 doubles (x, y,
   z), already scaled by the phase-correlation binning, or NULL for none. max_iterations <= 0
   means 100. D_out: nD*3 doubles, host memory. The host drives the iterations (one fused pass and
   one solve launch per iteration, the plain single-frame path). */
fa_status fa_align_frame(fa_frame* frame, const double* rigid_shift, int max_iterations, double* D_out,
                         fa_align_stats* stats);

/* Batched solve: n frames of one reference advance together, one fused multi-frame pass plus one
   multi-frame solve launch per trust-region iteration, iterations captured in a CUDA graph and
   run without host round-trips. rigid_shifts: n*3 doubles or NULL. D_out: n*nD*3 doubles, stats:
   n entries (may be NULL); host memory. Results per frame equal the frame aligned alone. */
fa_status fa_align_batch(fa_frame* const* frames, int n, const double* rigid_shifts, int max_iterations,
                         double* D_out, fa_align_stats* stats);

/* ---------------------------------------------------------------- phase correlation ----------- */

/* VolumePhaseCorrelator (FrameAligner/VolumePhaseCorrelator.cpp:29-139): FP64 cuFFT R2C of the
   windowed volume, hand-written cross-power normalisation and first-maximum argmax, integer
   shift wrapped to (-n/2, n/2]. `reference` is host memory (nz*ny*nx floats). */
fa_status fa_correlator_create(fa_context* ctx, const float* reference, int nz, int ny, int nx, fa_correlator** out);
fa_status fa_correlator_destroy(fa_correlator* c);
/* shift: 3 doubles (x, y, z). volume: host memory. */
fa_status fa_correlator_shift(fa_correlator* c, const float* volume, double* shift);
/* Same, volume in device memory. */
fa_status fa_correlator_shift_device(fa_correlator* c, const float* volume_device, double* shift);

/* ---------------------------------------------------------------- aligner --------------------- */

/* The per-frame flow of FrameWarpAligner (FrameAligner/FrameWarpAligner.cpp:77-105 setReference,
   117-219 addFrame) on the device: the +1 offset, the phase-correlation rigid start on the
   downsampled raw data, the starting-point choice and the trust-region solve, for a batch of
   frames at a time. RealignmentParameters (FrameAligner/AbstractFrameAligner.h:31-48) fields that
   this path reads are mirrored here. */
typedef struct fa_aligner fa_aligner;

typedef struct {
  int spatial_binning;       /* RealignmentParameters::spatial_binning: phase-correlation downsampling */
  int n_resampling_points;   /* nD = n_resampling_points * n_z + 1 (FrameWarpAligner.cpp:100) ... */
  int nD;                    /* ... unless nD > 0, which sets the control-point count directly */
  double smoothing;          /* smoothStack (FrameWarpAligner.cpp:46-64): sigma along x of the per-plane Gaussian
                                (sigma 1 along y, as the reference); 0: none; at most 32 */
  fa_precision precision;
  int max_iterations;        /* <= 0: 100 */
  double correlation_threshold;  /* RealignmentParameters::correlation_threshold (RealignmentResult::useFrame) */
  double coverage_threshold;     /* RealignmentParameters::coverage_threshold */
} fa_aligner_params;

/* RealignmentResult's metrics (FrameAligner/AbstractFrameAligner.h:51-66). */
typedef struct {
  double correlation;            /* correlation(warped, reference) over coverage > 0 (FrameWarpAligner.cpp:240) */
  double unaligned_correlation;  /* correlation(frame, reference) over the same mask (:241) */
  double coverage;               /* fraction of voxels with coverage > 0 (:243) */
  int use_frame;                 /* RealignmentResult::useFrame with the aligner's thresholds */
} fa_frame_result;

fa_status fa_aligner_create(fa_context* ctx, const fa_aligner_params* params, fa_aligner** out);
fa_status fa_aligner_destroy(fa_aligner* a);
/* FrameWarpAligner::setReference: `reference` is the raw reference (host memory, nz*ny*nx elements
   of dtype FA_F32 or FA_U16). */
fa_status fa_aligner_set_reference(fa_aligner* a, const void* reference, fa_dtype dtype, int nz, int ny, int nx,
                                   const fa_scan_params* scan);
/* The control-point count and parameter layout of the current reference. */
fa_status fa_aligner_info(const fa_aligner* a, int* nD, int* n_dim);
/* The aligner's warper (FrameWarpAligner::warper): the reference it aligns against, with the +1
   offset, for the warper-level calls (fa_warp_image, fa_shift_pixels, fa_get_hessian ...). Owned by
   the aligner; valid until its next fa_aligner_set_reference or fa_aligner_destroy. */
fa_status fa_aligner_reference(const fa_aligner* a, fa_reference** ref);
/* FrameWarpAligner::addFrame for n raw frames (host memory; frames[i] points at nz*ny*nx elements of
   dtype). D_out: n*nD*3 doubles, stats: n entries or NULL; host memory. Uploads overlap the device
   work when the frames are in page-locked memory; none is in flight when the call returns. */
fa_status fa_aligner_add_frames(fa_aligner* a, const void* const* frames, fa_dtype dtype, int n, double* D_out,
                                fa_align_stats* stats);
/* Same, frames already in device memory (frames[i] device pointers). */
fa_status fa_aligner_add_frames_device(fa_aligner* a, const void* const* frames, fa_dtype dtype, int n,
                                       double* D_out, fa_align_stats* stats);

/* The end of FrameWarpAligner::addFrame (FrameAligner/FrameWarpAligner.cpp:221-247) and its cached
   outputs, for n frames already aligned (D: n*nD*3, e.g. from fa_aligner_add_frames): the forward
   splat's coverage, the correlations and coverage fraction (results, may be NULL), and optionally
   per frame (arrays of n host pointers, or NULL; an entry may be NULL) the realigned image
   (getInterpolatedWarpedFrame :328-338, uint16), the intensity-preserving realigned image
   (getWarpedFrame :317-326, uint16) and the mask (getMask :340-346, the coverage, float).
   frames: raw frames in host memory (dtype FA_F32 or FA_U16). */
fa_status fa_aligner_results(fa_aligner* a, const void* const* frames, fa_dtype dtype, int n, const double* D,
                             fa_frame_result* results, uint16_t* const* realigned,
                             uint16_t* const* realigned_preserving, float* const* mask);

/* FrameWarpAligner::shiftPixel (FrameAligner/FrameWarpAligner.cpp:253-266) for n photons: each
   (x, y, z) moves by minus warpPoint(D, int(x), int(y), int(z)) (FrameWarper.cpp:397-419), the
   displacement of the voxel it was recorded in; points outside the volume stay. Host arrays,
   updated in place; D: nD*3 doubles of one frame. */
fa_status fa_shift_pixels(fa_reference* ref, const double* D, long long n, double* x, double* y, double* z);

/* FrameWarpAligner::writeRealignmentInfo (FrameAligner/FrameWarpAligner.cpp:288-314): the CSV of
   the scan parameters (as given, not processed), per-frame metrics and D (n_frames*nD*3 doubles).
   Host only; writes nothing when n_frames == 0. */
fa_status fa_write_realignment_info(const char* filename, const fa_scan_params* image_params, int n_frames, int nD,
                                    const double* D, const fa_frame_result* results);

/* ---------------------------------------------------------------- serving ---------------------- */

/* A device-resident request loop over several concurrent acquisitions (no single counterpart in the
   reference: each acquisition is one FrameWarpAligner, FrameAligner/FrameWarpAligner.cpp:77-251,
   whose addFrame calls the MEX pool issues from many threads, FrameAlignerMex.cpp:120). Each
   acquisition keeps its reference, gradient, Hessian, correlator and last solution on the device.
   Frames submitted from any thread are admitted into device slots as slot count and memory budget
   allow, uploaded and phase-correlated on the acquisition's stream, and then solved together with
   every other admitted frame of the same dimensionality and storage, one CUDA graph of
   iterations_per_launch x (fused pass, trust-region step) per launch, while later frames upload and
   correlate. A frame's result does not depend on which other frames share its launches. */
typedef struct fa_server fa_server;

typedef struct {
  size_t memory_budget;       /* device bytes frame slots may hold (0: 40 GiB) */
  int max_in_flight;          /* frames admitted and not finished, all acquisitions (0: 256) */
  int iterations_per_launch;  /* trust-region iterations per graph launch (0: 4) */
  int warm_start;             /* lag d >= 1: frame k's starting points are {0, 0, rigid, the solution of
                                 frame k - d of the same acquisition} (d = 1: the previous frame); frame k
                                 evaluates the first three at once and waits on the device for frame
                                 k - d's solution before the fourth; 0: no warm start (at most 64) */
  int shared_launches;        /* 0: each acquisition's frames have their own job table, graph and stream,
                                 and acquisitions overlap on the device; 1: acquisitions whose frames
                                 can share a kernel (same dimensionality, storage and precision) share
                                 the launches */
} fa_server_config;

typedef struct {
  long long submitted, completed, failed;
  long long in_flight, peak_in_flight;
  double p50_ms, p99_ms, mean_ms, max_ms;  /* per-frame latency: submission -> result on the host */
  double frames_per_s;                     /* completed / (last completion - first submission) */
  size_t slot_bytes, peak_slot_bytes;      /* device bytes held by frame slots */
  long long graph_launches;
} fa_server_stats;

fa_status fa_server_create(fa_context* ctx, const fa_server_config* cfg, fa_server** out);
/* Finishes every submitted frame, then releases the server and its acquisitions. */
fa_status fa_server_destroy(fa_server* s);
/* FrameWarpAligner::setReference for a new acquisition (reference: host memory, nz*ny*nx elements of
   reference_dtype, FA_F32 or FA_U16); its frames will be frame_dtype (FA_F32 or FA_U16). */
fa_status fa_server_add_acquisition(fa_server* s, const fa_aligner_params* params, const void* reference,
                                    fa_dtype reference_dtype, int nz, int ny, int nx, const fa_scan_params* scan,
                                    fa_dtype frame_dtype, int* acquisition);
fa_status fa_server_acquisition_info(fa_server* s, int acquisition, int* nD, int* n_dim);
/* Creates idle frame slots for an acquisition until it holds n_slots (device memory for frames and
   their solve state, within the memory budget), so that the first frames of a stream do not wait
   for allocations. FA_ERR_OOM when the budget or job table cannot hold them (the slots created so
   far stay). */
fa_status fa_server_reserve(fa_server* s, int acquisition, int n_slots);
/* FrameWarpAligner::addFrame, asynchronous: queues one raw frame (host memory, or device memory when
   frame_on_device) and returns its ticket. The frame's memory must stay valid and unchanged until its
   result has been collected; page-locked host memory lets the upload overlap other work. */
fa_status fa_server_submit(fa_server* s, int acquisition, const void* frame, int frame_on_device,
                           unsigned long long* ticket);
/* Waits up to timeout_s seconds (< 0: no limit) for a ticket's result and collects it: D_out nD*3
   doubles, stats and latency_ms may be NULL. FA_ERR_TIMEOUT leaves the result to a later call;
   FA_ERR_NOT_FOUND means the ticket is unknown or already collected. */
fa_status fa_server_wait(fa_server* s, unsigned long long ticket, double timeout_s, double* D_out,
                         fa_align_stats* stats, double* latency_ms);
fa_status fa_server_get_stats(fa_server* s, fa_server_stats* out);
/* Clears the latency record and counters (not the acquisitions or their warm starts). */
fa_status fa_server_reset_stats(fa_server* s);

/* ---------------------------------------------------------------- static-scratch evaluation --- */

/* No counterpart in the reference. For callers that cannot call cudaMalloc when they evaluate a
   frame (a host application that has reserved the device memory pool for its own allocator, or a
   real-time acquisition loop that must not allocate between frames): the same fused error + J^T e
   pass as fa_get_error / fa_get_jacobian on a frame held in the caller's own device memory
   (frame_device: nz*ny*nx elements, FA_F32 for an FA_PREC_F32 reference, FA_F16 for FA_PREC_MIXED,
   +1 offset applied), with every piece of scratch in one fixed 2 MiB device array inside the
   library, which each GPU that loads the library holds until exit. The call allocates no device or
   host memory; it runs on the legacy default stream and returns when f (host double) and jac (P host
   doubles) are written. Volumes whose scratch would exceed 2 MiB (about 21,000 tiles of the fused
   pass) are rejected with FA_ERR_BAD_ARG, and so is a D with a non-finite entry. The work runs on the
   reference's device; the caller's current device is restored before the call returns. The first
   call on each device looks up the array's device address (cudaGetSymbolAddress) with that device
   current; make it before any stream capture (a cudaDeviceReset invalidates that address together
   with every other handle of this library). All calls share the array, so calls that overlap on the
   GPU (other threads, other streams) race and must be serialised by the caller. */
fa_status fa_get_error_jacobian_static(const fa_reference* ref, const void* frame_device, fa_dtype dtype,
                                       const double* D, double* f, double* jac);

/* ---------------------------------------------------------------- measurement ----------------- */

/* Number of this library's kernels launched so far in the process (graph replays included). */
long long fa_kernel_launches(void);
/* Device time (CUDA events on the library's streams) of the last fa_aligner_add_frames* call, ms. */
fa_status fa_aligner_last_device_ms(const fa_aligner* a, double* ms);
/* The same call split: correlate_ms = device time from the call's start until every frame was
   converted and phase-correlated (uploads, conversion, window, transforms, peak), total_ms = all of
   it (the solve of the first frames overlaps the correlation of the later ones). */
fa_status fa_aligner_last_phase_ms(const fa_aligner* a, double* correlate_ms, double* total_ms);
/* Times the fused warp + error + J^T e pass alone: `launches` back-to-back launches over n
   registered frames (of one reference) at displacement D (nD*3 doubles, host memory), bracketed by
   CUDA events on the launching stream. ms_per_launch receives the average duration. */
fa_status fa_profile_eval(fa_frame* const* frames, int n, const double* D, int launches, double* ms_per_launch);

/* ---------------------------------------------------------------- test hooks ------------------ */

/* Runs the device trust-region subproblem solver (the step computation inside dlib's
   find_min_trust_region, called at FrameAligner/FrameWarpAligner.cpp:205-209) once on a given dense
   block-tridiagonal H (P x P, P = nD * n_dim, host memory) and gradient g; writes the step p and
   whether it lies on the trust-region boundary. Lets tests compare the device solver with the
   CPU statement of the same algorithm on identical inputs. */
fa_status fa_test_tr_subproblem(fa_context* ctx, int nD, int n_dim, const double* H, const double* g, double radius,
                                double* p, int* on_boundary);

/* Test hook (no reference counterpart): the device form of downsample (FrameAligner/
   AbstractFrameAligner.cpp:37-56) that the aligner applies before phase correlation when
   spatial_binning > 1 -- each output voxel (z, y / factor, x / factor) is the float sum of its
   factor x factor block, ceil-sized, the last block of a row or column ragged. volume: host memory,
   nz*ny*nx elements of dtype (FA_F32 or FA_U16); out: host memory, nz*ceil(ny/factor)*ceil(nx/factor)
   floats. Lets tests compare the kernel with the reference's loop bit for bit. */
fa_status fa_test_downsample(fa_context* ctx, const void* volume, fa_dtype dtype, int nz, int ny, int nx, int factor,
                             float* out);

/* Test hook (no reference counterpart): the phase-correlation surface of one FP32 volume (host
   memory, nz*ny*nx) against the correlator's reference -- the unnormalised inverse DFT of the
   normalised cross-power spectrum, nz*ny*nx doubles into host memory -- computed by the fused
   kx-plane passes (use_planes = 1; FA_ERR_UNSUPPORTED when the dimensions are outside them) or by
   cuFFT (use_planes = 0). Lets tests compare both with a CPU DFT. */
fa_status fa_test_correlation_surface(fa_correlator* c, const float* volume, int use_planes, double* surface);

/* Test hook (no reference counterpart, host only: no device work): the tables and launch shape the
   fused kx-plane passes would use for an nz x ny x nx volume. tw_x receives n_x complex twiddles
   (interleaved re, im): the stage twiddles of the nx/2-point row DFT, then W_nx^k for k = 0..nx/2
   from index x_post; tw_y the stage twiddles of the ny-point DFT (n_y). For every stage after the
   first (Ns > 1, radix R: radix 8 while at least 3 octaves are left, then 4 or 2), the table holds
   W_(Ns R)^(r k) at (r - 1) Ns + k, r = 1..R-1, k = 0..Ns-1. planes_per_cta is 0 when the (z, y)
   pass is split into y-line and z-column passes (planes of more than 8192 points or nz > 16), whose
   z DFT uses the same stage table for nz points. FA_ERR_UNSUPPORTED for dimensions that take the
   cuFFT path. Lets CPU tests check the tables and the pass structure without a GPU. */
fa_status fa_test_plane_tables(int nz, int ny, int nx, double* tw_x, int cap_x, int* n_x, int* x_post, double* tw_y,
                               int cap_y, int* n_y, int* rows_per_cta, int* planes_per_cta);

#ifdef __cplusplus
}
#endif
#endif /* FA_B200_H */
