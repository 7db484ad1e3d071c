/*
 * fa_oracle.h -- CPU restatement of frame-aligner's non-rigid warper path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library. Only tests/, the smoke() entry
 * and bench.py's CPU-baseline leg may load it. It is never part of the product path.
 *
 * Each function restates one piece of the reference (paths relative to the reference
 * project root):
 *   or_scan_init            FrameAligner/ImageScanParameters.h:7-20
 *   or_process_scan         FrameAligner/FrameWarper.cpp:223-236
 *   or_warper_create        FrameAligner/FrameWarper.cpp:186-205 (setReference), with
 *                           precomputeInterp 239-293, computeSteepestDecentImages 296-345,
 *                           computeHessian 347-395
 *   or_sobel3d              FrameAligner/Sobel3d.cpp:8-85
 *   or_warp_interpolated    FrameAligner/FrameWarper.cpp:31-69 (+ getZeroPadded FrameWarper.h:39-47)
 *   or_get_error            FrameAligner/FrameWarper.cpp:4-29,169-176
 *   or_get_jacobian         FrameAligner/FrameWarper.cpp:147-167,178-182
 *   or_warp_image           FrameAligner/FrameWarper.cpp:71-136 (intensity-preserving splat)
 *   or_warp_point           FrameAligner/FrameWarper.cpp:397-419
 *   or_downsample           FrameAligner/AbstractFrameAligner.cpp:37-56
 *   or_smooth_stack         FrameAligner/FrameWarpAligner.cpp:46-64 (cv::GaussianBlur stated, unpinned)
 *   or_correlation          FrameAligner/Cv3dUtils.cpp:57-81 (masked Pearson)
 *   or_trust_region         the project's trust-region algorithm (dlib find_min_trust_region is
 *                           called at FrameAligner/FrameWarpAligner.cpp:205-209 but its source is
 *                           not part of the reference; see the header of fa_oracle_tr.c)
 *   or_align_frame          FrameAligner/FrameWarpAligner.cpp:117-219 (starting points + solve)
 *
 * Pinning: tests/test_oracle_pin.py runs this restatement beside the reference's own
 * FrameWarper.cpp / Sobel3d.cpp / VolumePhaseCorrelator.cpp / OptimisationModel.cpp, compiled
 * unchanged from the reference tree against minimal container stand-ins (oracle/Makefile ->
 * oracle/_ref/libfa_ref.so), and requires bit-identical results.
 */
#ifndef FA_ORACLE_H
#define FA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double line_duration, interline_duration, pixel_duration;
  double frame_duration, interframe_duration, stack_duration;
  int n_x, n_y, n_z;
  int bidirectional;
} or_scan;

void or_scan_init(or_scan* s, double line_duration, double interline_duration, double interframe_duration,
                  int n_x, int n_y, int n_z, int bidirectional);
void or_process_scan(const or_scan* in, int nz, int nD, or_scan* out);

typedef struct or_warper or_warper;

/* Returns NULL and fills err (if non-NULL, >= 128 bytes) on failure. */
or_warper* or_warper_create(const float* reference, int nz, int ny, int nx, int nD, const or_scan* scan, char* err);
void or_warper_destroy(or_warper* w);
int or_warper_n_dim(const or_warper* w);
/* Copies of the precomputed state: Di/Df are N-voxel arrays, ranges is 2*nD ints (begin,end). */
void or_warper_precomp(const or_warper* w, uint16_t* Di, float* Df, int* ranges);
/* Dense (nD*n_dim)^2 Gauss-Newton Hessian H = J^T J, row-major. */
void or_warper_hessian(const or_warper* w, double* H);
/* Sobel gradient images of the reference (each N floats). */
void or_warper_gradient(const or_warper* w, float* gx, float* gy, float* gz);

/* D is nD x 3 doubles (x, y, z per control point). */
void or_warp_interpolated(const or_warper* w, const float* frame, const double* D, float invalid_value, float* out);
/* Sum of squared errors; err (N floats) receives the error image if non-NULL. */
double or_get_error(const or_warper* w, const float* frame, const double* D, float* err);
/* J^T e from an error image; jac has nD*n_dim doubles. */
void or_get_jacobian(const or_warper* w, const float* err, double* jac);
void or_warp_image(const or_warper* w, const float* frame, const double* D, float* wimg, float* coverage);
void or_warp_point(const or_warper* w, const double* D, int x, int y, int z, int spatial_binning, double* out3);

void or_sobel3d(const float* m, int nz, int ny, int nx, float* gx, float* gy, float* gz);
void or_downsample(const float* in, int nz, int ny, int nx, int factor, float* out);
/* smoothStack (FrameWarpAligner.cpp:46-64): per-plane Gaussian blur, sigma along x and 1 along y.
   Returns -1 if a kernel would exceed 257 taps. or_gaussian_kernel writes the n float weights and
   returns n. */
int or_smooth_stack(const float* in, int nz, int ny, int nx, double sigma, float* out);
int or_gaussian_kernel(double sigma, float* k, int max_n);
double or_correlation(const float* a, const float* b, const uint8_t* mask, long n);

typedef struct {
  int iterations;     /* outer trust-region iterations (subproblem solves) */
  int evaluations;    /* objective evaluations (starting points included for or_align_frame) */
  int accepted;       /* accepted steps */
  double f_final;
  double radius_final;
} or_tr_stats;

typedef double (*or_feval_fn)(void* ctx, const double* x);
typedef void (*or_geval_fn)(void* ctx, const double* x, double* g);

/* Minimise f from x (in/out) with the constant model Hessian H (P x P, row-major). */
int or_trust_region(int P, const double* H, double* x, double radius0, double min_delta, int max_iter,
                    or_feval_fn f, or_geval_fn g, void* ctx, or_tr_stats* st);
/* One trust-region subproblem: p minimises g.p + 0.5 p.H.p within |p| <= radius.
   Returns 1 if the radius bound was active, 0 otherwise. */
int or_tr_subproblem(int P, const double* H, const double* g, double radius, double eps, int max_iter, double* p);

/* Full per-frame non-rigid alignment: starting points {0, 0, rigid} evaluated, first minimum
   taken, then the trust region from radius 40 with the |delta f| < 1e-8 stop rule.
   rigid_shift = 3 doubles (already scaled by the phase-correlation binning).
   D_out = nD x 3 doubles. */
int or_align_frame(const or_warper* w, const float* frame, const double* rigid_shift, int max_iter, double* D_out,
                   or_tr_stats* st);
/* or_align_frame plus the serving loop's warm start: warm_D (nD x 3, or NULL) is a fourth starting
   point after {0, 0, rigid}, reached as x + (warm - x) from the chosen start and taken only if its
   value is strictly smaller. */
int or_align_frame_warm(const or_warper* w, const float* frame, const double* rigid_shift, const double* warm_D,
                        int max_iter, double* D_out, or_tr_stats* st);
/* The reference's threading model: frames spread over n_threads workers, one frame per worker
   at a time. frames = n_frames * N floats; D_out = n_frames * nD * 3. Returns 0 on success. */
int or_align_frames_mt(const or_warper* w, const float* frames, int n_frames, const double* rigid_shifts,
                       int max_iter, int n_threads, double* D_out, int* iterations_out);

#ifdef __cplusplus
}
#endif
#endif
