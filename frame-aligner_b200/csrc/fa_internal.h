// fa_internal.h -- device data layout shared by the kernels and the host runtime.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fa_b200.h"

namespace fa {

// One image row (fixed z, y) of the scan-time displacement model.
//   scan position xs = x, or nx-1-x on odd rows of a bidirectional scan;
//   interval Di(xs) = di0 + (xs >= xdi)                     (FrameWarper.cpp:258-260)
//   fraction Df(xs) ~= qbase + xs * dq - (Di - di0)          (FP32; exact tables only on the host)
//   storage range r(x) = r0 + (x >= xr)                      (D_range, FrameWarper.cpp:269-275)
//   x == xlast marks the last voxel of a range, whose steepest-descent weight is zero
//   (the exclusive loop ends at FrameWarper.cpp:315,333).
struct RowDesc {
  float qbase;
  int di0;
  int xdi;
  int r0;
  int xr;
  int xlast;
  int y;  // image row index within its plane
  int z;  // plane index
};

// Control-point parameters for the fused pass, per control point k (3 float4):
//   [0] integer part of D[k] (xyz), [1] fractional part of D[k], [2] D[k+1] - D[k].
// d(x) = int(D[k]) + (frac(D[k]) + Df * (D[k+1]-D[k])) keeps the FP32 fraction exact to ~1e-7 px.
constexpr int kDParamF4 = 3;

// Partial sums of one tile: f, then g for three consecutive control points starting at c0.
constexpr int kPartialDoubles = 12;  // [f, c0, g(3 x 3), pad]

// Storage of a frame slot: FP32 or FP16 values (the +1 offset of FrameWarpAligner.cpp:142 already
// applied), or raw uint16 photon counts to which the kernels add 1 when they read them.
enum FrameKind : int { kFrameF32 = 0, kFrameF16 = 1, kFrameRawU16 = 2 };

// Frame solve phases (device trust region).
enum Phase : int {
  kPhaseStartZero = 0,   // trial = zero displacement
  kPhaseStartRigid = 1,  // trial = rigid shift
  kPhaseTrial = 2,       // trial = x + p
  kPhaseDone = 3,
  kPhaseStartLast = 4,   // trial = an earlier frame's solution (warm start)
  kPhaseWaitWarm = 5,    // cold starting points done; out of the passes until the warm-start vector
                         // has been written (resumed by the compact pass)
  kPhaseStartPair = 6    // both cold starting points in one pass: zero (dparams, partials) and the
                         // rigid shift (dparams2, partials2); persistent fused pass only
};

struct FrameState {
  double f;        // f(x)
  double f_prev;   // value at the previous stop-rule check
  double f_start;  // f at the zero start
  double radius;
  int iter;
  int accepted;
  int evaluations;
  int have_prev;
  int boundary;    // last subproblem step was on the trust-region boundary
  int phase;
  int max_iter;
  int hit_max;
  double rigid[3];
  int use_warm;    // *warm holds a fourth starting point
  int pad_;
  double* warm;    // P doubles or null: read by kPhaseStartLast when use_warm; the solution is
                   // written here when the solve finishes
  long long* warm_seq;  // sequence number of the frame whose solution *warm holds (null: no warm start)
  long long warm_need;  // the writer this frame's warm start must come from
  long long seq;        // this frame's sequence number, stored to *warm_seq with its solution
};

// Where a finished frame's solve is reported (host-mapped memory): the final FrameState, then the
// P accepted parameters.
constexpr int kReportHeaderBytes = (int)sizeof(FrameState);

// Everything a kernel needs about one reference (device-resident copy).
struct RefDev {
  int nz, ny, nx, nD, n_dim;
  int n_rows;
  long long N;
  int bidir;
  float dq;
  int tile_rows;
  int n_tiles;
  int P;
  int tune_mb;         // fused pass: CTAs per SM the register budget is sized for (2, 3 or 4), launches of many frames
  int tune_grid_mult;  // persistent fused pass: CTAs per SM launched
  int tune_mb_small;   // the same for launches of one or a few frames (single-frame, static-scratch, serving)
  const RowDesc* rows;
  const int* tile_c0;      // per tile: storage range index of its first voxel
  const int2* ctrl_tiles;  // per control point: tiles [x, y) whose partial slots may hold it
  const float* ref32;
  const float* gx32;
  const float* gy32;
  const float* gz32;
  // Mixed precision: BF16 reference and gradient interleaved per group of four consecutive voxels
  // (voxels 4g .. 4g+3: reference, gx, gy, gz, four values each; 32 bytes, two 16-byte loads).
  const __nv_bfloat16* q16;
  const double* Hd;  // nD blocks of n_dim x n_dim (diagonal), row-major
  const double* Hl;  // nD blocks (block k couples k and k-1; block 0 unused)
  double h_inf;      // max_i sum_j |H_ij| (ascending j), the subproblem's bracket bound
  double h_mindiag;  // min_i H_ii
  // The band Cholesky factor of H itself (lambda = 0), the same for every frame and iteration of the
  // reference: P rows of 2 * n_dim entries and P reciprocal diagonals, or null; chol0_ok = 0 when H
  // is not positive definite.
  const double* L0;
  const double* inv0;
  int chol0_ok;
};

// h_inf and h_mindiag of a block-tridiagonal H from its blocks (host), summing |H_ij| over ascending
// j within the band like the dense loop over all j (whose other terms are exact zeros).
inline void band_bounds(const double* Hd, const double* Hl, int nD, int nd, double* h_inf, double* h_mindiag) {
  const int P = nD * nd, nn = nd * nd;
  double hinf = 0.0, mind = Hd[0];
  for (int i = 0; i < P; i++) {
    const int b = i / nd, a = i % nd;
    const int j0 = b > 0 ? (b - 1) * nd : 0, j1 = (b + 2) * nd < P ? (b + 2) * nd : P;
    double r = 0.0;
    for (int j = j0; j < j1; j++) {
      const int bj = j / nd, c = j % nd;
      double v;
      if (bj == b)
        v = Hd[b * nn + a * nd + c];
      else if (bj + 1 == b)
        v = Hl[b * nn + a * nd + c];
      else
        v = Hl[bj * nn + c * nd + a];
      r += v < 0 ? -v : v;
    }
    if (r > hinf) hinf = r;
    const double d = Hd[b * nn + a * nd + a];
    if (d < mind) mind = d;
  }
  *h_inf = hinf;
  *h_mindiag = mind;
}

// One frame in a fused pass / solve launch.
// Zero halo around every frame slot: taps that leave the volume read these zeros, which is the
// reference's zero padding (getZeroPadded, FrameWarper.h:39-47) without per-tap bounds checks.
// X is a multiple of 4 so that every 4-element window of a row stays aligned.
constexpr int kHaloX = 8;
constexpr int kHaloY = 2;
constexpr int kHaloZ = 2;  // planes, for volumes with nz > 1

struct Job {
  const RefDev* ref;      // device pointer
  const void* frame;      // device pointer to voxel (0, 0, 0); FrameKind storage
  long long fplane;       // elements between planes of the frame
  int fpitch;             // elements between rows of the frame
  int fpad;               // 1: the frame carries the kHalo* zero halo
  float4* dparams;        // nD * kDParamF4 (trial point of this job)
  double* partials;       // n_tiles * kPartialDoubles
  float4* dparams2;       // the rigid starting point while the phase is kPhaseStartPair
  double* partials2;      // its tile partial sums (n_tiles * kPartialDoubles)
  FrameState* state;      // solve state (may be null for a bare evaluation)
  double* x;              // P: accepted parameters
  double* g;              // P: gradient at x
  double* p;              // P: trial step
  double* gt;             // P: gradient at the trial point
  double* work;           // solve scratch (band Cholesky etc.)
  double* result;         // [f, g(P)] of the last pass (bare evaluation)
  void* report;           // host-mapped FrameState + P doubles written when the solve finishes, or null
};

// A frame entering a batched solve (written by the host, applied on the device by launch_activate).
struct Activation {
  int job;       // index in the job table
  int use_warm;  // 1: *warm is a starting point
  int max_iter;
  int pair;      // 1: evaluate both cold starting points in one pass (kPhaseStartPair)
  double rigid[3];
  double* warm;          // FrameState::warm (null: none)
  long long* warm_seq;   // FrameState::warm_seq
  long long warm_need;   // FrameState::warm_need
  long long seq;         // FrameState::seq
};

}  // namespace fa
