// fa_solve.cu -- device-side trust-region solver (FP64). Built with -fmad=false: every product and
// sum is rounded separately, in the same order as the CPU statement of the algorithm, so that given
// identical f, g and H the device takes bit-identical steps.
//
// Algorithm (the reference calls dlib::find_min_trust_region at FrameAligner/FrameWarpAligner.cpp:
// 205-209 with objective_delta_stop_strategy(1e-8) and radius 40; dlib's source is not part of the
// reference tree, so this is the project's own statement of the method):
//   outer loop: Nocedal & Wright, Numerical Optimization (2nd ed.), Algorithm 4.1 with eta = 0,
//     Delta_max = 1000; rho < 1/4 shrinks Delta by 4, rho > 3/4 on the boundary doubles it; a
//     rejected step leaves f unchanged, so the |delta f| < 1e-8 rule ends the solve.
//   subproblem: More & Sorensen (1983) Newton iteration on 1/|p(lambda)| - 1/Delta with a
//     safeguarded bracket, eps = 0.1, at most 20 factorisations, using a block-tridiagonal
//     Cholesky of H + lambda I (H = J^T J has n_dim x n_dim blocks, |i - j| <= 1).
#include <float.h>

#include "fa_device.cuh"

namespace fa {

namespace {

constexpr double kDblEps = 2.220446049250313080847e-16;
constexpr double kMinDelta = 1e-8;
constexpr double kRadius0 = 40.0;
constexpr double kRadiusMax = 1000.0;

template <int ND>
struct Band {
  static constexpr int nd = ND;
  const double* Hd;
  const double* Hl;
  int nD, P;
  double hinf, mindiag;  // band_bounds of H
  // band_chol(lambda = 0) computed once per reference (RefDev::L0), or null
  const double* L0 = nullptr;
  const double* inv0 = nullptr;
  int chol0_ok = 0;
};

// Band factor storage: row i of block b holds 2*n_dim entries, the columns of block b-1 then those of
// block b.

// Cholesky of H + lambda I by block rows, fully unrolled over the n_dim x n_dim blocks. Each entry
// L_ij accumulates A_ij (+ lambda) minus L_ik L_jk over ascending k -- the previous block's columns
// first, then the earlier columns of its own block -- which is the dense algorithm's order (its
// other terms are exact zeros). inv[i] = 1 / L_ii; off-diagonal entries multiply by it.
template <int ND>
__device__ int band_chol(const Band<ND>& B, double lambda, double* L, double* inv) {
  constexpr int NN = ND * ND;
  double C[ND][ND];   // L rows of block b, columns of block b-1
  double Dg[ND][ND];  // L rows of block b, its own columns (lower triangle)
  double Dp[ND][ND];  // previous block's own-column L (rows of block b-1)
#pragma unroll
  for (int r = 0; r < ND; r++)
#pragma unroll
    for (int c = 0; c < ND; c++) Dp[r][c] = 0.0;
  for (int b = 0; b < B.nD; b++) {
    const double* hd = B.Hd + b * NN;
    const double* hl = B.Hl + b * NN;
    const int i0 = b * ND;
    if (b > 0) {
#pragma unroll
      for (int r = 0; r < ND; r++)
#pragma unroll
        for (int c = 0; c < ND; c++) {
          double s = hl[r * ND + c];
#pragma unroll
          for (int k = 0; k < c; k++) s -= C[r][k] * Dp[c][k];
          C[r][c] = s * inv[i0 - ND + c];
        }
    }
#pragma unroll
    for (int r = 0; r < ND; r++) {
#pragma unroll
      for (int c = 0; c <= r; c++) {
        double s = hd[r * ND + c] + (r == c ? lambda : 0.0);
        if (b > 0) {
#pragma unroll
          for (int k = 0; k < ND; k++) s -= C[r][k] * C[c][k];
        }
#pragma unroll
        for (int k = 0; k < c; k++) s -= Dg[r][k] * Dg[c][k];
        if (r == c) {
          if (!(s > 0.0)) return -1;
          const double d = sqrt(s);
          Dg[r][r] = d;
          inv[i0 + r] = 1.0 / d;
        } else {
          Dg[r][c] = s * inv[i0 + c];
        }
      }
    }
    // store row i0 + r as [block b-1 columns | block b columns] (2 * ND entries)
#pragma unroll
    for (int r = 0; r < ND; r++) {
      double* row = L + (i0 + r) * 2 * ND;
#pragma unroll
      for (int c = 0; c < ND; c++) {
        row[c] = b > 0 ? C[r][c] : 0.0;
        row[ND + c] = c <= r ? Dg[r][c] : 0.0;
        Dp[r][c] = c <= r ? Dg[r][c] : 0.0;
      }
    }
  }
  return 0;
}

// L y = b by block rows (ascending k per entry, as the dense forward substitution).
template <int ND>
__device__ void band_forward(const Band<ND>& B, const double* L, const double* inv, const double* b, double* y) {
  for (int blk = 0; blk < B.nD; blk++) {
    const int i0 = blk * ND;
#pragma unroll
    for (int r = 0; r < ND; r++) {
      const double* row = L + (i0 + r) * 2 * ND;
      double s = b[i0 + r];
      if (blk > 0) {
#pragma unroll
        for (int k = 0; k < ND; k++) s -= row[k] * y[i0 - ND + k];
      }
#pragma unroll
      for (int k = 0; k < r; k++) s -= row[ND + k] * y[i0 + k];
      y[i0 + r] = s * inv[i0 + r];
    }
  }
}

// L^T x = y by block rows from the end (ascending k per entry, as the dense back substitution).
template <int ND>
__device__ void band_backward(const Band<ND>& B, const double* L, const double* inv, const double* y, double* x) {
  for (int blk = B.nD - 1; blk >= 0; blk--) {
    const int i0 = blk * ND;
#pragma unroll
    for (int r = ND - 1; r >= 0; r--) {
      double s = y[i0 + r];
#pragma unroll
      for (int k = r + 1; k < ND; k++) s -= L[(i0 + k) * 2 * ND + ND + r] * x[i0 + k];
      if (blk + 1 < B.nD) {
#pragma unroll
        for (int k = 0; k < ND; k++) s -= L[(i0 + ND + k) * 2 * ND + r] * x[i0 + ND + k];
      }
      x[i0 + r] = s * inv[i0 + r];
    }
  }
}

__device__ double norm2(int n, const double* v) {
  double s = 0;
  for (int i = 0; i < n; i++) s += v[i] * v[i];
  return sqrt(s);
}

template <int ND>
__device__ int subproblem(const Band<ND>& B, const double* g, double radius, double eps, int max_iter, double* p,
                          double* work) {
  const int P = B.P;
  double* L = work;
  double* inv = work + P * 2 * B.nd;
  double* y = inv + P;
  double* rhs = y + P;
  const double gnorm = norm2(P, g);
  if (gnorm == 0.0) {
    for (int i = 0; i < P; i++) p[i] = 0.0;
    return 0;
  }
  const double hinf = B.hinf, mindiag = B.mindiag;
  double lam_hi = gnorm / radius + hinf;
  double lam_lo = gnorm / radius - hinf;
  if (-mindiag > lam_lo) lam_lo = -mindiag;
  if (lam_lo < 0) lam_lo = 0;
  int have_p = 0, boundary = 1;
  double lambda = 0.0;
  for (int i = 0; i < P; i++) rhs[i] = -g[i];
  for (int it = 0; it < max_iter; it++) {
    // H + 0 I is the same matrix for every frame and step of the reference: its factor is computed
    // once (by this same band_chol, so the values are identical) and reused
    const double* Lc = L;
    const double* ic = inv;
    bool ok;
    if (lambda == 0.0 && B.L0 != nullptr) {
      ok = B.chol0_ok != 0;
      Lc = B.L0;
      ic = B.inv0;
    } else {
      ok = band_chol(B, lambda, L, inv) == 0;
    }
    if (!ok) {
      if (lambda > lam_lo) lam_lo = lambda;
      const double a = sqrt(lam_lo * lam_hi), b = lam_lo + 0.001 * (lam_hi - lam_lo);
      lambda = a > b ? a : b;
      continue;
    }
    band_forward(B, Lc, ic, rhs, y);
    band_backward(B, Lc, ic, y, p);
    have_p = 1;
    const double pn = norm2(P, p);
    if (lambda == 0.0 && pn <= radius) {
      boundary = 0;
      break;
    }
    if (fabs(pn - radius) <= eps * radius) break;
    if (pn < radius) {
      if (lambda < lam_hi) lam_hi = lambda;
    } else {
      if (lambda > lam_lo) lam_lo = lambda;
    }
    band_forward(B, Lc, ic, p, y);
    const double qn = norm2(P, y);
    const double r = pn / qn;
    double next = lambda + r * r * (pn - radius) / radius;
    if (!(next > lam_lo && next < lam_hi)) {
      const double a = sqrt(lam_lo * lam_hi), b = lam_lo + 0.001 * (lam_hi - lam_lo);
      next = a > b ? a : b;
    }
    lambda = next;
  }
  if (!have_p) {
    for (int i = 0; i < P; i++) p[i] = -g[i] * (radius / gnorm);
  } else if (boundary) {
    const double pn = norm2(P, p);
    if (pn > radius) {
      const double s = radius / pn;
      for (int i = 0; i < P; i++) p[i] *= s;
    }
  }
  return boundary;
}

// Predicted reduction -(g.p + 0.5 p.H.p) with the dense algorithm's summation order: row i of H p
// sums over ascending j within the band (blocks b-1, b, b+1 of row block b).
template <int ND>
__device__ double predicted(const Band<ND>& B, const double* g, const double* p) {
  constexpr int NN = ND * ND;
  double gp = 0, pHp = 0;
  for (int b = 0; b < B.nD; b++) {
    const double* hl0 = B.Hl + b * NN;        // block (b, b-1)
    const double* hd = B.Hd + b * NN;         // block (b, b)
    const double* hl1 = B.Hl + (b + 1) * NN;  // block (b+1, b), read transposed
#pragma unroll
    for (int a = 0; a < ND; a++) {
      const int i = b * ND + a;
      double s = 0;
      if (b > 0) {
#pragma unroll
        for (int c = 0; c < ND; c++) s += hl0[a * ND + c] * p[(b - 1) * ND + c];
      }
#pragma unroll
      for (int c = 0; c < ND; c++) s += hd[a * ND + c] * p[b * ND + c];
      if (b + 1 < B.nD) {
#pragma unroll
        for (int c = 0; c < ND; c++) s += hl1[c * ND + a] * p[(b + 1) * ND + c];
      }
      gp += g[i] * p[i];
      pHp += p[i] * s;
    }
  }
  return -(gp + 0.5 * pHp);
}

// Start a new trust-region iteration if the stop rule allows it. Returns false when done.
template <int ND>
__device__ bool loop_top(FrameState* S, const Band<ND>& B, const double* g, double* p, double* work) {
  if (S->max_iter > 0 && S->iter >= S->max_iter) {
    S->hit_max = 1;
    return false;
  }
  if (S->have_prev && fabs(S->f - S->f_prev) < kMinDelta) return false;
  S->have_prev = 1;
  S->f_prev = S->f;
  S->iter++;
  S->boundary = subproblem(B, g, S->radius, 0.1, 20, p, work);
  return true;
}

}  // namespace

// Doubles of shared memory one frame's solve uses when staged: Hessian blocks, band factor,
// 1/L_ii, two work vectors, g and p, and a copy of the reference's cached factor of H (and its 1/L_ii),
// which the serial chain of every interior step reads.
__host__ __device__ inline long long solve_smem_doubles(int nD, int nd) {
  const long long P = (long long)nD * nd;
  return 2LL * nD * nd * nd + 2 * (P * 2 * nd) + 6 * P;
}

// The trust-region state machine for one frame after a fused pass at its trial point (thread 0).
template <int ND>
__device__ void state_step(const Job& job, FrameState* S, const RefDev& R, const double* Hd, const double* Hl,
                           const double* L0, const double* inv0, double* gv, double* pv, double* work, double ft,
                           double ft2) {
  const int P = R.P, nd = ND;
  Band<ND> B{Hd, Hl, R.nD, P, R.h_inf, R.h_mindiag, L0, inv0, R.chol0_ok};
  double* x = job.x;
  double* g = gv;
  double* p = pv;
  const double* gt = job.gt;
  bool go_top = false, done = false;
  int next = kPhaseTrial;
  S->evaluations++;
  switch (S->phase) {
    case kPhaseStartZero: {
      S->f_start = ft;
      for (int i = 0; i < P; i++) g[i] = gt[i];
      bool rigid = false;
      for (int c = 0; c < nd; c++) rigid = rigid || (S->rigid[c] != 0.0);
      if (rigid) {
        for (int k = 0; k < R.nD; k++)
          for (int c = 0; c < nd; c++) p[k * nd + c] = S->rigid[c];
        next = kPhaseStartRigid;
      } else {
        S->f = ft;
        if (S->use_warm && S->warm != nullptr) {
          next = kPhaseWaitWarm;
        } else {
          go_top = true;
        }
      }
      break;
    }
    case kPhaseStartPair: {
      // Both cold starting points from one pass: ft, gt at zero; ft2 and (in p) its gradient at the
      // rigid shift. The same choice as kPhaseStartZero followed by kPhaseStartRigid.
      S->evaluations++;
      S->f_start = ft;
      if (ft2 < ft) {
        for (int k = 0; k < R.nD; k++)
          for (int c = 0; c < nd; c++) {
            x[k * nd + c] = S->rigid[c];
            g[k * nd + c] = p[k * nd + c];
          }
        S->f = ft2;
      } else {
        for (int i = 0; i < P; i++) g[i] = gt[i];
        S->f = ft;
      }
      if (S->use_warm && S->warm != nullptr) {
        next = kPhaseWaitWarm;
      } else {
        go_top = true;
      }
      break;
    }
    case kPhaseStartRigid: {
      // Starting points {0, 0, rigid}: std::min_element keeps the first minimum
      // (FrameWarpAligner.cpp:194-198).
      if (ft < S->f_start) {
        for (int i = 0; i < P; i++) {
          x[i] = p[i];
          g[i] = gt[i];
        }
        S->f = ft;
      } else {
        S->f = S->f_start;
      }
      if (S->use_warm && S->warm != nullptr) {
        // the warm start waits (out of the passes) until the earlier frame's solution is written;
        // the compact pass then sets p = warm - x and the trial point
        next = kPhaseWaitWarm;
      } else {
        go_top = true;
      }
      break;
    }
    case kPhaseStartLast: {
      // Warm start: the previous frame's solution as a fourth starting point after {0, 0, rigid};
      // only a strictly smaller value replaces the current start (first minimum kept). The trial
      // point was x + (warm - x), and that is the point taken.
      if (ft < S->f) {
        for (int i = 0; i < P; i++) {
          x[i] = x[i] + p[i];
          g[i] = gt[i];
        }
        S->f = ft;
      }
      go_top = true;
      break;
    }
    case kPhaseTrial: {
      const double pred = predicted(B, g, p);
      const double meas = S->f - ft;
      if (fabs(pred) <= fabs(meas) * kDblEps) {
        done = true;
        break;
      }
      const double rho = meas / fabs(pred);
      if (!isfinite(rho)) {
        done = true;
        break;
      }
      if (rho < 0.25) {
        S->radius *= 0.25;
        if (S->radius <= kRadius0 * kDblEps) {
          done = true;
          break;
        }
      } else if (rho > 0.75 && S->boundary) {
        S->radius = 2 * S->radius < kRadiusMax ? 2 * S->radius : kRadiusMax;
      }
      if (rho > 0) {
        for (int i = 0; i < P; i++) {
          x[i] = x[i] + p[i];
          g[i] = gt[i];
        }
        S->f = ft;
        S->accepted++;
      }
      if (!loop_top(S, B, g, p, work)) done = true;
      break;
    }
    default:
      done = true;
  }
  if (go_top) {
    for (int i = 0; i < P; i++) p[i] = 0.0;
    S->radius = kRadius0;
    S->iter = 0;
    S->have_prev = 0;
    if (!loop_top(S, B, g, p, work)) done = true;
  }
  S->phase = done ? kPhaseDone : next;
  }

__global__ void __launch_bounds__(kSolveThreads, 1) solve_kernel(const Job* __restrict__ jobs, int smem_cap_doubles,
                                                                 const int* __restrict__ active,
                                                                 const int* __restrict__ n_active) {
  extern __shared__ double s_dyn[];
  if (active != nullptr && (int)blockIdx.x >= *n_active) return;
  const Job& job = jobs[active != nullptr ? active[blockIdx.x] : blockIdx.x];
  FrameState* S = job.state;
  if (S->phase == kPhaseDone || S->phase == kPhaseWaitWarm) return;
  const RefDev& R = *job.ref;
  __shared__ double s_f, s_f2;
  reduce_partials(R, job.partials, &s_f, job.gt);
  // paired start: the rigid point's sums, its gradient into p (free until the first step)
  const bool pair = S->phase == kPhaseStartPair;
  if (pair) reduce_partials(R, job.partials2, &s_f2, job.p);
  __syncthreads();
  // Stage the Hessian blocks, g and p in shared memory when they fit; otherwise work in global.
  const int nn = R.n_dim * R.n_dim;
  const bool staged = solve_smem_doubles(R.nD, R.n_dim) <= smem_cap_doubles;
  const double* Hd = R.Hd;
  const double* Hl = R.Hl;
  double* work = job.work;
  double* gv = job.g;
  double* pv = job.p;
  const double* L0 = R.L0;
  const double* inv0 = R.inv0;
  if (staged) {
    double* sHd = s_dyn;
    double* sHl = sHd + R.nD * nn;
    double* sg = sHl + R.nD * nn;
    double* sp = sg + R.P;
    for (int i = threadIdx.x; i < R.nD * nn; i += blockDim.x) {
      sHd[i] = R.Hd[i];
      sHl[i] = R.Hl[i];
    }
    for (int i = threadIdx.x; i < R.P; i += blockDim.x) {
      sg[i] = job.g[i];
      sp[i] = job.p[i];
    }
    Hd = sHd;
    Hl = sHl;
    gv = sg;
    pv = sp;
    work = sp + R.P;
    if (R.L0 != nullptr) {  // after the subproblem's work area (factor, 1/L_ii, two vectors)
      double* sL0 = work + R.P * 2 * R.n_dim + 3 * R.P;
      double* sinv0 = sL0 + R.P * 2 * R.n_dim;
      for (int i = threadIdx.x; i < R.P * 2 * R.n_dim; i += blockDim.x) sL0[i] = R.L0[i];
      for (int i = threadIdx.x; i < R.P; i += blockDim.x) sinv0[i] = R.inv0[i];
      L0 = sL0;
      inv0 = sinv0;
    }
    __syncthreads();
  }
  const int P = R.P;
  if (threadIdx.x == 0) {
    if (R.n_dim == 3)
      state_step<3>(job, S, R, Hd, Hl, L0, inv0, gv, pv, work, s_f, pair ? s_f2 : 0.0);
    else
      state_step<2>(job, S, R, Hd, Hl, L0, inv0, gv, pv, work, s_f, pair ? s_f2 : 0.0);
  }
  __syncthreads();
  if (staged) {
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
      job.g[i] = gv[i];
      job.p[i] = pv[i];
    }
    __syncthreads();
  }
  if (S->phase == kPhaseDone) {
    // Finished in this step: report the state and parameters, and keep them as the warm start.
    if (job.report != nullptr) {
      if (threadIdx.x == 0) *static_cast<FrameState*>(job.report) = *S;
      double* xr = reinterpret_cast<double*>(static_cast<char*>(job.report) + kReportHeaderBytes);
      for (int i = threadIdx.x; i < P; i += blockDim.x) xr[i] = job.x[i];
    }
    if (S->warm != nullptr) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) S->warm[i] = job.x[i];
      if (threadIdx.x == 0 && S->warm_seq != nullptr) *S->warm_seq = S->seq;  // read by later launches
    }
    return;
  }
  if (S->phase == kPhaseWaitWarm) return;
  // Next trial point D = x + p, as the fused pass's control-point parameters.
  write_trial_dparams(job, R, threadIdx.x, blockDim.x);
}

cudaError_t launch_solve(const Job* jobs_dev, int n_jobs, int max_nD, int n_dim, cudaStream_t s, const int* active,
                         const int* n_active) {
  constexpr long long kCapBytes = 200 * 1024;
  long long need = solve_smem_doubles(max_nD, n_dim) * (long long)sizeof(double);
  int smem = need <= kCapBytes ? (int)need : 0;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
  }
  solve_kernel<<<n_jobs, kSolveThreads, smem, s>>>(jobs_dev, smem / (int)sizeof(double), active, n_active);
  return cudaGetLastError();
}

__global__ void chol0_kernel(const double* Hd, const double* Hl, int nD, int nd, double* L0, double* inv0, int* ok) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (nd == 3) {
    Band<3> B{Hd, Hl, nD, nD * 3, 0.0, 0.0};
    *ok = band_chol(B, 0.0, L0, inv0) == 0;
  } else {
    Band<2> B{Hd, Hl, nD, nD * 2, 0.0, 0.0};
    *ok = band_chol(B, 0.0, L0, inv0) == 0;
  }
}

cudaError_t launch_chol0(const double* Hd, const double* Hl, int nD, int nd, double* L0, double* inv0, int* ok,
                         cudaStream_t s) {
  chol0_kernel<<<1, 32, 0, s>>>(Hd, Hl, nD, nd, L0, inv0, ok);
  return cudaGetLastError();
}

__global__ void test_subproblem_kernel(const double* Hd, const double* Hl, int nD, int nd, double hinf,
                                       double mindiag, const double* g, double radius, double* p, int* boundary,
                                       double* work) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  // work: P*(2*nd) + 3*P doubles
  if (nd == 3) {
    Band<3> B{Hd, Hl, nD, nD * 3, hinf, mindiag};
    *boundary = subproblem(B, g, radius, 0.1, 20, p, work);
  } else {
    Band<2> B{Hd, Hl, nD, nD * 2, hinf, mindiag};
    *boundary = subproblem(B, g, radius, 0.1, 20, p, work);
  }
}

cudaError_t launch_test_subproblem(const double* Hd, const double* Hl, int nD, int nd, double hinf, double mindiag,
                                   const double* g, double radius, double* p_out, int* boundary_out, double* work,
                                   cudaStream_t s) {
  test_subproblem_kernel<<<1, 32, 0, s>>>(Hd, Hl, nD, nd, hinf, mindiag, g, radius, p_out, boundary_out, work);
  return cudaGetLastError();
}

}  // namespace fa
