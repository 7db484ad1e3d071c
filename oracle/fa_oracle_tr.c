/*
 * fa_oracle_tr.c -- the project's trust-region solver, CPU form (TEST INFRASTRUCTURE ONLY).
 *
 * The reference calls dlib::find_min_trust_region(objective_delta_stop_strategy(1e-8), model, x,
 * 40) at FrameAligner/FrameWarpAligner.cpp:205-209. dlib is an external, unversioned dependency
 * (FrameAligner/CMakeLists.txt:10, find_package(dlib REQUIRED), no lockfile) whose source is not
 * in the reference tree, so its exact step rules cannot be checked here: parity at this boundary is
 * UNPINNED. The CUDA library and this oracle share one algorithm instead, specified here:
 *
 *  Outer loop (Nocedal & Wright, Numerical Optimization 2nd ed., Algorithm 4.1, with eta = 0,
 *  Delta_max = 1000, Delta_0 = 40):
 *    f, g at x.  Before each iteration the stop rule is checked: after the first iteration, stop
 *    once |f - f_previous_check| < min_delta (1e-8), or after max_iter iterations.
 *    p = subproblem(H, g, Delta)
 *    f_new = f(x + p); predicted = -(g.p + 0.5 p.H.p); measured = f - f_new
 *    stop if |predicted| <= |measured| * DBL_EPSILON (the model step has vanished)
 *    rho = measured / |predicted|; stop if rho is not finite
 *    rho < 0.25 -> Delta *= 0.25 (stop if Delta <= Delta_0 * DBL_EPSILON)
 *    else rho > 0.75 and the step was on the trust-region boundary -> Delta = min(1000, 2 Delta)
 *    rho > 0 -> accept: x += p, f = f_new, g = g(x)
 *  Because f is unchanged after a rejected step, the |delta f| rule ends the solve at the first
 *  rejected step.
 *
 *  Subproblem (More & Sorensen, "Computing a trust region step", SIAM J. Sci. Stat. Comput. 4,
 *  1983; Nocedal & Wright Algorithm 4.3 with safeguards): lambda = 0 first; if H is positive
 *  definite and |p(0)| <= Delta the Newton step is returned. Otherwise Newton iterations on
 *  1/|p(lambda)| - 1/Delta with the update lambda += (|p|/|q|)^2 (|p| - Delta)/Delta, q = L^-1 p,
 *  kept inside the bracket [lambda_L, lambda_U] (lambda_U = |g|/Delta + |H|_inf,
 *  lambda_L = max(0, -min H_ii, |g|/Delta - |H|_inf)); a failed Cholesky raises lambda_L. The
 *  Cholesky factor keeps 1/L_ii per row; off-diagonal entries and the triangular solves multiply by
 *  it rather than divide.
 *  Stop when ||p| - Delta| <= eps * Delta (eps = 0.1) or after 20 iterations; a final step longer
 *  than Delta is scaled back onto the boundary.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fa_oracle.h"

/* Dense Cholesky of A + lambda I into L (lower, row-major) with inv[i] = 1 / L[i][i]; the
   off-diagonal entries and the triangular solves multiply by inv instead of dividing.
   Returns 0 on success. */
static int chol_shift(int n, const double* A, double lambda, double* L, double* inv) {
  for (int i = 0; i < n; i++) {
    for (int j = 0; j <= i; j++) {
      double s = A[(size_t)i * n + j] + (i == j ? lambda : 0.0);
      for (int k = 0; k < j; k++) s -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
      if (i == j) {
        if (!(s > 0.0)) return -1;
        L[(size_t)i * n + i] = sqrt(s);
        inv[i] = 1.0 / L[(size_t)i * n + i];
      } else {
        L[(size_t)i * n + j] = s * inv[j];
      }
    }
    for (int j = i + 1; j < n; j++) L[(size_t)i * n + j] = 0.0;
  }
  return 0;
}

static void forward(int n, const double* L, const double* inv, const double* b, double* y) {
  for (int i = 0; i < n; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= L[(size_t)i * n + k] * y[k];
    y[i] = s * inv[i];
  }
}

static void backward(int n, const double* L, const double* inv, const double* y, double* x) {
  for (int i = n - 1; i >= 0; i--) {
    double s = y[i];
    for (int k = i + 1; k < n; k++) s -= L[(size_t)k * n + i] * x[k];
    x[i] = s * inv[i];
  }
}

static double norm2(int n, const double* v) {
  double s = 0;
  for (int i = 0; i < n; i++) s += v[i] * v[i];
  return sqrt(s);
}

int or_tr_subproblem(int P, const double* H, const double* g, double radius, double eps, int max_iter, double* p) {
  double gnorm = norm2(P, g);
  if (gnorm == 0.0) {
    memset(p, 0, sizeof(double) * (size_t)P);
    return 0;
  }
  double hinf = 0, mindiag = H[0];
  for (int i = 0; i < P; i++) {
    double r = 0;
    for (int j = 0; j < P; j++) r += fabs(H[(size_t)i * P + j]);
    if (r > hinf) hinf = r;
    if (H[(size_t)i * P + i] < mindiag) mindiag = H[(size_t)i * P + i];
  }
  double lam_hi = gnorm / radius + hinf;
  double lam_lo = gnorm / radius - hinf;
  if (-mindiag > lam_lo) lam_lo = -mindiag;
  if (lam_lo < 0) lam_lo = 0;
  double* L = (double*)malloc(sizeof(double) * (size_t)P * P);
  double* inv = (double*)malloc(sizeof(double) * (size_t)P);
  double* y = (double*)malloc(sizeof(double) * (size_t)P);
  double* rhs = (double*)malloc(sizeof(double) * (size_t)P);
  int have_p = 0, boundary = 1;
  double lambda = 0.0;
  for (int i = 0; i < P; i++) rhs[i] = -g[i];
  for (int it = 0; it < max_iter; it++) {
    if (chol_shift(P, H, lambda, L, inv) != 0) {
      if (lambda > lam_lo) lam_lo = lambda;
      double a = sqrt(lam_lo * lam_hi), b = lam_lo + 0.001 * (lam_hi - lam_lo);
      lambda = a > b ? a : b;
      continue;
    }
    forward(P, L, inv, rhs, y);
    backward(P, L, inv, y, p);
    have_p = 1;
    double pn = norm2(P, p);
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
    forward(P, L, inv, p, y); /* q = L^-1 p */
    double qn = norm2(P, y);
    double r = pn / qn;
    double next = lambda + r * r * (pn - radius) / radius;
    if (!(next > lam_lo && next < lam_hi)) {
      double a = sqrt(lam_lo * lam_hi), b = lam_lo + 0.001 * (lam_hi - lam_lo);
      next = a > b ? a : b;
    }
    lambda = next;
  }
  if (!have_p) {
    for (int i = 0; i < P; i++) p[i] = -g[i] * (radius / gnorm);
  } else if (boundary) {
    double pn = norm2(P, p);
    if (pn > radius) {
      double s = radius / pn;
      for (int i = 0; i < P; i++) p[i] *= s;
    }
  }
  free(L);
  free(inv);
  free(y);
  free(rhs);
  return boundary;
}

int or_trust_region(int P, const double* H, double* x, double radius0, double min_delta, int max_iter,
                    or_feval_fn f, or_geval_fn gfn, void* ctx, or_tr_stats* st) {
  double* g = (double*)malloc(sizeof(double) * (size_t)P);
  double* p = (double*)malloc(sizeof(double) * (size_t)P);
  double* xn = (double*)malloc(sizeof(double) * (size_t)P);
  double* Hp = (double*)malloc(sizeof(double) * (size_t)P);
  double radius = radius0;
  double fx = f(ctx, x);
  gfn(ctx, x, g);
  int iter = 0, accepted = 0, have_prev = 0;
  double f_prev = 0;
  for (;;) {
    if (max_iter > 0 && iter >= max_iter) break;
    if (have_prev && fabs(fx - f_prev) < min_delta) break;
    have_prev = 1;
    f_prev = fx;
    iter++;
    int boundary = or_tr_subproblem(P, H, g, radius, 0.1, 20, p);
    for (int i = 0; i < P; i++) xn[i] = x[i] + p[i];
    double fn = f(ctx, xn);
    double gp = 0, pHp = 0;
    for (int i = 0; i < P; i++) {
      double s = 0;
      for (int j = 0; j < P; j++) s += H[(size_t)i * P + j] * p[j];
      Hp[i] = s;
    }
    for (int i = 0; i < P; i++) {
      gp += g[i] * p[i];
      pHp += p[i] * Hp[i];
    }
    double predicted = -(gp + 0.5 * pHp);
    double measured = fx - fn;
    if (fabs(predicted) <= fabs(measured) * DBL_EPSILON) break;
    double rho = measured / fabs(predicted);
    if (!isfinite(rho)) break;
    if (rho < 0.25) {
      radius *= 0.25;
      if (radius <= radius0 * DBL_EPSILON) break;
    } else if (rho > 0.75 && boundary) {
      radius = 2 * radius < 1000 ? 2 * radius : 1000;
    }
    if (rho > 0) {
      memcpy(x, xn, sizeof(double) * (size_t)P);
      fx = fn;
      gfn(ctx, x, g);
      accepted++;
    }
  }
  if (st) {
    st->iterations = iter;
    st->accepted = accepted;
    st->f_final = fx;
    st->radius_final = radius;
  }
  free(g);
  free(p);
  free(xn);
  free(Hp);
  return 0;
}
