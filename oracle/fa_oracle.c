/*
 * fa_oracle.c -- CPU restatement of frame-aligner's warper path (TEST INFRASTRUCTURE ONLY;
 * see fa_oracle.h for the function -> reference file:line map).
 *
 * Arithmetic types follow the reference exactly: images and gradients are float, scan times,
 * coordinates and interpolation weights are double, products of two floats are rounded to float
 * before being added to a double accumulator. Built with -ffp-contract=off so that no
 * multiply-add is fused (the reference is built for SSE3, which has no FMA).
 */
#include "fa_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct or_warper {
  int nz, ny, nx, nD, n_dim;
  long N;
  or_scan scan;
  float* ref;      /* N */
  uint16_t* Di;    /* N */
  float* Df;       /* N */
  int* rbegin;     /* nD */
  int* rend;       /* nD */
  float* gx;       /* N: Sobel gradient of the reference */
  float* gy;
  float* gz;
  /* Steepest-descent images VI_i over [vi0[i], vi1[i]) (reference: OffsetVector<Point3f>). */
  long* vi0;
  long* vi1;
  float** vi;      /* per control point: (vi1-vi0) x 3 floats */
  double* H;       /* P x P */
};

/* ImageScanParameters::ImageScanParameters, ImageScanParameters.h:7-20 */
void or_scan_init(or_scan* s, double line_duration, double interline_duration, double interframe_duration,
                  int n_x, int n_y, int n_z, int bidirectional) {
  s->line_duration = line_duration;
  s->interline_duration = interline_duration;
  s->interframe_duration = interframe_duration;
  s->n_x = n_x < 1 ? 1 : n_x;
  s->n_y = n_y < 1 ? 1 : n_y;
  s->n_z = n_z;
  if (s->interline_duration < s->line_duration) s->interline_duration = 1.01 * s->line_duration;
  s->pixel_duration = s->line_duration / s->n_x;
  s->frame_duration = s->n_y * s->interline_duration;
  s->stack_duration = (s->n_z - 1) * s->interframe_duration + s->frame_duration;
  /* The reference constructor leaves `bidirectional` unset (ImageScanParameters.h:7-8);
     callers must state it, so it is an explicit argument here. */
  s->bidirectional = bidirectional;
}

/* AbstractFrameWarper::processScanParameters, FrameWarper.cpp:223-236 */
void or_process_scan(const or_scan* in, int nz, int nD, or_scan* out) {
  *out = *in;
  double frame_interval_max = nz * in->frame_duration / (nD - nz);
  if ((in->interframe_duration - in->frame_duration) > frame_interval_max) {
    out->interframe_duration = out->frame_duration + frame_interval_max;
    out->stack_duration = (nz - 1) * out->interframe_duration + out->frame_duration;
  }
}

/* Sobel3d.cpp:8-21 (X), 23-36 (Y), 38-58 (Z) */
static void apply_filter(const float* m, float* out, int nz, int ny, int nx, int axis, const float f[3],
                         const float e1[2], const float e2[2]) {
#define AT(a, z, y, x) a[((long)(z) * ny + (y)) * nx + (x)]
  if (axis == 2) {
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 1; x < nx - 1; x++)
          AT(out, z, y, x) = f[0] * AT(m, z, y, x - 1) + f[1] * AT(m, z, y, x) + f[2] * AT(m, z, y, x + 1);
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
        AT(out, z, y, 0) = e1[0] * AT(m, z, y, 0) + e1[1] * AT(m, z, y, 1);
        AT(out, z, y, nx - 1) = e2[0] * AT(m, z, y, nx - 1) + e2[1] * AT(m, z, y, nx - 2);
      }
  } else if (axis == 1) {
    for (int z = 0; z < nz; z++)
      for (int y = 1; y < ny - 1; y++)
        for (int x = 0; x < nx; x++)
          AT(out, z, y, x) = f[0] * AT(m, z, y - 1, x) + f[1] * AT(m, z, y, x) + f[2] * AT(m, z, y + 1, x);
    for (int z = 0; z < nz; z++)
      for (int x = 0; x < nx; x++) {
        AT(out, z, 0, x) = e1[0] * AT(m, z, 0, x) + e1[1] * AT(m, z, 1, x);
        AT(out, z, ny - 1, x) = e2[0] * AT(m, z, ny - 1, x) + e2[1] * AT(m, z, ny - 2, x);
      }
  } else {
    if (nz == 1) {
      memcpy(out, m, sizeof(float) * (size_t)ny * nx);
      return;
    }
    for (int z = 1; z < nz - 1; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++)
          AT(out, z, y, x) = f[0] * AT(m, z - 1, y, x) + f[1] * AT(m, z, y, x) + f[2] * AT(m, z + 1, y, x);
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        AT(out, 0, y, x) = e1[0] * AT(m, 0, y, x) + e1[1] * AT(m, 1, y, x);
        AT(out, nz - 1, y, x) = e2[0] * AT(m, nz - 1, y, x) + e2[1] * AT(m, nz - 2, y, x);
      }
  }
#undef AT
}

/* sobel3d, Sobel3d.cpp:60-85 */
void or_sobel3d(const float* m, int nz, int ny, int nx, float* gx, float* gy, float* gz) {
  size_t n = (size_t)nz * ny * nx;
  float* a = (float*)malloc(n * sizeof(float));
  float* b = (float*)malloc(n * sizeof(float));
  float* c = (float*)malloc(n * sizeof(float));
  const float a1[3] = {1.0f / 4.0f, 2.0f / 4.0f, 1.0f / 4.0f};
  const float a2[2] = {2.0f / 3.0f, 2.0f / 3.0f};
  const float a3[2] = {2.0f / 3.0f, 2.0f / 3.0f};
  const float s1[3] = {-0.5f, 0.0f, 0.5f};
  const float s2[2] = {-0.5f, 0.5f};
  const float s3[2] = {0.5f, -0.5f};
  apply_filter(m, a, nz, ny, nx, 2, a1, a2, a3);
  apply_filter(a, b, nz, ny, nx, 1, a1, a2, a3);
  apply_filter(a, c, nz, ny, nx, 0, a1, a2, a3);
  apply_filter(b, gz, nz, ny, nx, 0, s1, s2, s3);
  apply_filter(c, gy, nz, ny, nx, 1, s1, s2, s3);
  apply_filter(m, a, nz, ny, nx, 1, a1, a2, a3);
  apply_filter(a, b, nz, ny, nx, 0, a1, a2, a3);
  apply_filter(b, gx, nz, ny, nx, 2, s1, s2, s3);
  free(a);
  free(b);
  free(c);
}

/* AbstractFrameWarper::precomputeInterp, FrameWarper.cpp:239-293 */
static int precompute_interp(or_warper* w, char* err) {
  or_scan p;
  or_process_scan(&w->scan, w->nz, w->nD, &p);
  int nD = w->nD;
  for (int k = 0; k < nD; k++) w->rbegin[k] = w->rend[k] = 0;
  int i = 0;
  int last_i = -1;
  for (int z = 0; z < w->nz; z++)
    for (int y = 0; y < w->ny; y++)
      for (int x = 0; x < w->nx; x++) {
        double t = z * p.interframe_duration + y * p.interline_duration + x * p.pixel_duration;
        double Di_xy;
        double f = modf(t / p.stack_duration * (nD - 1), &Di_xy);
        i = (int)Di_xy;
        int x_true = x;
        if (w->scan.bidirectional && ((y % 2) == 1)) x_true = w->nx - x - 1;
        long idx = ((long)z * w->ny + y) * w->nx + x_true;
        w->Di[idx] = (uint16_t)i;
        w->Df[idx] = (float)f;
        if (i > last_i) {
          if (i < 0 || i >= nD) {
            if (err) snprintf(err, 128, "Something went wrong");
            return -1;
          }
          w->rbegin[i] = (int)idx;
          if (last_i >= 0) w->rend[last_i] = w->rbegin[i] - 1;
          last_i = i;
        }
      }
  if ((long)i != (long)nD - 2) {
    if (err) snprintf(err, 128, "Something went wrong");
    return -1;
  }
  w->rend[i] = (int)(w->N - 1);
  for (int k = 0; k < nD; k++) {
    int a = k - 1 < 0 ? 0 : k - 1;
    int b = k < nD - 2 ? k : nD - 2;
    long i0 = w->rbegin[a];
    long i1 = w->rend[b];
    w->vi0[k] = i0;
    w->vi1[k] = i1 < i0 ? i0 : i1;
    long n = w->vi1[k] - w->vi0[k];
    w->vi[k] = (float*)calloc((size_t)(n > 0 ? n : 1) * 3, sizeof(float));
  }
  return 0;
}

static inline float* vi_at(const or_warper* w, int k, long p) { return w->vi[k] + (p - w->vi0[k]) * 3; }

/* AbstractFrameWarper::computeSteepestDecentImages, FrameWarper.cpp:296-345 */
static void steepest_descent(or_warper* w) {
  int nD = w->nD;
  for (int k = 1; k < nD; k++) {
    long p0 = w->rbegin[k - 1], p1 = w->rend[k - 1];
    if (w->vi1[k] - w->vi0[k] > 0)
      for (long p = p0; p < p1; p++) {
        /* Scan geometries whose ranges are not increasing in storage order would make the
           reference write outside the OffsetVector; the restatement skips those voxels. */
        if (p < w->vi0[k] || p >= w->vi1[k]) continue;
        float* dp = vi_at(w, k, p);
        double jac = w->Df[p];
        dp[0] = (float)(w->gx[p] * jac);
        dp[1] = (float)(w->gy[p] * jac);
        if (w->n_dim == 3) dp[2] = (float)(w->gz[p] * jac);
      }
  }
  for (int k = 0; k < nD - 1; k++) {
    long p0 = w->rbegin[k], p1 = w->rend[k];
    for (long p = p0; p < p1; p++) {
      if (p < w->vi0[k] || p >= w->vi1[k]) continue;
      float* dp = vi_at(w, k, p);
      double jac = 1 - w->Df[p]; /* int - float: evaluated in float, as in the reference */
      dp[0] = (float)(w->gx[p] * jac);
      dp[1] = (float)(w->gy[p] * jac);
      if (w->n_dim == 3) dp[2] = (float)(w->gz[p] * jac);
    }
  }
}

/* OffsetVector::at, FrameWarper.h:72-77 */
static inline float vi_get(const or_warper* w, int k, long p, int d) {
  if (p < w->vi0[k] || p > w->vi1[k]) return 0.0f;
  return vi_at(w, k, p)[d];
}

/* computeHessianEntry / computeHessian, FrameWarper.cpp:347-395 */
static double hessian_entry(const or_warper* w, int pi, int pj) {
  int nd = w->n_dim;
  int i = pi / nd, j = pj / nd, di = pi % nd, dj = pj % nd;
  if (j > i) return hessian_entry(w, pj, pi);
  if ((i - j) > 1) return 0;
  long p0 = w->vi0[i] > w->vi0[j] ? w->vi0[i] : w->vi0[j];
  long p1 = w->vi1[i] < w->vi1[j] ? w->vi1[i] : w->vi1[j];
  double h = 0;
  for (long p = p0; p < p1; p++) {
    float prod = vi_get(w, i, p, di) * vi_get(w, j, p, dj);
    h += prod;
  }
  return h;
}

or_warper* or_warper_create(const float* reference, int nz, int ny, int nx, int nD, const or_scan* scan, char* err) {
  if (nz < 1 || ny < 2 || nx < 2 || nD < 2) {
    if (err) snprintf(err, 128, "bad dimensions");
    return NULL;
  }
  or_warper* w = (or_warper*)calloc(1, sizeof(or_warper));
  w->nz = nz;
  w->ny = ny;
  w->nx = nx;
  w->nD = nD;
  w->N = (long)nz * ny * nx;
  w->n_dim = nz > 1 ? 3 : 2;
  w->scan = *scan;
  size_t N = (size_t)w->N;
  w->ref = (float*)malloc(N * sizeof(float));
  memcpy(w->ref, reference, N * sizeof(float));
  w->Di = (uint16_t*)malloc(N * sizeof(uint16_t));
  w->Df = (float*)malloc(N * sizeof(float));
  w->rbegin = (int*)calloc((size_t)nD, sizeof(int));
  w->rend = (int*)calloc((size_t)nD, sizeof(int));
  w->vi0 = (long*)calloc((size_t)nD, sizeof(long));
  w->vi1 = (long*)calloc((size_t)nD, sizeof(long));
  w->vi = (float**)calloc((size_t)nD, sizeof(float*));
  if (precompute_interp(w, err) != 0) {
    or_warper_destroy(w);
    return NULL;
  }
  w->gx = (float*)malloc(N * sizeof(float));
  w->gy = (float*)malloc(N * sizeof(float));
  w->gz = (float*)malloc(N * sizeof(float));
  or_sobel3d(w->ref, nz, ny, nx, w->gx, w->gy, w->gz);
  steepest_descent(w);
  int P = nD * w->n_dim;
  w->H = (double*)malloc(sizeof(double) * (size_t)P * P);
  for (int i = 0; i < P; i++)
    for (int j = 0; j <= i; j++) {
      double h = hessian_entry(w, i, j);
      w->H[(size_t)i * P + j] = h;
      w->H[(size_t)j * P + i] = h;
    }
  return w;
}

void or_warper_destroy(or_warper* w) {
  if (!w) return;
  if (w->vi)
    for (int k = 0; k < w->nD; k++) free(w->vi[k]);
  free(w->vi);
  free(w->vi0);
  free(w->vi1);
  free(w->ref);
  free(w->Di);
  free(w->Df);
  free(w->rbegin);
  free(w->rend);
  free(w->gx);
  free(w->gy);
  free(w->gz);
  free(w->H);
  free(w);
}

int or_warper_n_dim(const or_warper* w) { return w->n_dim; }

void or_warper_precomp(const or_warper* w, uint16_t* Di, float* Df, int* ranges) {
  if (Di) memcpy(Di, w->Di, sizeof(uint16_t) * (size_t)w->N);
  if (Df) memcpy(Df, w->Df, sizeof(float) * (size_t)w->N);
  if (ranges)
    for (int k = 0; k < w->nD; k++) {
      ranges[2 * k] = w->rbegin[k];
      ranges[2 * k + 1] = w->rend[k];
    }
}

void or_warper_hessian(const or_warper* w, double* H) {
  int P = w->nD * w->n_dim;
  memcpy(H, w->H, sizeof(double) * (size_t)P * P);
}

void or_warper_gradient(const or_warper* w, float* gx, float* gy, float* gz) {
  size_t n = (size_t)w->N * sizeof(float);
  if (gx) memcpy(gx, w->gx, n);
  if (gy) memcpy(gy, w->gy, n);
  if (gz) memcpy(gz, w->gz, n);
}

/* AbstractFrameWarper::warpPoint, FrameWarper.cpp:397-419 */
void or_warp_point(const or_warper* w, const double* D, int x, int y, int z, int spatial_binning, double* out3) {
  double factor = 1.0 / spatial_binning;
  int xs = (int)(x / factor);
  int ys = (int)(y / factor);
  if ((xs < 0) || (xs >= w->nx) || (ys < 0) || (ys >= w->ny) || (z < 0) || (z >= w->nz)) {
    out3[0] = out3[1] = out3[2] = 0;
    return;
  }
  long loc = ((long)z * w->ny + ys) * w->nx + xs;
  double f = w->Df[loc];
  int i = w->Di[loc];
  for (int c = 0; c < 3; c++) {
    double v = f * D[3 * (i + 1) + c] + (1 - f) * D[3 * i + c];
    out3[c] = v * factor;
  }
}

/* getZeroPadded, FrameWarper.h:39-47. A 2-D image ignores z (the reference never passes a
   non-zero plane there as long as the displacement has no z component). */
static inline float zero_padded(const float* img, int nz, int ny, int nx, int z, int y, int x) {
  int valid = (x >= 0) && (x < nx) && (y >= 0) && (y < ny) && ((nz == 1) || ((z >= 0) && (z < nz)));
  if (!valid) return 0.0f;
  if (nz == 1) z = 0;
  return img[((long)z * ny + y) * nx + x];
}

/* CpuFrameWarper::warpImageInterpolated, FrameWarper.cpp:31-69 */
void or_warp_interpolated(const or_warper* w, const float* img, const double* D, float invalid_value, float* out) {
  int nz = w->nz, ny = w->ny, nx = w->nx;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        double d[3];
        or_warp_point(w, D, x, y, z, 1, d);
        double lx = d[0] + x, ly = d[1] + y, lz = d[2] + z;
        int x0 = (int)floor(lx), y0 = (int)floor(ly), z0 = (int)floor(lz);
        double fx = lx - x0, fy = ly - y0, fz = lz - z0;
        int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
        float px = (float)((1 - fz) * (zero_padded(img, nz, ny, nx, z0, y0, x0) * (1 - fy) * (1 - fx) +
                                       zero_padded(img, nz, ny, nx, z0, y1, x0) * (fy) * (1 - fx) +
                                       zero_padded(img, nz, ny, nx, z0, y0, x1) * (1 - fy) * (fx) +
                                       zero_padded(img, nz, ny, nx, z0, y1, x1) * (fy) * (fx)));
        if (w->n_dim == 3)
          px = (float)(px + fz * (zero_padded(img, nz, ny, nx, z1, y0, x0) * (1 - fy) * (1 - fx) +
                                  zero_padded(img, nz, ny, nx, z1, y1, x0) * (fy) * (1 - fx) +
                                  zero_padded(img, nz, ny, nx, z1, y0, x1) * (1 - fy) * (fx) +
                                  zero_padded(img, nz, ny, nx, z1, y1, x1) * (fy) * (fx)));
        if (px == 0) px = invalid_value;
        out[((long)z * ny + y) * nx + x] = px;
      }
}

/* CpuFrameWarper::getError + computeErrorImage, FrameWarper.cpp:169-176, 4-29 */
double or_get_error(const or_warper* w, const float* frame, const double* D, float* err) {
  size_t N = (size_t)w->N;
  float* wimg = (float*)malloc(N * sizeof(float));
  float* e = err ? err : (float*)malloc(N * sizeof(float));
  or_warp_interpolated(w, frame, D, -1.0f, wimg);
  for (size_t p = 0; p < N; p++) e[p] = wimg[p] - w->ref[p];
  double ms_error = 0;
  for (size_t p = 0; p < N; p++) {
    if (wimg[p] >= 0) {
      float sq = e[p] * e[p];
      ms_error += sq;
    } else {
      e[p] = 0;
      wimg[p] = 0;
    }
  }
  free(wimg);
  if (!err) free(e);
  return ms_error;
}

/* AbstractFrameWarper::computeJacobian, FrameWarper.cpp:147-167 */
void or_get_jacobian(const or_warper* w, const float* err, double* jac) {
  int nd = w->n_dim;
  int P = w->nD * nd;
  for (int k = 0; k < P; k++) jac[k] = 0;
  for (int i = 0; i < w->nD; i++) {
    long p0 = w->vi0[i], p1 = w->vi1[i];
    for (long p = p0; p < p1; p++) {
      const float* v = vi_at(w, i, p);
      float t0 = v[0] * err[p];
      float t1 = v[1] * err[p];
      jac[i * nd] += t0;
      jac[i * nd + 1] += t1;
      if (nd == 3) {
        float t2 = v[2] * err[p];
        jac[i * nd + 2] += t2;
      }
    }
  }
}

/* AbstractFrameWarper::warpImage, FrameWarper.cpp:71-136 (forward splat + coverage) */
void or_warp_image(const or_warper* w, const float* img, const double* D, float* wimg, float* coverage) {
  int nz = w->nz, ny = w->ny, nx = w->nx;
  size_t N = (size_t)w->N;
  for (size_t p = 0; p < N; p++) wimg[p] = coverage[p] = 0;
#define AT(a, z, y, x) a[((long)(z) * ny + (y)) * nx + (x)]
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        double d[3];
        or_warp_point(w, D, x, y, z, 1, d);
        double lx = x - d[0], ly = y - d[1], lz = z - d[2];
        int x0 = (int)floor(lx), y0 = (int)floor(ly), z0 = (int)floor(lz);
        double fx = lx - x0, fy = ly - y0, fz = lz - z0;
        /* The reference clamps loc after loc0/locf are taken; those clamps change nothing used
           below (FrameWarper.cpp:87-94). */
        int x1 = x0, y1 = y0, z1 = z0;
        if (x1 < nx - 1) x1++;
        if (y1 < ny - 1) y1++;
        if (z1 < nz - 1) z1++;
        int valid = (x0 >= 0) && (y0 >= 0) && (x0 <= nx - 1) && (y0 <= ny - 1);
        if (nz > 1) valid = valid && (z0 >= 0) && (z0 <= nz - 1);
        if (valid) {
          float v = AT(img, z, y, x);
          AT(wimg, z0, y0, x0) += (1 - fy) * (1 - fx) * (1 - fz) * v;
          AT(wimg, z0, y1, x0) += (fy) * (1 - fx) * (1 - fz) * v;
          AT(wimg, z0, y0, x1) += (1 - fy) * (fx) * (1 - fz) * v;
          AT(wimg, z0, y1, x1) += (fy) * (fx) * (1 - fz) * v;
          AT(wimg, z1, y0, x0) += (1 - fy) * (1 - fx) * fz * v;
          AT(wimg, z1, y1, x0) += (fy) * (1 - fx) * fz * v;
          AT(wimg, z1, y0, x1) += (1 - fy) * (fx) * fz * v;
          AT(wimg, z1, y1, x1) += (fy) * (fx) * fz * v;
          AT(coverage, z0, y0, x0) += (1 - fy) * (1 - fx) * (1 - fz);
          AT(coverage, z0, y1, x0) += (fy) * (1 - fx) * (1 - fz);
          AT(coverage, z0, y0, x1) += (1 - fy) * (fx) * (1 - fz);
          AT(coverage, z0, y1, x1) += (fy) * (fx) * (1 - fz);
          AT(coverage, z1, y0, x0) += (1 - fy) * (1 - fx) * fz;
          AT(coverage, z1, y1, x0) += (fy) * (1 - fx) * fz;
          AT(coverage, z1, y0, x1) += (1 - fy) * (fx) * fz;
          AT(coverage, z1, y1, x1) += (fy) * (fx) * fz;
        }
      }
#undef AT
}

/* downsample, AbstractFrameAligner.cpp:37-56 */
void or_downsample(const float* in, int nz, int ny, int nx, int factor, float* out) {
  int nh = (int)ceil(ny / (double)factor);
  int nw = (int)ceil(nx / (double)factor);
  for (long i = 0; i < (long)nz * nh * nw; i++) out[i] = 0;
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++)
        out[((long)z * nh + y / factor) * nw + x / factor] += in[((long)z * ny + y) * nx + x];
}

/* smoothStack, FrameWarpAligner.cpp:46-64: per plane cv::GaussianBlur(plane, Size(0, 0), sigma, 1)
   on float data. OpenCV is not part of this build, so this states its documented algorithm (parity
   with OpenCV itself is unpinned): kernel size cvRound(8 s + 1) | 1 for float images; weights
   exp(-x^2 / (2 s^2)) at x = i - (n - 1) / 2, rounded to float, summed in double and scaled by the
   reciprocal of the sum (rounded to float again); a row pass summing taps in kernel order, then a
   column pass in the symmetric form k_c T[y] + sum_k k_{c+k} (T[y-k] + T[y+k]); BORDER_REFLECT_101
   at the edges; float arithmetic with every product and sum rounded. */
int or_gaussian_kernel(double sigma, float* k, int max_n) {
  int n = (int)nearbyint(sigma * 8 + 1) | 1;
  if (n > max_n) return -1;
  double scale2 = -0.5 / (sigma * sigma), sum = 0;
  for (int i = 0; i < n; i++) {
    double x = i - (n - 1) * 0.5;
    k[i] = (float)exp(scale2 * x * x);
    sum += k[i];
  }
  sum = 1.0 / sum;
  for (int i = 0; i < n; i++) k[i] = (float)(k[i] * sum);
  return n;
}

static int reflect101(int p, int n) {
  if (n == 1) return 0;
  while (p < 0 || p >= n) {
    if (p < 0) p = -p;
    if (p >= n) p = 2 * n - 2 - p;
  }
  return p;
}

int or_smooth_stack(const float* in, int nz, int ny, int nx, double sigma, float* out) {
  float kx[257], ky[257];
  int nkx = or_gaussian_kernel(sigma, kx, 257), nky = or_gaussian_kernel(1.0, ky, 257);
  if (nkx < 0 || nky < 0) return -1;
  int rx = nkx / 2, ry = nky / 2;
  float* t = (float*)malloc(sizeof(float) * (size_t)ny * nx);
  for (int z = 0; z < nz; z++) {
    const float* src = in + (size_t)z * ny * nx;
    float* dst = out + (size_t)z * ny * nx;
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        float s = kx[0] * src[(size_t)y * nx + reflect101(x - rx, nx)];
        for (int i = 1; i < nkx; i++) s += kx[i] * src[(size_t)y * nx + reflect101(x + i - rx, nx)];
        t[(size_t)y * nx + x] = s;
      }
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        float s = ky[ry] * t[(size_t)y * nx + x];
        for (int k = 1; k <= ry; k++)
          s += ky[ry + k] * (t[(size_t)reflect101(y - k, ny) * nx + x] + t[(size_t)reflect101(y + k, ny) * nx + x]);
        dst[(size_t)y * nx + x] = s;
      }
  }
  free(t);
  return 0;
}

/* correlation, Cv3dUtils.cpp:57-81: covariance over the mask divided by the product of the
   population standard deviations over the mask. */
double or_correlation(const float* a, const float* b, const uint8_t* mask, long n) {
  double sa = 0, sb = 0, saa = 0, sbb = 0, cnt = 0;
  for (long i = 0; i < n; i++)
    if (mask[i]) {
      sa += a[i];
      sb += b[i];
      saa += (double)a[i] * a[i];
      sbb += (double)b[i] * b[i];
      cnt += 1;
    }
  if (cnt == 0) return 0;
  double ma = sa / cnt, mb = sb / cnt;
  double va = saa / cnt - ma * ma, vb = sbb / cnt - mb * mb;
  double sda = sqrt(va > 0 ? va : 0), sdb = sqrt(vb > 0 ? vb : 0);
  double cov = 0;
  for (long i = 0; i < n; i++)
    if (mask[i]) cov += ((double)a[i] - ma) * ((double)b[i] - mb);
  cov /= cnt;
  return cov / (sda * sdb);
}

/* ---------------- per-frame alignment driver (FrameWarpAligner.cpp:117-219) ---------------- */

typedef struct {
  const or_warper* w;
  const float* frame;
  float* err;        /* error image of the last objective evaluation */
  double* last_x;
  double* D;
  int have_last;
  int evaluations;
} or_model;

static void col_to_D(const or_warper* w, const double* x, double* D) {
  int nd = w->n_dim;
  for (int i = 0; i < w->nD; i++) {
    D[3 * i] = x[i * nd];
    D[3 * i + 1] = x[i * nd + 1];
    D[3 * i + 2] = nd == 3 ? x[i * nd + 2] : 0.0;
  }
}

/* OptimisationModel::operator(), OptimisationModel.cpp:45-53 */
static double model_f(void* ctx, const double* x) {
  or_model* m = (or_model*)ctx;
  int P = m->w->nD * m->w->n_dim;
  col_to_D(m->w, x, m->D);
  double f = or_get_error(m->w, m->frame, m->D, m->err);
  memcpy(m->last_x, x, sizeof(double) * (size_t)P);
  m->have_last = 1;
  m->evaluations++;
  return f;
}

/* OptimisationModel::get_derivative_and_hessian, OptimisationModel.cpp:55-62: J^T e from the
   error image that the last objective evaluation on this frame left behind. */
static void model_g(void* ctx, const double* x, double* g) {
  or_model* m = (or_model*)ctx;
  int P = m->w->nD * m->w->n_dim;
  if (!m->have_last || memcmp(m->last_x, x, sizeof(double) * (size_t)P) != 0) model_f(ctx, x);
  or_get_jacobian(m->w, m->err, g);
}

int or_align_frame(const or_warper* w, const float* frame, const double* rigid_shift, int max_iter, double* D_out,
                   or_tr_stats* st) {
  return or_align_frame_warm(w, frame, rigid_shift, NULL, max_iter, D_out, st);
}

int or_align_frame_warm(const or_warper* w, const float* frame, const double* rigid_shift, const double* warm_D,
                        int max_iter, double* D_out, or_tr_stats* st) {
  int nd = w->n_dim, nD = w->nD, P = nD * nd;
  or_model m;
  memset(&m, 0, sizeof(m));
  m.w = w;
  m.frame = frame;
  m.err = (float*)malloc(sizeof(float) * (size_t)w->N);
  m.last_x = (double*)malloc(sizeof(double) * (size_t)P);
  m.D = (double*)malloc(sizeof(double) * 3 * (size_t)nD);
  double* start[3];
  for (int s = 0; s < 3; s++) start[s] = (double*)calloc((size_t)P, sizeof(double));
  for (int i = 0; i < nD; i++)
    for (int c = 0; c < nd; c++) start[2][i * nd + c] = rigid_shift[c];
  /* FrameWarpAligner.cpp:194-198: evaluate each starting point, take the first minimum. */
  double fe[3];
  for (int s = 0; s < 3; s++) fe[s] = model_f(&m, start[s]);
  int best = 0;
  for (int s = 1; s < 3; s++)
    if (fe[s] < fe[best]) best = s;
  double* x = (double*)malloc(sizeof(double) * (size_t)P);
  memcpy(x, start[best], sizeof(double) * (size_t)P);
  if (warm_D) {
    /* Warm start (the serving loop's extension): the previous frame's solution is a fourth
       candidate, reached as x + (warm - x) from the chosen start and kept only if strictly better. */
    double* t = (double*)malloc(sizeof(double) * (size_t)P);
    for (int k = 0; k < nD; k++)
      for (int c = 0; c < nd; c++) {
        int i = k * nd + c;
        double p = warm_D[3 * k + c] - x[i];
        t[i] = x[i] + p;
      }
    if (model_f(&m, t) < fe[best]) memcpy(x, t, sizeof(double) * (size_t)P);
    free(t);
  }
  or_tr_stats local;
  if (!st) st = &local;
  int rc = or_trust_region(P, w->H, x, 40.0, 1e-8, max_iter, model_f, model_g, &m, st);
  st->evaluations = m.evaluations;
  col_to_D(w, x, D_out);
  for (int s = 0; s < 3; s++) free(start[s]);
  free(x);
  free(m.err);
  free(m.last_x);
  free(m.D);
  return rc;
}

typedef struct {
  const or_warper* w;
  const float* frames;
  const double* rigid;
  int n_frames, max_iter, n_threads, tid;
  double* D_out;
  int* iters;
} or_mt_job;

static void* mt_worker(void* arg) {
  or_mt_job* j = (or_mt_job*)arg;
  for (int f = j->tid; f < j->n_frames; f += j->n_threads) {
    or_tr_stats st;
    or_align_frame(j->w, j->frames + (size_t)f * j->w->N, j->rigid ? j->rigid + 3 * f : (const double[3]){0, 0, 0},
                   j->max_iter, j->D_out + (size_t)f * 3 * j->w->nD, &st);
    if (j->iters) j->iters[f] = st.iterations;
  }
  return NULL;
}

int or_align_frames_mt(const or_warper* w, const float* frames, int n_frames, const double* rigid_shifts,
                       int max_iter, int n_threads, double* D_out, int* iterations_out) {
  if (n_threads < 1) n_threads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  or_mt_job* jobs = (or_mt_job*)malloc(sizeof(or_mt_job) * (size_t)n_threads);
  for (int t = 0; t < n_threads; t++) {
    or_mt_job j = {w, frames, rigid_shifts, n_frames, max_iter, n_threads, t, D_out, iterations_out};
    jobs[t] = j;
    pthread_create(&th[t], NULL, mt_worker, &jobs[t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
  return 0;
}
