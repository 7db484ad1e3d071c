/*
 * fa_synth.c -- seeded synthetic acquisitions for tests and benchmarks (host code).
 *
 * A reference is a background plus a sum of axis-aligned anisotropic Gaussian blobs. A frame is
 * that continuous reference sampled at x - d(t(x)), where d is the scan-time piecewise-linear
 * displacement of the warper model (control points D, interval from the voxel's scan time exactly as
 * FrameAligner/FrameWarper.cpp:252-267 computes it), so a frame aligned with D_true reproduces the
 * reference up to noise. Random parameters (blob positions, widths, amplitudes, D_true, Poisson
 * noise) are drawn by the Python caller; this file only evaluates the deterministic sums.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>

typedef struct {
  int nz, ny, nx;
  int n_blobs;
  const double* blobs; /* n_blobs x 7: mu_x, mu_y, mu_z, sigma_x, sigma_y, sigma_z, amplitude */
  double background;
  double scale;
  /* displacement model (D == NULL renders the undisplaced reference) */
  const double* D; /* nD x 3 */
  int nD;
  double t_pixel, t_line, t_plane, t_stack; /* processed scan durations */
  int bidirectional;
  float* out;
  int row0, row1; /* rows [row0, row1) of the nz*ny rows */
} synth_job;

static void* render_rows(void* arg) {
  synth_job* j = (synth_job*)arg;
  const int nx = j->nx;
  double* dx = (double*)malloc(sizeof(double) * (size_t)nx);
  double* dy = (double*)malloc(sizeof(double) * (size_t)nx);
  double* dz = (double*)malloc(sizeof(double) * (size_t)nx);
  double* acc = (double*)malloc(sizeof(double) * (size_t)nx);
  for (int row = j->row0; row < j->row1; row++) {
    int z = row / j->ny, y = row % j->ny;
    double dmin[3] = {0, 0, 0}, dmax[3] = {0, 0, 0};
    for (int x = 0; x < nx; x++) {
      double d[3] = {0, 0, 0};
      if (j->D) {
        int xs = (j->bidirectional && (y % 2 == 1)) ? nx - 1 - x : x;
        double t = z * j->t_plane + y * j->t_line + xs * j->t_pixel;
        double q = t / j->t_stack * (j->nD - 1);
        int i = (int)floor(q);
        if (i > j->nD - 2) i = j->nD - 2;
        if (i < 0) i = 0;
        double f = q - i;
        for (int c = 0; c < 3; c++) d[c] = f * j->D[3 * (i + 1) + c] + (1 - f) * j->D[3 * i + c];
      }
      dx[x] = d[0];
      dy[x] = d[1];
      dz[x] = d[2];
      for (int c = 0; c < 3; c++) {
        if (x == 0 || d[c] < dmin[c]) dmin[c] = d[c];
        if (x == 0 || d[c] > dmax[c]) dmax[c] = d[c];
      }
      acc[x] = j->background;
    }
    for (int b = 0; b < j->n_blobs; b++) {
      const double* p = j->blobs + 7 * b;
      double mx = p[0], my = p[1], mz = p[2], sx = p[3], sy = p[4], sz = p[5], a = p[6];
      /* sample position is (x - dx, y - dy, z - dz): skip blobs more than 6 sigma away */
      double ylo = y - dmax[1], yhi = y - dmin[1];
      double ry = (my < ylo) ? ylo - my : (my > yhi ? my - yhi : 0.0);
      if (ry > 6 * sy) continue;
      if (j->nz > 1) {
        double zlo = z - dmax[2], zhi = z - dmin[2];
        double rz = (mz < zlo) ? zlo - mz : (mz > zhi ? mz - zhi : 0.0);
        if (rz > 6 * sz) continue;
      }
      int xa = (int)floor(mx - 6 * sx + dmin[0]) - 1, xb = (int)ceil(mx + 6 * sx + dmax[0]) + 1;
      if (xa < 0) xa = 0;
      if (xb > nx - 1) xb = nx - 1;
      for (int x = xa; x <= xb; x++) {
        double u = (x - dx[x] - mx) / sx, v = (y - dy[x] - my) / sy;
        double e = u * u + v * v;
        if (j->nz > 1) {
          double w = (z - dz[x] - mz) / sz;
          e += w * w;
        }
        acc[x] += a * exp(-0.5 * e);
      }
    }
    float* o = j->out + (size_t)row * nx;
    for (int x = 0; x < nx; x++) o[x] = (float)(acc[x] * j->scale);
  }
  free(dx);
  free(dy);
  free(dz);
  free(acc);
  return NULL;
}

/* Renders one volume (see the file comment). scan = {t_pixel, t_line, t_plane, t_stack}. */
int fa_synth_render(int nz, int ny, int nx, const double* blobs, int n_blobs, double background, double scale,
                    const double* D, int nD, const double* scan, int bidirectional, int n_threads, float* out) {
  if (n_threads < 1) n_threads = 1;
  int rows = nz * ny;
  if (n_threads > rows) n_threads = rows;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)n_threads);
  synth_job* jobs = (synth_job*)malloc(sizeof(synth_job) * (size_t)n_threads);
  for (int t = 0; t < n_threads; t++) {
    synth_job j;
    j.nz = nz;
    j.ny = ny;
    j.nx = nx;
    j.n_blobs = n_blobs;
    j.blobs = blobs;
    j.background = background;
    j.scale = scale;
    j.D = D;
    j.nD = nD;
    j.t_pixel = scan ? scan[0] : 0;
    j.t_line = scan ? scan[1] : 0;
    j.t_plane = scan ? scan[2] : 0;
    j.t_stack = scan ? scan[3] : 1;
    j.bidirectional = bidirectional;
    j.out = out;
    j.row0 = (int)((long)rows * t / n_threads);
    j.row1 = (int)((long)rows * (t + 1) / n_threads);
    jobs[t] = j;
    pthread_create(&th[t], NULL, render_rows, &jobs[t]);
  }
  for (int t = 0; t < n_threads; t++) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
  return 0;
}
