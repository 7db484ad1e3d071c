// Direct-DFT implementation of the FFTW stand-in declared in fftw3.h (test infrastructure only).
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <vector>

typedef std::complex<double> cplx;

struct fa_shim_fftw_plan_s {
  bool r2c;
  std::vector<int> n;
  double* real;
  cplx* spec;
};

static void dft_line(cplx* data, long n, long stride, int sign, std::vector<cplx>& tmp) {
  // out[k] = sum_j in[j] * exp(sign * 2 pi i j k / n), twiddles tabulated per call
  const double two_pi = 6.283185307179586476925286766559;
  std::vector<cplx> tw((size_t)n);
  for (long m = 0; m < n; m++) {
    double a = sign * two_pi * (double)m / (double)n;
    tw[(size_t)m] = cplx(std::cos(a), std::sin(a));
  }
  tmp.assign((size_t)n, cplx(0, 0));
  for (long k = 0; k < n; k++) {
    cplx acc(0, 0);
    long m = 0;
    for (long j = 0; j < n; j++) {
      acc += data[j * stride] * tw[(size_t)m];
      m += k;
      if (m >= n) m -= n;
    }
    tmp[(size_t)k] = acc;
  }
  for (long k = 0; k < n; k++) data[k * stride] = tmp[(size_t)k];
}

extern "C" fftw_plan fftw_plan_dft_r2c(int rank, const int* n, double* in, fftw_complex* out, unsigned) {
  fa_shim_fftw_plan_s* p = new fa_shim_fftw_plan_s;
  p->r2c = true;
  p->n.assign(n, n + rank);
  p->real = in;
  p->spec = reinterpret_cast<cplx*>(out);
  return p;
}

extern "C" fftw_plan fftw_plan_dft_c2r(int rank, const int* n, fftw_complex* in, double* out, unsigned) {
  fa_shim_fftw_plan_s* p = new fa_shim_fftw_plan_s;
  p->r2c = false;
  p->n.assign(n, n + rank);
  p->real = out;
  p->spec = reinterpret_cast<cplx*>(in);
  return p;
}

extern "C" void fftw_destroy_plan(fftw_plan p) { delete p; }

extern "C" void fftw_execute(const fftw_plan p) {
  const int rank = (int)p->n.size();
  const long nx = p->n[rank - 1];
  const long nh = nx / 2 + 1;
  long outer = 1;
  for (int d = 0; d < rank - 1; d++) outer *= p->n[d];
  std::vector<cplx> tmp, line((size_t)nx);
  if (p->r2c) {
    // last axis: real -> half spectrum
    for (long o = 0; o < outer; o++) {
      for (long j = 0; j < nx; j++) line[(size_t)j] = cplx(p->real[o * nx + j], 0.0);
      dft_line(line.data(), nx, 1, -1, tmp);
      for (long k = 0; k < nh; k++) p->spec[o * nh + k] = line[(size_t)k];
    }
    // remaining axes, complex, from the second-to-last outward
    long inner = nh;
    for (int d = rank - 2; d >= 0; d--) {
      long len = p->n[d];
      long block = inner * len;
      long nblocks = (outer * nh) / block;
      for (long b = 0; b < nblocks; b++)
        for (long i = 0; i < inner; i++) dft_line(p->spec + b * block + i, len, inner, -1, tmp);
      inner = block;
    }
  } else {
    std::vector<cplx> spec(p->spec, p->spec + outer * nh);
    long inner = nh;
    for (int d = rank - 2; d >= 0; d--) {
      long len = p->n[d];
      long block = inner * len;
      long nblocks = (outer * nh) / block;
      for (long b = 0; b < nblocks; b++)
        for (long i = 0; i < inner; i++) dft_line(spec.data() + b * block + i, len, inner, +1, tmp);
      inner = block;
    }
    // last axis: Hermitian half spectrum -> real
    const double two_pi = 6.283185307179586476925286766559;
    for (long o = 0; o < outer; o++) {
      const cplx* s = spec.data() + o * nh;
      for (long x = 0; x < nx; x++) {
        double acc = s[0].real();
        long kmax = (nx % 2 == 0) ? nx / 2 - 1 : (nx - 1) / 2;
        for (long k = 1; k <= kmax; k++) {
          long m = (k * x) % nx;
          double a = two_pi * (double)m / (double)nx;
          acc += 2.0 * (s[k].real() * std::cos(a) - s[k].imag() * std::sin(a));
        }
        if (nx % 2 == 0) acc += s[nx / 2].real() * ((x % 2) ? -1.0 : 1.0);
        p->real[o * nx + x] = acc;
      }
    }
  }
}
