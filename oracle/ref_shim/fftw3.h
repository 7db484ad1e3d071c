// Stand-in for the four FFTW3 calls that frame-aligner's VolumePhaseCorrelator.cpp makes
// (TEST INFRASTRUCTURE ONLY). The transforms follow FFTW's documented definitions: an
// unnormalised forward r2c DFT (exponent sign -1) of a row-major rank-d real array into
// n0 x ... x (n_{d-1}/2+1) complex values, and the unnormalised inverse c2r (exponent sign
// +1) that assumes Hermitian input. Computed by direct per-axis DFTs in double: slow, exact
// to rounding, and only meant for the small volumes the parity tests use.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct fa_shim_fftw_plan_s* fftw_plan;
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_r2c(int rank, const int* n, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r(int rank, const int* n, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
