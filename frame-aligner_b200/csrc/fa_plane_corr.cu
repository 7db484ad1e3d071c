// fa_plane_corr.cu -- the phase correlator's FP64 transforms as three fused passes over a batch of
// frames (power-of-two volumes with nz <= 16, 8 <= ny <= 2048, 16 <= nx <= 4096 and an (nz, ny) plane of at most
// 8192 points), instead of window + cuFFT D2Z (three axis passes) + normalise + cuFFT Z2D (three
// axis passes) + argmax. The computed quantity is the reference's
// (VolumePhaseCorrelator.cpp:57-103): the windowed frame's 3-D DFT times the conjugate of the
// reference's, divided by its modulus + DBL_MIN, transformed back, first maximum.
//
//   plane_rows_fwd_kernel   window (the reference's separately rounded FP64 products) and the real
//                           DFT along x of G rows, as an nx/2-point complex DFT of the packed row
//                           (even samples real, odd samples imaginary) and the split into the
//                           nx/2 + 1 half-spectrum bins; written as planes spec[kx][z][y]
//   plane_yz_kernel         per kx plane (nz x ny, on chip): DFT along y, DFT along z, times the
//                           reference's conjugate spectrum, normalised, inverse along z and y; or,
//                           for the reference itself, the conjugate of the forward plane
//   plane_rows_inv_argmax   the inverse real DFT along x of G rows (the half-spectrum folded into
//                           an nx/2-point complex inverse DFT) and the first maximum of the real
//                           surface in flat (z, y, x) order, per CTA; then phase_argmax_final
//
// Planes too large for one CTA (nz * ny > 8192 or nz > 16, power-of-two nz >= 8) split the middle
// pass in three: plane_y_kernel (DFT of y lines, in place), plane_z_kernel (per kx plane and block of
// y columns: DFT along z, cross-power with the reference, inverse DFT along z) and plane_y_kernel
// again (inverse), so every volume of these dimensions stays off cuFFT.
//
// DFTs along a row are Stockham radix-8/4/2 stages in shared memory (line l, element i at
// l * (L + 1) + (i ^ ((i >> 3) & 7)): conflict-free for the stride-R writes of every stage and for
// column reads across lines); the z DFT (<= 16 points) runs in registers, one (kx, y) column per
// thread. Twiddles W_L^m = exp(-2 pi i m / L) come from tables rounded from long double on the host.
// The inverse transforms are unnormalised (a positive scale does not move the maximum).
#include <cooperative_groups.h>
#include <float.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "fa_kernels.cuh"

namespace fa {

namespace {

__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
  return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}
// a * w (forward) or a * conj(w) (inverse)
template <bool INV>
__device__ __forceinline__ double2 cmul_tw(double2 a, double2 w) {
  return INV ? make_double2(fma(a.x, w.x, a.y * w.y), fma(a.y, w.x, -a.x * w.y)) : cmul(a, w);
}
// a * (-i) (forward) or a * (+i) (inverse)
template <bool INV>
__device__ __forceinline__ double2 rot(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

constexpr double kS2 = 0.70710678118654752440;   // cos(pi/4)
constexpr double kC8 = 0.92387953251128675613;   // cos(pi/8)
constexpr double kS8 = 0.38268343236508977173;   // sin(pi/8)

template <bool INV>
__device__ __forceinline__ void dft2(double2& a0, double2& a1) {
  const double2 t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2& a0, double2& a1, double2& a2, double2& a3) {
  const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = rot<INV>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

// W_8^1 and W_8^3 (forward) or their conjugates (inverse)
template <bool INV>
__device__ __forceinline__ double2 w8_1(double2 a) {
  return INV ? make_double2(kS2 * (a.x - a.y), kS2 * (a.x + a.y)) : make_double2(kS2 * (a.x + a.y), kS2 * (a.y - a.x));
}
template <bool INV>
__device__ __forceinline__ double2 w8_3(double2 a) {
  return INV ? make_double2(-kS2 * (a.x + a.y), kS2 * (a.x - a.y))
             : make_double2(kS2 * (a.y - a.x), -kS2 * (a.x + a.y));
}

template <bool INV>
__device__ __forceinline__ void dft8(double2* a) {
  double2 e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
  double2 o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  o1 = w8_1<INV>(o1);
  o2 = rot<INV>(o2);
  o3 = w8_3<INV>(o3);
  a[0] = cadd(e0, o0);
  a[4] = csub(e0, o0);
  a[1] = cadd(e1, o1);
  a[5] = csub(e1, o1);
  a[2] = cadd(e2, o2);
  a[6] = csub(e2, o2);
  a[3] = cadd(e3, o3);
  a[7] = csub(e3, o3);
}

// W_16^e (forward) for the exponents a 4 x 4 split needs
__device__ __forceinline__ double2 w16(int e) {
  switch (e) {
    case 1: return make_double2(kC8, -kS8);
    case 2: return make_double2(kS2, -kS2);
    case 3: return make_double2(kS8, -kC8);
    case 4: return make_double2(0.0, -1.0);
    case 6: return make_double2(-kS2, -kS2);
    case 9: return make_double2(-kC8, kS8);
    default: return make_double2(1.0, 0.0);
  }
}

// 16 points as 4 x 4: X[k1 + 4 k2] = sum_n2 W_4^(n2 k2) W_16^(n2 k1) sum_n1 W_4^(n1 k1) a[4 n1 + n2]
template <bool INV>
__device__ __forceinline__ void dft16(double2* a) {
  double2 b[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
    b[n2][0] = a[n2];
    b[n2][1] = a[n2 + 4];
    b[n2][2] = a[n2 + 8];
    b[n2][3] = a[n2 + 12];
    dft4<INV>(b[n2][0], b[n2][1], b[n2][2], b[n2][3]);
#pragma unroll
    for (int k1 = 1; k1 < 4; k1++)
      if (n2 > 0) b[n2][k1] = cmul_tw<INV>(b[n2][k1], w16(n2 * k1));
  }
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    double2 c0 = b[0][k1], c1 = b[1][k1], c2 = b[2][k1], c3 = b[3][k1];
    dft4<INV>(c0, c1, c2, c3);
    a[k1] = c0;
    a[k1 + 4] = c1;
    a[k1 + 8] = c2;
    a[k1 + 12] = c3;
  }
}

// In-register DFT of R points (natural order in and out).
template <int R, bool INV>
__device__ __forceinline__ void dft(double2* a) {
  if constexpr (R == 2) dft2<INV>(a[0], a[1]);
  else if constexpr (R == 4) dft4<INV>(a[0], a[1], a[2], a[3]);
  else if constexpr (R == 8) dft8<INV>(a);
  else if constexpr (R == 16) dft16<INV>(a);
}

// One Stockham radix-R stage over `lines` lines of L = 2^LOG2L points. Butterfly j of line l reads
// x[j + r L/R] (load(l, i)), twiddles them by W_(Ns R)^(r k) with k = j mod Ns, takes the R-point
// DFT and writes y[((j - k) R + k) + r Ns] (store(l, i, v)). Every thread first loads all of its
// butterflies (NB at most), so global loads are in flight together. In place in shared memory the
// block synchronises between the reads and the writes (SYNC_MID) and after the writes (SYNC_END).
// The stage's twiddles sit at tw[OFF + (r - 1) Ns + k] in shared memory (contiguous in k, so the
// lanes of a warp read distinct banks). The sizes are template constants.
template <int R, int NB, bool INV, int LOG2L, int LOG2NS, int OFF, int T, bool SYNC_MID, bool SYNC_END, class Load,
          class Store>
__device__ __forceinline__ void stockham_stage(int lines, const double2* tw, Load load, Store store) {
  constexpr int log2R = R == 8 ? 3 : (R == 4 ? 2 : 1);
  constexpr int log2q = LOG2L - log2R;
  constexpr int q = 1 << log2q;
  constexpr int Ns = 1 << LOG2NS;
  const int nb = lines << log2q;
  double2 a[NB][R];
#pragma unroll
  for (int u = 0; u < NB; u++) {
    const int b = threadIdx.x + u * T;
    if (b < nb) {
      const int l = b >> log2q, j = b & (q - 1);
#pragma unroll
      for (int r = 0; r < R; r++) a[u][r] = load(l, j + (r << log2q));
    }
  }
#pragma unroll
  for (int u = 0; u < NB; u++) {
    const int b = threadIdx.x + u * T;
    if (b < nb) {
      if (Ns > 1) {
        const int k = b & (Ns - 1);  // j mod Ns (Ns <= q)
#pragma unroll
        for (int r = 1; r < R; r++) a[u][r] = cmul_tw<INV>(a[u][r], tw[OFF + (r - 1) * Ns + k]);
      }
      dft<R, INV>(a[u]);
    }
  }
  if (SYNC_MID) __syncthreads();
#pragma unroll
  for (int u = 0; u < NB; u++) {
    const int b = threadIdx.x + u * T;
    if (b < nb) {
      const int l = b >> log2q, j = b & (q - 1);
      const int k = j & (Ns - 1);
      const int o = ((j - k) << log2R) + k;
#pragma unroll
      for (int r = 0; r < R; r++) store(l, o + (r << LOG2NS), a[u][r]);
    }
  }
  if (SYNC_END) __syncthreads();
}

// Radix-8 stages, then one radix-4 or radix-2 stage, over lines in shared memory (line stride
// L + 1, element i at i ^ ((i >> 3) & 7)); OFF advances by the (R - 1) Ns twiddles of every stage
// after the first (stage_table on the host lays them out in the same order). The first stage reads
// through `first` unless FIRST_SMEM, the last writes through `last` unless LAST_SMEM; a stage that
// writes shared memory ends with a barrier.
template <bool INV, int EPT, int LOG2L, int T, bool FIRST_SMEM, bool LAST_SMEM, int LOG2NS = 0, int OFF = 0,
          class First, class Last>
__device__ __forceinline__ void fft_rows_t(double2* sm, int lines, const double2* tw, First first, Last last) {
  constexpr int S = (1 << LOG2L) + 1;
  constexpr int rem = LOG2L - LOG2NS;
  constexpr int log2R = rem >= 3 ? 3 : rem;
  constexpr int R = 1 << log2R;
  constexpr bool is_first = LOG2NS == 0, is_last = LOG2NS + log2R == LOG2L;
  constexpr bool in_smem = !is_first || FIRST_SMEM, out_smem = !is_last || LAST_SMEM;
  auto load = [&](int l, int i) -> double2 {
    if constexpr (in_smem) return sm[l * S + swz(i)];
    else return first(l, i);
  };
  auto store = [&](int l, int i, double2 v) {
    if constexpr (out_smem) sm[l * S + swz(i)] = v;
    else last(l, i, v);
  };
  stockham_stage<R, EPT / R, INV, LOG2L, LOG2NS, OFF, T, in_smem && out_smem, out_smem>(lines, tw, load, store);
  if constexpr (!is_last)
    fft_rows_t<INV, EPT, LOG2L, T, FIRST_SMEM, LAST_SMEM, LOG2NS + log2R, OFF + (LOG2NS > 0 ? (R - 1) << LOG2NS : 0)>(
        sm, lines, tw, first, last);
}

// DFT of every line of 2^log2L points (3 <= log2L <= 11) by a block of T threads, with the stage
// twiddles of stage_table(2^log2L) at tw. lines * 2^log2L <= EPT * T. The caller synchronises
// before a first stage that reads shared memory.
template <bool INV, int EPT, int T, bool FIRST_SMEM, bool LAST_SMEM, class First, class Last>
__device__ __forceinline__ void fft_rows(double2* sm, int lines, int log2L, const double2* tw, First first,
                                         Last last) {
  switch (log2L) {
    case 3: fft_rows_t<INV, EPT, 3, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 4: fft_rows_t<INV, EPT, 4, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 5: fft_rows_t<INV, EPT, 5, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 6: fft_rows_t<INV, EPT, 6, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 7: fft_rows_t<INV, EPT, 7, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 8: fft_rows_t<INV, EPT, 8, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 9: fft_rows_t<INV, EPT, 9, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 10: fft_rows_t<INV, EPT, 10, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    case 11: fft_rows_t<INV, EPT, 11, T, FIRST_SMEM, LAST_SMEM>(sm, lines, tw, first, last); break;
    default: break;
  }
}

}  // namespace

// Neither: the first stage reads shared memory / the last writes it.
struct NoIo {
  __device__ double2 operator()(int, int) const { return make_double2(0.0, 0.0); }
  __device__ void operator()(int, int, double2) const {}
};

namespace {

constexpr int kRowThreads = 256;
constexpr int kRowEPT = 8;      // G * nx/2 <= 2048 points per row CTA
constexpr int kPlaneThreads = 512;
constexpr int kPlaneEPT = 16;   // PP * nz * ny <= 8192 points per plane CTA

// Global -> shared staging in 16-byte chunks: chunk i is read from src_of(i) and written to
// dst_of(i), with K loads of each thread in flight before the first store. Published by the
// caller's next barrier.
template <int K, class SrcOf, class DstOf>
__device__ __forceinline__ void stage16(int n, SrcOf src_of, DstOf dst_of) {
  for (int base = 0; base < n; base += K * (int)blockDim.x) {
    uint4 v[K];
#pragma unroll
    for (int u = 0; u < K; u++) {
      const int i = base + (int)threadIdx.x + u * (int)blockDim.x;
      if (i < n) v[u] = __ldg(src_of(i));
    }
#pragma unroll
    for (int u = 0; u < K; u++) {
      const int i = base + (int)threadIdx.x + u * (int)blockDim.x;
      if (i < n) *dst_of(i) = v[u];
    }
  }
}

// Row-pass shared memory: G lines of S = nx/2 + 1 points, then the nx twiddle slots (double2).
__host__ __device__ inline size_t rows_smem_bytes(const PlaneDims& d) {
  const size_t G = (size_t)1 << d.log2G;
  return (G * ((d.nx >> 1) + 1) + d.nx) * 16;
}

// SLOT: -1, or the FrameKind of the slots written from the same loads (SlotOut).
template <bool U16, int SLOT>
__global__ void __launch_bounds__(kRowThreads) plane_rows_fwd_kernel(const void* const* __restrict__ vols,
                                                                     const double* __restrict__ wy,
                                                                     const double* __restrict__ wx,
                                                                     const double2* __restrict__ tw_x, PlaneDims d,
                                                                     double2* __restrict__ spec, SlotOut slot) {
  extern __shared__ double2 sm[];
  const int M = d.nx >> 1, S = M + 1, G = 1 << d.log2G;
  double2* tws = sm + G * S;
  const int r0 = blockIdx.x << d.log2G;
  const void* vol = vols[blockIdx.y];
  void* const slot_base = SLOT >= 0 ? const_cast<void*>(slot.ptrs[blockIdx.y]) : nullptr;
  // the twiddles (published by the first stage's closing barrier; the first stage needs none)
  stage16<4>(
      d.n_twx, [&](int i) { return reinterpret_cast<const uint4*>(tw_x) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  // the first stage reads the frame: point m of row g is (v[2m], v[2m + 1]), windowed as
  // (double)v * ((1 * wy[y]) * wx[x]) with each product rounded (VolumePhaseCorrelator.cpp:62-63)
  auto first = [&](int g, int m) -> double2 {
    const int r = r0 + g;
    const long long off = (long long)r * d.nx + 2 * m;
    float v0, v1;
    unsigned q0 = 0, q1 = 0;
    if (U16) {
      const ushort2 q = __ldg(reinterpret_cast<const ushort2*>(static_cast<const unsigned short*>(vol) + off));
      v0 = (float)q.x;
      v1 = (float)q.y;
      q0 = q.x;
      q1 = q.y;
    } else {
      const float2 f = __ldg(reinterpret_cast<const float2*>(static_cast<const float*>(vol) + off));
      v0 = f.x;
      v1 = f.y;
    }
    if constexpr (SLOT >= 0) {
      // the slot conversion of these two values (count + 1 saturated, or value + 1 rounded to the
      // slot's type), at (z, y, 2m) of this frame's slot
      const long long so = (long long)(r >> d.log2ny) * slot.plane + (long long)(r & (d.ny - 1)) * slot.pitch + 2 * m;
      void* dst = slot_base;
      if constexpr (SLOT == kFrameRawU16) {
        const unsigned lo = min(q0 + 1u, 65535u), hi = min(q1 + 1u, 65535u);
        *reinterpret_cast<unsigned*>(static_cast<unsigned short*>(dst) + so) = lo | (hi << 16);
      } else if constexpr (SLOT == kFrameF16) {
        *reinterpret_cast<__half2*>(static_cast<__half*>(dst) + so) =
            __halves2half2(__float2half_rn(v0 + 1.0f), __float2half_rn(v1 + 1.0f));
      } else {
        *reinterpret_cast<float2*>(static_cast<float*>(dst) + so) = make_float2(v0 + 1.0f, v1 + 1.0f);
      }
    }
    const double wrow = __dmul_rn(1.0, __ldg(wy + (r & (d.ny - 1))));
    const double2 w = __ldg(reinterpret_cast<const double2*>(wx) + m);
    return make_double2(__dmul_rn((double)v0, __dmul_rn(wrow, w.x)), __dmul_rn((double)v1, __dmul_rn(wrow, w.y)));
  };
  fft_rows<false, kRowEPT, kRowThreads, false, true>(sm, G, d.log2M, tws, first, NoIo{});
  // X[k] = (Z[k] + conj Z[M-k]) / 2 - i W_nx^k (Z[k] - conj Z[M-k]) / 2, k = 0..M, to plane k
  double2* out = spec + (long long)blockIdx.y * d.n_complex;
  for (int idx = threadIdx.x; idx < ((M + 1) << d.log2G); idx += blockDim.x) {
    const int k = idx >> d.log2G, g = idx & (G - 1);
    const double2 zk = sm[g * S + swz(k & (M - 1))];
    const double2 zm = sm[g * S + swz((M - k) & (M - 1))];
    const double2 e = make_double2(zk.x + zm.x, zk.y - zm.y);
    const double2 wd = cmul(make_double2(zk.x - zm.x, zk.y + zm.y), tws[d.tw_x_post + k]);
    out[(long long)k * d.rows + r0 + g] = make_double2(0.5 * (e.x + wd.y), 0.5 * (e.y - wd.x));
  }
}

// z / |z| of z = a * b (VolumePhaseCorrelator.cpp:70-75 divides by |z| + DBL_MIN, which only
// matters for z = 0: zero stays zero here too). One reciprocal square root instead of a hypot and
// two divisions: the result differs from the reference's rounding by a few ulp, well inside the
// rounding differences of the transforms themselves.
__device__ __forceinline__ double2 cross_power(double2 a, double2 b) {
  const double re = fma(a.x, b.x, -a.y * b.y);
  const double im = fma(a.x, b.y, a.y * b.x);
  const double q = fma(re, re, im * im);
  const double r = q > 0.0 ? rsqrt(q) : 0.0;
  return make_double2(re * r, im * r);
}

// Planes p0 .. p0 + PP - 1 of the batch's plane array (frame-major, nx/2 + 1 planes per frame).
// REF: out = conj(forward DFT over (z, y)); otherwise out = inverse(normalised forward * ref_conj).
// Shared memory: PP * NZ lines of S = ny + 1 points, then the ny twiddles W_ny^m.
template <int NZ, bool REF>
__global__ void __launch_bounds__(kPlaneThreads, 1) plane_yz_kernel(const double2* in, double2* out,
                                                                    const double2* __restrict__ ref_conj,
                                                                    const double2* __restrict__ tw_y, PlaneDims d,
                                                                    long long n_planes) {
  extern __shared__ double2 sm[];
  const int ny = d.ny, S = ny + 1;
  const int plane = NZ * ny;
  const long long p0 = (long long)blockIdx.x * d.PP;
  const int pp = (int)min((long long)d.PP, n_planes - p0);
  const int E = pp * plane;
  double2* tws = sm + d.PP * NZ * S;
  const double2* src = in + p0 * plane;
  stage16<4>(
      d.n_twy, [&](int i) { return reinterpret_cast<const uint4*>(tw_y) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  // the first stage reads the planes (in may be out: each CTA reads its own planes before it
  // writes them)
  auto first = [&](int l, int i) -> double2 { return src[l * ny + i]; };
  fft_rows<false, kPlaneEPT, kPlaneThreads, false, true>(sm, pp * NZ, d.log2ny, tws, first, NoIo{});
  const int M1 = (d.nx >> 1) + 1;
  for (int c = threadIdx.x; c < pp * ny; c += blockDim.x) {
    const int p = c >> d.log2ny, y = c & (ny - 1);
    double2 a[NZ];
    double2* col = sm + (p * NZ) * S + swz(y);
    if (REF) {
#pragma unroll
      for (int z = 0; z < NZ; z++) a[z] = col[z * S];
      dft<NZ, false>(a);
#pragma unroll
      for (int z = 0; z < NZ; z++) a[z].y = -a[z].y;
    } else {
      // the reference's spectrum in two halves: the first half's loads overlap the forward DFT
      constexpr int kH = (NZ + 1) / 2;
      const int k = (int)((p0 + p) % M1);
      const double2* rc = ref_conj + (long long)k * plane + y;
      double2 b[kH];
#pragma unroll
      for (int z = 0; z < kH; z++) b[z] = __ldg(rc + z * ny);
#pragma unroll
      for (int z = 0; z < NZ; z++) a[z] = col[z * S];
      dft<NZ, false>(a);
#pragma unroll
      for (int z = 0; z < kH; z++) a[z] = cross_power(a[z], b[z]);
#pragma unroll
      for (int z = kH; z < NZ; z++) b[z - kH] = __ldg(rc + z * ny);
#pragma unroll
      for (int z = kH; z < NZ; z++) a[z] = cross_power(a[z], b[z - kH]);
      dft<NZ, true>(a);
    }
#pragma unroll
    for (int z = 0; z < NZ; z++) col[z * S] = a[z];
  }
  __syncthreads();
  double2* dst = out + p0 * plane;
  if (!REF) {
    // the last inverse stage writes the planes
    auto last = [&](int l, int i, double2 v) { dst[l * ny + i] = v; };
    fft_rows<true, kPlaneEPT, kPlaneThreads, true, false>(sm, pp * NZ, d.log2ny, tws, NoIo{}, last);
  } else {
#pragma unroll
    for (int u = 0; u < kPlaneEPT; u++) {
      const int idx = threadIdx.x + u * kPlaneThreads;
      if (idx < E) dst[idx] = sm[(idx >> d.log2ny) * S + swz(idx & (ny - 1))];
    }
  }
}

// The same pass for planes of exactly 8192 points (nz in {4, 8, 16}), one plane per pair of CTAs
// (a 2-CTA cluster), so that each CTA needs half the shared memory and two fit per SM. CTA r holds
// the z lines [r NZ/2, (r + 1) NZ/2) and runs their y DFTs; after a cluster barrier it takes the z
// columns y in [r ny/2, (r + 1) ny/2), reading the other CTA's half of each column from that CTA's
// shared memory (distributed shared memory) and writing it back there; after a second barrier each
// CTA runs its own lines' inverse y DFTs. The arithmetic is plane_yz_kernel's, in the same order.
constexpr int kPairThreads = 256;
constexpr int kPairEPT = 16;  // NZ/2 * ny = 4096 points per CTA

template <int NZ, bool REF>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kPairThreads, 2)
    plane_yz_pair_kernel(const double2* in, double2* out, const double2* __restrict__ ref_conj,
                         const double2* __restrict__ tw_y, PlaneDims d) {
  namespace cg = cooperative_groups;
  extern __shared__ double2 sm[];
  constexpr int H = NZ / 2;  // z lines per CTA
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int ny = d.ny, S = ny + 1;
  const int plane = NZ * ny;
  const long long p = blockIdx.x >> 1;
  double2* tws = sm + H * S;
  stage16<4>(
      d.n_twy, [&](int i) { return reinterpret_cast<const uint4*>(tw_y) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  // this CTA's lines (in may be out: each CTA reads its own lines before it writes them)
  const double2* src = in + p * plane + (long long)r * H * ny;
  auto first = [&](int l, int i) -> double2 { return src[l * ny + i]; };
  fft_rows<false, kPairEPT, kPairThreads, false, true>(sm, H, d.log2ny, tws, first, NoIo{});
  cluster.sync();  // both halves transformed along y, visible to the other CTA
  // lines 0 .. H-1 live in CTA 0, lines H .. NZ-1 in CTA 1
  double2* lo = r == 0 ? sm : cluster.map_shared_rank(sm, 0);
  double2* hi = r == 1 ? sm : cluster.map_shared_rank(sm, 1);
  const int M1 = (d.nx >> 1) + 1;
  const int half = ny >> 1;
  for (int c = threadIdx.x; c < half; c += blockDim.x) {
    const int y = r * half + c;
    const int o = swz(y);
    double2 a[NZ];
#pragma unroll
    for (int z = 0; z < H; z++) {
      a[z] = lo[z * S + o];
      a[H + z] = hi[z * S + o];
    }
    if (REF) {
      dft<NZ, false>(a);
#pragma unroll
      for (int z = 0; z < NZ; z++) a[z].y = -a[z].y;
    } else {
      constexpr int kH = (NZ + 1) / 2;
      const int k = (int)(p % M1);
      const double2* rc = ref_conj + (long long)k * plane + y;
      double2 b[kH];
#pragma unroll
      for (int z = 0; z < kH; z++) b[z] = __ldg(rc + z * ny);
      dft<NZ, false>(a);
#pragma unroll
      for (int z = 0; z < kH; z++) a[z] = cross_power(a[z], b[z]);
#pragma unroll
      for (int z = kH; z < NZ; z++) b[z - kH] = __ldg(rc + z * ny);
#pragma unroll
      for (int z = kH; z < NZ; z++) a[z] = cross_power(a[z], b[z - kH]);
      dft<NZ, true>(a);
    }
#pragma unroll
    for (int z = 0; z < H; z++) {
      lo[z * S + o] = a[z];
      hi[z * S + o] = a[H + z];
    }
  }
  cluster.sync();  // every column written back; no shared-memory access crosses CTAs after this
  double2* dst = out + p * plane + (long long)r * H * ny;
  if (!REF) {
    auto last = [&](int l, int i, double2 v) { dst[l * ny + i] = v; };
    fft_rows<true, kPairEPT, kPairThreads, true, false>(sm, H, d.log2ny, tws, NoIo{}, last);
  } else {
    const int E = H * ny;
#pragma unroll
    for (int u = 0; u < kPairEPT; u++) {
      const int idx = threadIdx.x + u * kPairThreads;
      if (idx < E) dst[idx] = sm[(idx >> d.log2ny) * S + swz(idx & (ny - 1))];
    }
  }
}

// Split (z, y) pass. Lines of ny points along y, in place in the batch's plane array (line l = plane
// p, plane z at offset l * ny of spec[kx][z][y]), d.LY lines per CTA; the first stage reads global
// memory and the last writes it (ny >= 16: at least two stages, so a CTA reads all its lines before
// it writes any). Shared memory: LY lines of S = ny + 1 points, then the ny twiddle slots.
template <bool INV>
__global__ void __launch_bounds__(kPlaneThreads, 1) plane_y_kernel(double2* spec, const double2* __restrict__ tw_y,
                                                                   PlaneDims d, long long n_lines) {
  extern __shared__ double2 sm[];
  const int ny = d.ny, S = ny + 1;
  const long long l0 = (long long)blockIdx.x * d.LY;
  const int nl = (int)min((long long)d.LY, n_lines - l0);
  double2* tws = sm + d.LY * S;
  double2* base = spec + l0 * ny;
  stage16<4>(
      d.n_twy, [&](int i) { return reinterpret_cast<const uint4*>(tw_y) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  auto first = [&](int l, int i) -> double2 { return base[(long long)l * ny + i]; };
  auto last = [&](int l, int i, double2 v) { base[(long long)l * ny + i] = v; };
  fft_rows<INV, kPlaneEPT, kPlaneThreads, false, false>(sm, nl, d.log2ny, tws, first, last);
}

// Split (z, y) pass, z columns: CTA = plane p of the batch x YB = 2^log2YB consecutive y. The
// columns are staged with loads along y (line yy = column y0 + yy, element z), transformed along z
// in shared memory, then multiplied by the reference's conjugate spectrum and normalised (or, for
// the reference, conjugated and written to ref_out), transformed back and stored along y.
// Shared memory: YB lines of S = nz + 1 points, then the nz twiddle slots.
template <bool REF>
__global__ void __launch_bounds__(kPlaneThreads, 1) plane_z_kernel(double2* spec, double2* ref_out,
                                                                   const double2* __restrict__ ref_conj,
                                                                   const double2* __restrict__ tw_z, PlaneDims d) {
  extern __shared__ double2 sm[];
  const int nz = d.nz, ny = d.ny, S = nz + 1, YB = 1 << d.log2YB;
  const int yblocks = ny >> d.log2YB;
  const long long p = blockIdx.x / yblocks;
  const int y0 = (int)(blockIdx.x - p * yblocks) << d.log2YB;
  const long long plane = (long long)nz * ny;
  double2* col = spec + p * plane + y0;
  double2* tws = sm + YB * S;
  const int E = nz << d.log2YB;
  stage16<4>(
      d.n_twz, [&](int i) { return reinterpret_cast<const uint4*>(tw_z) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int z = idx >> d.log2YB, yy = idx & (YB - 1);
    sm[yy * S + swz(z)] = col[(long long)z * ny + yy];
  }
  __syncthreads();
  fft_rows<false, kPlaneEPT, kPlaneThreads, true, true>(sm, YB, d.log2nz, tws, NoIo{}, NoIo{});
  if (REF) {
    double2* dst = ref_out + p * plane + y0;
    for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
      const int z = idx >> d.log2YB, yy = idx & (YB - 1);
      const double2 v = sm[yy * S + swz(z)];
      dst[(long long)z * ny + yy] = make_double2(v.x, -v.y);
    }
    return;
  }
  const int M1 = (d.nx >> 1) + 1;
  const double2* rc = ref_conj + (p % M1) * plane + y0;
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int z = idx >> d.log2YB, yy = idx & (YB - 1);
    double2* e = sm + yy * S + swz(z);
    *e = cross_power(*e, __ldg(rc + (long long)z * ny + yy));
  }
  __syncthreads();
  fft_rows<true, kPlaneEPT, kPlaneThreads, true, true>(sm, YB, d.log2nz, tws, NoIo{}, NoIo{});
  for (int idx = threadIdx.x; idx < E; idx += blockDim.x) {
    const int z = idx >> d.log2YB, yy = idx & (YB - 1);
    col[(long long)z * ny + yy] = sm[yy * S + swz(z)];
  }
}

// (value, index), greater value then smaller index; NaN never wins (phase_argmax_blocks' rule).
__device__ __forceinline__ void better(double& v, long long& i, double v2, long long i2) {
  if (v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// Z[k] = (X[k] + conj X[M-k]) + i W_nx^-k (X[k] - conj X[M-k]): the nx/2-point inverse DFT of Z
// holds the even samples of the real inverse in its real parts and the odd ones in its imaginary
// parts.
__device__ __forceinline__ double2 fold(double2 xa, double2 xb, double2 w) {
  const double2 e = make_double2(xa.x + xb.x, xa.y - xb.y);
  const double2 o = cmul_tw<true>(make_double2(xa.x - xb.x, xa.y + xb.y), w);
  return make_double2(e.x - o.y, e.y + o.x);
}

// Shared memory as plane_rows_fwd_kernel's (bin M of line g at its unswizzled place M).
__global__ void __launch_bounds__(kRowThreads) plane_rows_inv_argmax_kernel(const double2* __restrict__ spec,
                                                                            const double2* __restrict__ tw_x,
                                                                            PlaneDims d, double* __restrict__ bval,
                                                                            long long* __restrict__ bidx,
                                                                            double* __restrict__ surface) {
  extern __shared__ double2 sm[];
  const int M = d.nx >> 1, S = M + 1, G = 1 << d.log2G, H = M >> 1;
  double2* tws = sm + G * S;
  const int r0 = blockIdx.x << d.log2G;
  const double2* in = spec + (long long)blockIdx.y * d.n_complex;
  stage16<4>(
      d.n_twx, [&](int i) { return reinterpret_cast<const uint4*>(tw_x) + i; },
      [&](int i) { return reinterpret_cast<uint4*>(tws) + i; });
  // Bins k and M - k of each row, folded as they arrive (the fold's twiddles from global memory, so
  // that it need not wait for the staged table): four pairs per thread in flight.
  {
    constexpr int K = 4;
    const int n_pairs = (H + 1) << d.log2G;
    for (int base = 0; base < n_pairs; base += K * (int)blockDim.x) {
      double2 xk[K], xm[K];
#pragma unroll
      for (int u = 0; u < K; u++) {
        const int idx = base + (int)threadIdx.x + u * (int)blockDim.x;
        if (idx < n_pairs) {
          const int k = idx >> d.log2G, g = idx & (G - 1);
          xk[u] = in[(long long)k * d.rows + r0 + g];
          xm[u] = in[(long long)(M - k) * d.rows + r0 + g];
        }
      }
#pragma unroll
      for (int u = 0; u < K; u++) {
        const int idx = base + (int)threadIdx.x + u * (int)blockDim.x;
        if (idx < n_pairs) {
          const int k = idx >> d.log2G, g = idx & (G - 1);
          double2* line = sm + g * S;
          const int ik = swz(k), im = k == 0 ? M : swz(M - k);
          line[ik] = fold(xk[u], xm[u], __ldg(tw_x + d.tw_x_post + k));
          if (k > 0 && k < H) line[im] = fold(xm[u], xk[u], __ldg(tw_x + d.tw_x_post + M - k));
        }
      }
    }
  }
  __syncthreads();
  // the last inverse stage feeds the first-maximum search (and the optional surface)
  double v = -DBL_MAX;
  long long best = 0x7fffffffffffffffLL;
  double* surf = surface ? surface + (long long)blockIdx.y * d.n_el : nullptr;
  auto last = [&](int g, int m, double2 z) {
    const long long f = (long long)(r0 + g) * d.nx + 2 * m;
    better(v, best, z.x, f);
    better(v, best, z.y, f + 1);
    if (surf) *reinterpret_cast<double2*>(surf + f) = z;
  };
  fft_rows<true, kRowEPT, kRowThreads, true, false>(sm, G, d.log2M, tws, NoIo{}, last);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double v2 = __shfl_down_sync(0xffffffffu, v, o);
    const long long i2 = __shfl_down_sync(0xffffffffu, best, o);
    better(v, best, v2, i2);
  }
  __shared__ double wv[kRowThreads / 32];
  __shared__ long long wi[kRowThreads / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    wv[warp] = v;
    wi[warp] = best;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) better(v, best, wv[w], wi[w]);
    bval[(long long)blockIdx.y * gridDim.x + blockIdx.x] = v;
    bidx[(long long)blockIdx.y * gridDim.x + blockIdx.x] = best;
  }
}

// spec[kx][r] (planes) -> out[r][kx] (cuFFT's half-spectrum order), r = z * ny + y
__global__ void plane_to_rows_kernel(const double2* __restrict__ in, double2* __restrict__ out, int rows, int M1,
                                     long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / rows, r = i - k * rows;
    out[r * M1 + k] = in[i];
  }
}

template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

int ilog2(long long v) {
  int l = 0;
  while ((1LL << l) < v) l++;
  return l;
}

bool pow2(long long v) { return v > 0 && (v & (v - 1)) == 0; }

}  // namespace

namespace {

// exp(-2 pi i m / n), rounded from long double; exact at the quarter turns.
double2 unit_root(long long m, long long n) {
  m %= n;
  if (m == 0) return make_double2(1.0, 0.0);
  if (4 * m == n) return make_double2(0.0, -1.0);
  if (2 * m == n) return make_double2(-1.0, 0.0);
  if (4 * m == 3 * n) return make_double2(0.0, 1.0);
  const long double a = 6.283185307179586476925286766559L * (long double)m / (long double)n;
  return make_double2((double)cosl(a), (double)-sinl(a));
}

// Stage twiddles of an L-point transform in fft_rows_t's order: for every stage after the first
// (Ns > 1, radix R), W_(Ns R)^(r k) at (r - 1) Ns + k, r = 1..R-1, k = 0..Ns-1.
void stage_table(int L, std::vector<double2>* t) {
  const int log2L = ilog2(L);
  for (int log2Ns = 0; log2Ns < log2L;) {
    const int log2R = std::min(3, log2L - log2Ns);
    const int R = 1 << log2R, Ns = 1 << log2Ns;
    if (Ns > 1)
      for (int r = 1; r < R; r++)
        for (int k = 0; k < Ns; k++) t->push_back(unit_root((long long)r * k, (long long)Ns * R));
    log2Ns += log2R;
  }
}

int stage_count(int L) {
  std::vector<double2> t;
  stage_table(L, &t);
  return (int)t.size();
}

}  // namespace

void plane_twiddles(const PlaneDims& d, std::vector<double2>* tw_x, std::vector<double2>* tw_y,
                    std::vector<double2>* tw_z) {
  tw_x->clear();
  tw_y->clear();
  tw_z->clear();
  stage_table(d.nx / 2, tw_x);
  for (int k = 0; k <= d.nx / 2; k++) tw_x->push_back(unit_root(k, d.nx));  // W_nx^k, k = 0..nx/2
  stage_table(d.ny, tw_y);
  if (d.split) stage_table(d.nz, tw_z);
}

bool plane_dims(int nz, int ny, int nx, PlaneDims* d) {
  if (!pow2(nz) || !pow2(ny) || !pow2(nx) || ny < 8 || ny > 2048 || nx < 16 || nx > 4096) return false;
  const bool fits = nz <= 16 && (long long)nz * ny <= kPlaneThreads * kPlaneEPT;
  // split pass: z columns of 8 .. 1024 points (at least 8 columns per CTA), y lines of >= 16 points
  if (!fits && (nz < 8 || nz > 1024 || ny < 16)) return false;
  d->split = !fits;
  d->log2nz = ilog2(nz);
  d->LY = std::max(1, (kPlaneThreads * kPlaneEPT) / ny);
  d->log2YB = ilog2(std::min<long long>(ny, (kPlaneThreads * kPlaneEPT) / nz));
  d->n_twz = d->split ? stage_count(nz) : 0;
  d->nz = nz;
  d->ny = ny;
  d->nx = nx;
  d->rows = nz * ny;
  d->log2M = ilog2(nx / 2);
  d->log2ny = ilog2(ny);
  int G = 8;
  while (G > 1 && ((long long)G * (nx / 2) > (long long)kRowThreads * kRowEPT || G > d->rows)) G >>= 1;
  d->log2G = ilog2(G);
  d->PP = d->split ? 0 : std::max(1, (kPlaneThreads * kPlaneEPT) / (nz * ny));
  d->n_complex = (long long)(nx / 2 + 1) * d->rows;
  d->n_el = (long long)nx * d->rows;
  d->tw_x_post = stage_count(nx / 2);
  d->n_twx = d->tw_x_post + nx / 2 + 1;  // <= nx: the twiddle slots of the row passes
  d->n_twy = stage_count(ny);            // <  ny
  return true;
}

int plane_blocks_per_frame(const PlaneDims& d) { return d.rows >> d.log2G; }

namespace {
template <bool U16, int SLOT>
cudaError_t launch_rows_fwd(const PlaneDims& d, const void* const* vols, int batch, const double* wy,
                            const double* wx, const double2* tw_x, double2* spec, cudaStream_t s, const SlotOut& so) {
  const size_t smem = rows_smem_bytes(d);
  cudaError_t e = allow_smem(plane_rows_fwd_kernel<U16, SLOT>, smem);
  if (e != cudaSuccess) return e;
  plane_rows_fwd_kernel<U16, SLOT><<<dim3(d.rows >> d.log2G, batch), kRowThreads, smem, s>>>(vols, wy, wx, tw_x, d,
                                                                                             spec, so);
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_plane_rows_fwd(const PlaneDims& d, const void* const* vols, int in_kind, int batch,
                                  const double* wy, const double* wx, const double2* tw_x, double2* spec,
                                  cudaStream_t s, const SlotOut* slot) {
  const SlotOut so = slot ? *slot : SlotOut{nullptr, -1, 0, 0};
  const int k = slot ? slot->kind : -1;
  if (in_kind == FA_U16) {
    if (k == kFrameRawU16) return launch_rows_fwd<true, kFrameRawU16>(d, vols, batch, wy, wx, tw_x, spec, s, so);
    if (k == kFrameF16) return launch_rows_fwd<true, kFrameF16>(d, vols, batch, wy, wx, tw_x, spec, s, so);
    if (k == kFrameF32) return launch_rows_fwd<true, kFrameF32>(d, vols, batch, wy, wx, tw_x, spec, s, so);
    return launch_rows_fwd<true, -1>(d, vols, batch, wy, wx, tw_x, spec, s, so);
  }
  if (k == kFrameF16) return launch_rows_fwd<false, kFrameF16>(d, vols, batch, wy, wx, tw_x, spec, s, so);
  if (k == kFrameF32) return launch_rows_fwd<false, kFrameF32>(d, vols, batch, wy, wx, tw_x, spec, s, so);
  return launch_rows_fwd<false, -1>(d, vols, batch, wy, wx, tw_x, spec, s, so);
}

namespace {
template <int NZ, bool REF>
cudaError_t launch_yz(const PlaneDims& d, const double2* in, double2* out, const double2* ref_conj,
                      const double2* tw_y, long long n_planes, cudaStream_t s) {
  if constexpr (NZ >= 4) {
    if ((long long)NZ * d.ny == 2LL * kPairThreads * kPairEPT) {  // one plane per pair of CTAs
      const size_t smem = ((size_t)(NZ / 2) * (d.ny + 1) + d.ny) * sizeof(double2);
      cudaError_t e = allow_smem(plane_yz_pair_kernel<NZ, REF>, smem);
      if (e != cudaSuccess) return e;
      plane_yz_pair_kernel<NZ, REF><<<(unsigned)(2 * n_planes), kPairThreads, smem, s>>>(in, out, ref_conj, tw_y, d);
      return cudaGetLastError();
    }
  }
  const size_t smem = ((size_t)d.PP * NZ * (d.ny + 1) + d.ny) * sizeof(double2);
  cudaError_t e = allow_smem(plane_yz_kernel<NZ, REF>, smem);
  if (e != cudaSuccess) return e;
  const long long grid = (n_planes + d.PP - 1) / d.PP;
  plane_yz_kernel<NZ, REF><<<(unsigned)grid, kPlaneThreads, smem, s>>>(in, out, ref_conj, tw_y, d, n_planes);
  return cudaGetLastError();
}

template <bool REF>
cudaError_t launch_yz_nz(const PlaneDims& d, const double2* in, double2* out, const double2* ref_conj,
                         const double2* tw_y, long long n_planes, cudaStream_t s) {
  switch (d.nz) {
    case 1: return launch_yz<1, REF>(d, in, out, ref_conj, tw_y, n_planes, s);
    case 2: return launch_yz<2, REF>(d, in, out, ref_conj, tw_y, n_planes, s);
    case 4: return launch_yz<4, REF>(d, in, out, ref_conj, tw_y, n_planes, s);
    case 8: return launch_yz<8, REF>(d, in, out, ref_conj, tw_y, n_planes, s);
    case 16: return launch_yz<16, REF>(d, in, out, ref_conj, tw_y, n_planes, s);
    default: return cudaErrorInvalidValue;
  }
}
}  // namespace

cudaError_t launch_plane_yz(const PlaneDims& d, const double2* in, double2* out, const double2* ref_conj,
                            const double2* tw_y, int batch, bool reference, cudaStream_t s) {
  const long long n_planes = (long long)batch * ((d.nx >> 1) + 1);
  return reference ? launch_yz_nz<true>(d, in, out, nullptr, tw_y, n_planes, s)
                   : launch_yz_nz<false>(d, in, out, ref_conj, tw_y, n_planes, s);
}

cudaError_t launch_plane_yz_split(const PlaneDims& d, double2* spec, double2* ref_conj, const double2* tw_y,
                                  const double2* tw_z, int batch, bool reference, cudaStream_t s) {
  if (!d.split) return cudaErrorInvalidValue;
  const long long n_planes = (long long)batch * ((d.nx >> 1) + 1);
  const long long n_lines = n_planes * d.nz;
  const size_t smem_y = ((size_t)d.LY * (d.ny + 1) + d.ny) * sizeof(double2);
  const size_t smem_z = (((size_t)1 << d.log2YB) * (d.nz + 1) + d.nz) * sizeof(double2);
  const long long grid_y = (n_lines + d.LY - 1) / d.LY;
  const long long grid_z = n_planes * (d.ny >> d.log2YB);
  cudaError_t e = allow_smem(plane_y_kernel<false>, smem_y);
  if (e == cudaSuccess) e = allow_smem(plane_y_kernel<true>, smem_y);
  if (e == cudaSuccess) e = allow_smem(plane_z_kernel<false>, smem_z);
  if (e == cudaSuccess) e = allow_smem(plane_z_kernel<true>, smem_z);
  if (e != cudaSuccess) return e;
  plane_y_kernel<false><<<(unsigned)grid_y, kPlaneThreads, smem_y, s>>>(spec, tw_y, d, n_lines);
  if (reference) {
    plane_z_kernel<true><<<(unsigned)grid_z, kPlaneThreads, smem_z, s>>>(spec, ref_conj, nullptr, tw_z, d);
    return cudaGetLastError();
  }
  plane_z_kernel<false><<<(unsigned)grid_z, kPlaneThreads, smem_z, s>>>(spec, nullptr, ref_conj, tw_z, d);
  plane_y_kernel<true><<<(unsigned)grid_y, kPlaneThreads, smem_y, s>>>(spec, tw_y, d, n_lines);
  return cudaGetLastError();
}

cudaError_t launch_plane_to_rows(const PlaneDims& d, const double2* in, double2* out, cudaStream_t s) {
  const int blocks = (int)std::min<long long>((d.n_complex + 255) / 256, 148 * 8);
  plane_to_rows_kernel<<<blocks, 256, 0, s>>>(in, out, d.rows, (d.nx >> 1) + 1, d.n_complex);
  return cudaGetLastError();
}

cudaError_t launch_plane_rows_inv_argmax(const PlaneDims& d, const double2* spec, int batch, const double2* tw_x,
                                         double* bval, long long* bidx, double* surface, cudaStream_t s) {
  const size_t smem = rows_smem_bytes(d);
  cudaError_t e = allow_smem(plane_rows_inv_argmax_kernel, smem);
  if (e != cudaSuccess) return e;
  plane_rows_inv_argmax_kernel<<<dim3(d.rows >> d.log2G, batch), kRowThreads, smem, s>>>(spec, tw_x, d, bval, bidx,
                                                                                         surface);
  return cudaGetLastError();
}

}  // namespace fa
