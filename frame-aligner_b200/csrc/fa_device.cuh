// fa_device.cuh -- device helpers shared by several translation units.
#pragma once

#include "fa_kernels.cuh"

namespace fa {

// ------------------------------------------------------------------ loads ------------------------

template <typename T>
__device__ __forceinline__ float ldf(const T* p);
template <>
__device__ __forceinline__ float ldf<float>(const float* p) { return __ldg(p); }
template <>
__device__ __forceinline__ float ldf<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <>
__device__ __forceinline__ float ldf<__nv_bfloat16>(const __nv_bfloat16* p) { return __bfloat162float(__ldg(p)); }

// uint16 frame storage holding photon count + 1 (FrameWarpAligner.cpp:142), saturated at 65535; the
// zero halo stays zero. Reads are exact: 2^23 + u is representable, so subtracting the magic
// constant converts without a conversion instruction.
struct RawU16 {
  unsigned short v;
};
__device__ __forceinline__ float u16f(unsigned u) { return __uint_as_float(0x4B000000u | u) - 8388608.0f; }
template <>
__device__ __forceinline__ float ldf<RawU16>(const RawU16* p) {
  return u16f(__ldg(reinterpret_cast<const unsigned short*>(p)));
}

// Compile-time kernel configuration: dimensionality, frame storage type, reference storage type.
template <int N, typename FT, typename RT>
struct KCfg {
  static constexpr int nd = N;
  using F = FT;
  using R = RT;
};

// Calls f(KCfg<...>{}) for the runtime combination (n_dim, frame kind, BF16 reference or not).
template <typename Fn>
inline cudaError_t dispatch_cfg(int n_dim, int kind, bool ref_bf16, Fn&& f) {
  if (n_dim == 3) {
    if (kind == kFrameRawU16) return ref_bf16 ? f(KCfg<3, RawU16, __nv_bfloat16>{}) : f(KCfg<3, RawU16, float>{});
    if (kind == kFrameF16) return ref_bf16 ? f(KCfg<3, __half, __nv_bfloat16>{}) : f(KCfg<3, __half, float>{});
    return ref_bf16 ? f(KCfg<3, float, __nv_bfloat16>{}) : f(KCfg<3, float, float>{});
  }
  if (kind == kFrameRawU16) return ref_bf16 ? f(KCfg<2, RawU16, __nv_bfloat16>{}) : f(KCfg<2, RawU16, float>{});
  if (kind == kFrameF16) return ref_bf16 ? f(KCfg<2, __half, __nv_bfloat16>{}) : f(KCfg<2, __half, float>{});
  return ref_bf16 ? f(KCfg<2, float, __nv_bfloat16>{}) : f(KCfg<2, float, float>{});
}

// ------------------------------------------------------------------ per-voxel model --------------

// Interval, fraction and storage-range bookkeeping of one voxel (see RowDesc).
struct VoxelModel {
  int di;      // displacement interval
  float f;     // fraction within it
  int r;       // storage range (steepest-descent images)
  bool last;   // last voxel of its storage range
};

__device__ __forceinline__ VoxelModel voxel_model(const RowDesc& rd, int x, int nx, bool flip, bool bidir, float dq) {
  VoxelModel v;
  const int xs = flip ? nx - 1 - x : x;
  v.di = rd.di0 + (xs >= rd.xdi ? 1 : 0);
  float f = fmaf((float)xs, dq, rd.qbase) - (float)(v.di - rd.di0);
  v.f = fminf(fmaxf(f, 0.0f), 1.0f);
  v.r = bidir ? rd.r0 + (x >= rd.xr ? 1 : 0) : v.di;
  v.last = (x == rd.xlast);
  return v;
}

// Zero-padded trilinear (bilinear for NDIM == 2) sample of the frame at (x, y, z) + d, where
// d = int(D) + frac(D) + f * dD from the control-point parameters P (3 float4). Returns the
// interpolated value; exactly 0 when every contributing tap is outside (getZeroPadded,
// FrameWarper.h:39-47).
template <int NDIM, typename FT>
__device__ __forceinline__ float sample(const FT* __restrict__ fr, long long fplane, int fpitch, const float4* P, float f,
                                        int x, int y, int z, int nx, int ny, int nz) {
  const float4 n = P[0], ph = P[1], dd = P[2];
  const float tx = fmaf(f, dd.x, ph.x);
  const float ty = fmaf(f, dd.y, ph.y);
  const float flx = floorf(tx), fly = floorf(ty);
  const float wx = tx - flx, wy = ty - fly;
  const int ix = x + (int)n.x + (int)flx;
  const int iy = y + (int)n.y + (int)fly;
  const bool vx0 = (unsigned)ix < (unsigned)nx, vx1 = (unsigned)(ix + 1) < (unsigned)nx;
  const bool vy0 = (unsigned)iy < (unsigned)ny, vy1 = (unsigned)(iy + 1) < (unsigned)ny;
  if (NDIM == 2) {
    const long long b = (long long)iy * fpitch + ix;
    const float v00 = (vy0 && vx0) ? ldf(fr + b) : 0.0f;
    const float v01 = (vy0 && vx1) ? ldf(fr + b + 1) : 0.0f;
    const float v10 = (vy1 && vx0) ? ldf(fr + b + fpitch) : 0.0f;
    const float v11 = (vy1 && vx1) ? ldf(fr + b + fpitch + 1) : 0.0f;
    const float c0 = fmaf(wx, v01 - v00, v00);
    const float c1 = fmaf(wx, v11 - v10, v10);
    return fmaf(wy, c1 - c0, c0);
  } else {
    const float tz = fmaf(f, dd.z, ph.z);
    const float flz = floorf(tz);
    const float wz = tz - flz;
    const int iz = z + (int)n.z + (int)flz;
    const bool vz0 = (unsigned)iz < (unsigned)nz, vz1 = (unsigned)(iz + 1) < (unsigned)nz;
    const long long b = (long long)iz * fplane + (long long)iy * fpitch + ix;
    const float v000 = (vz0 && vy0 && vx0) ? ldf(fr + b) : 0.0f;
    const float v001 = (vz0 && vy0 && vx1) ? ldf(fr + b + 1) : 0.0f;
    const float v010 = (vz0 && vy1 && vx0) ? ldf(fr + b + fpitch) : 0.0f;
    const float v011 = (vz0 && vy1 && vx1) ? ldf(fr + b + fpitch + 1) : 0.0f;
    const float v100 = (vz1 && vy0 && vx0) ? ldf(fr + b + fplane) : 0.0f;
    const float v101 = (vz1 && vy0 && vx1) ? ldf(fr + b + fplane + 1) : 0.0f;
    const float v110 = (vz1 && vy1 && vx0) ? ldf(fr + b + fplane + fpitch) : 0.0f;
    const float v111 = (vz1 && vy1 && vx1) ? ldf(fr + b + fplane + fpitch + 1) : 0.0f;
    const float c00 = fmaf(wx, v001 - v000, v000);
    const float c01 = fmaf(wx, v011 - v010, v010);
    const float c10 = fmaf(wx, v101 - v100, v100);
    const float c11 = fmaf(wx, v111 - v110, v110);
    const float c0 = fmaf(wy, c01 - c00, c00);
    const float c1 = fmaf(wy, c11 - c10, c10);
    return fmaf(wz, c1 - c0, c0);
  }
}

constexpr int kWin = 5;  // control points [c0-1, c0+4) cover every interval a tile can touch

// f = sum over tiles (thread-strided runs, then a fixed tree); g[c] = sum over the tiles listed in
// ctrl_tiles[c], in tile order.
__device__ __forceinline__ void reduce_partials(const RefDev& R, const double* __restrict__ parts, double* f_out, double* g_out) {
  __shared__ double sf[kSolveThreads];
  double acc = 0.0;
  for (int t = threadIdx.x; t < R.n_tiles; t += blockDim.x) acc += parts[(long long)t * kPartialDoubles];
  sf[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sf[threadIdx.x] += sf[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *f_out = sf[0];
  const int nd = R.n_dim;
  for (int i = threadIdx.x; i < R.P; i += blockDim.x) {
    const int c = i / nd, k = i % nd;
    const int2 tr = R.ctrl_tiles[c];
    double a = 0.0;
#pragma unroll 8
    for (int t = tr.x; t < tr.y; t++) {
      const double* pt = parts + (long long)t * kPartialDoubles;
      const int s = c - R.tile_c0[t];
      const double v = (s >= 0 && s < 3) ? pt[2 + s * 3 + k] : 0.0;
      a += v;
    }
    g_out[i] = a;
  }
  __syncthreads();
}

// Control-point parameters (kDParamF4 float4 per control point) of the trial point D = x + p, from
// job.x and job.p; control points k = t0, t0 + stride, ...
__device__ __forceinline__ void write_trial_dparams(const Job& job, const RefDev& R, int t0, int stride) {
  const int nd = R.n_dim;
  for (int k = t0; k < R.nD; k += stride) {
    double d[3], dn[3];
    for (int c = 0; c < 3; c++) {
      d[c] = c < nd ? job.x[k * nd + c] + job.p[k * nd + c] : 0.0;
      dn[c] = (c < nd && k + 1 < R.nD) ? job.x[(k + 1) * nd + c] + job.p[(k + 1) * nd + c] : d[c];
    }
    const double f0 = floor(d[0]), f1 = floor(d[1]), f2 = floor(d[2]);
    job.dparams[k * kDParamF4 + 0] = make_float4((float)f0, (float)f1, (float)f2, 0.f);
    job.dparams[k * kDParamF4 + 1] = make_float4((float)(d[0] - f0), (float)(d[1] - f1), (float)(d[2] - f2), 0.f);
    job.dparams[k * kDParamF4 + 2] =
        make_float4((float)(dn[0] - d[0]), (float)(dn[1] - d[1]), (float)(dn[2] - d[2]), 0.f);
  }
}

// Control-point parameters of the displacement D[k] = d for every control point (a rigid shift):
// the values write_trial_dparams produces for x + p = d, computed the same way.
__device__ __forceinline__ void write_const_dparams(float4* dp, int nD, int nd, const double* d3, int t0, int stride) {
  double d[3];
  for (int c = 0; c < 3; c++) d[c] = c < nd ? 0.0 + d3[c] : 0.0;
  const double f0 = floor(d[0]), f1 = floor(d[1]), f2 = floor(d[2]);
  for (int k = t0; k < nD; k += stride) {
    dp[k * kDParamF4 + 0] = make_float4((float)f0, (float)f1, (float)f2, 0.f);
    dp[k * kDParamF4 + 1] = make_float4((float)(d[0] - f0), (float)(d[1] - f1), (float)(d[2] - f2), 0.f);
    dp[k * kDParamF4 + 2] = make_float4((float)(d[0] - d[0]), (float)(d[1] - d[1]), (float)(d[2] - d[2]), 0.f);
  }
}

}  // namespace fa
