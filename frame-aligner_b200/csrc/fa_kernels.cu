// fa_kernels.cu -- sm_100a kernels of the warper path.
//
//   sobel_tiled_kernel  Sobel3d (FrameAligner/Sobel3d.cpp:8-85), bit-exact float arithmetic
//   hessian_*       computeSteepestDecentImages + computeHessian (FrameWarper.cpp:296-395)
//   eval_kernel     fused warpImageInterpolated + computeErrorImage + computeJacobian
//                   (FrameWarper.cpp:4-69,147-176): one HBM pass per frame evaluation
//   reduce_kernel   deterministic tile -> frame reduction of f and J^T e
//   warp_kernel     warpImageInterpolated output image
//
// Layout: volumes {nz, ny, nx}, x fastest. A tile is `tile_rows` consecutive image rows; the host
// picks tile_rows so that a tile meets at most two storage ranges (three control points).
#include <algorithm>

#include "fa_device.cuh"

namespace fa {

// ------------------------------------------------------------------ Sobel3d ----------------------

// One separable pass at position i of an axis of length n (Sobel3d.cpp:8-58): interior
// f0*G(i-1) + f1*G(i) + f2*G(i+1); edges e1 = {e1a*G(0) + e1b*G(1)}, e2 = {e2a*G(n-1) + e2b*G(n-2)}.
// Float products and sums are rounded one by one (no FMA), as in the reference build.
template <typename G>
__device__ __forceinline__ float pass(int i, int n, bool copy_if_single, const float* f, const float* e1,
                                      const float* e2, G get) {
  if (n == 1 && copy_if_single) return get(i);
  if (i == 0) return __fadd_rn(__fmul_rn(e1[0], get(0)), __fmul_rn(e1[1], get(1)));
  if (i == n - 1) return __fadd_rn(__fmul_rn(e2[0], get(n - 1)), __fmul_rn(e2[1], get(n - 2)));
  return __fadd_rn(__fadd_rn(__fmul_rn(f[0], get(i - 1)), __fmul_rn(f[1], get(i))), __fmul_rn(f[2], get(i + 1)));
}

// Sobel3d (Sobel3d.cpp:60-85) with each separable pass computed once per voxel: a CTA takes a tile of
// kSbZ x kSbY x kSbX outputs, loads the reference over the tile plus a one-voxel halo (clipped to the
// volume) into shared memory and forms the intermediate images there -- a = Sx(m) and a' = Sy(m) on
// the halo, then b = Sy(a), c = Sz(a), b' = Sz(a'), then gz = Dz(b), gy = Dy(c), gx = Dx(b'). Every
// value is produced by `pass` with the global index along its axis, so the edge rules apply at the
// volume's faces and every product and sum is rounded in the reference's order: gx = Dx(Sz(Sy(m))),
// gy = Dy(Sz(Sx(m))), gz = Dz(Sy(Sx(m))) (Sobel3d.cpp:73-84), bit for bit.
constexpr int kSbX = 32, kSbY = 8, kSbZ = 4;
constexpr int kSbHX = kSbX + 2, kSbHY = kSbY + 2, kSbHZ = kSbZ + 2;
constexpr int kSbVol = kSbHX * kSbHY * kSbHZ;

__global__ void __launch_bounds__(256) sobel_tiled_kernel(const float* __restrict__ m, int nz, int ny, int nx,
                                                          float* __restrict__ gx, float* __restrict__ gy,
                                                          float* __restrict__ gz) {
  __shared__ float sM[kSbVol];   // m, later b
  __shared__ float sA[kSbVol];   // a = Sx(m)
  __shared__ float sA2[kSbVol];  // a' = Sy(m)
  __shared__ float sC[kSbVol];   // c = Sz(a)
  __shared__ float sB2[kSbVol];  // b' = Sz(a')
  const float sm[3] = {1.0f / 4.0f, 2.0f / 4.0f, 1.0f / 4.0f};
  const float se[2] = {2.0f / 3.0f, 2.0f / 3.0f};
  const float dm[3] = {-0.5f, 0.0f, 0.5f};
  const float de1[2] = {-0.5f, 0.5f};
  const float de2[2] = {0.5f, -0.5f};
  const int x0 = blockIdx.x * kSbX, y0 = blockIdx.y * kSbY, z0 = blockIdx.z * kSbZ;
  // local index of global (z, y, x): origin at (z0 - 1, y0 - 1, x0 - 1)
  auto L = [&](int z, int y, int x) { return ((z - z0 + 1) * kSbHY + (y - y0 + 1)) * kSbHX + (x - x0 + 1); };
  // a range [lo, hi) of global positions along an axis, clipped to the volume
  const int hz0 = max(z0 - 1, 0), hz1 = min(z0 + kSbZ + 1, nz), tz1 = min(z0 + kSbZ, nz);
  const int hy0 = max(y0 - 1, 0), hy1 = min(y0 + kSbY + 1, ny), ty1 = min(y0 + kSbY, ny);
  const int hx0 = max(x0 - 1, 0), hx1 = min(x0 + kSbX + 1, nx), tx1 = min(x0 + kSbX, nx);
  // run f(z, y, x) over a box
  auto box = [&](int za, int zb, int ya, int yb, int xa, int xb, auto f) {
    const int wx = xb - xa, wy = yb - ya, n = (zb - za) * wy * wx;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int x = xa + i % wx, r = i / wx;
      f(za + r / wy, ya + r % wy, x);
    }
  };
  box(hz0, hz1, hy0, hy1, hx0, hx1,
      [&](int z, int y, int x) { sM[L(z, y, x)] = __ldg(m + ((long long)z * ny + y) * nx + x); });
  __syncthreads();
  // a = Sx(m) on (halo z, halo y, tile x); a' = Sy(m) on (halo z, tile y, halo x)
  box(hz0, hz1, hy0, hy1, x0, tx1, [&](int z, int y, int x) {
    sA[L(z, y, x)] = pass(x, nx, false, sm, se, se, [&](int k) { return sM[L(z, y, k)]; });
  });
  box(hz0, hz1, y0, ty1, hx0, hx1, [&](int z, int y, int x) {
    sA2[L(z, y, x)] = pass(y, ny, false, sm, se, se, [&](int k) { return sM[L(z, k, x)]; });
  });
  __syncthreads();
  // b = Sy(a) on (halo z, tile y, tile x) into sM; c = Sz(a) on (tile z, halo y, tile x);
  // b' = Sz(a') on (tile z, tile y, halo x)
  box(hz0, hz1, y0, ty1, x0, tx1, [&](int z, int y, int x) {
    sM[L(z, y, x)] = pass(y, ny, false, sm, se, se, [&](int k) { return sA[L(z, k, x)]; });
  });
  box(z0, tz1, hy0, hy1, x0, tx1, [&](int z, int y, int x) {
    sC[L(z, y, x)] = pass(z, nz, true, sm, se, se, [&](int k) { return sA[L(k, y, x)]; });
  });
  box(z0, tz1, y0, ty1, hx0, hx1, [&](int z, int y, int x) {
    sB2[L(z, y, x)] = pass(z, nz, true, sm, se, se, [&](int k) { return sA2[L(k, y, x)]; });
  });
  __syncthreads();
  box(z0, tz1, y0, ty1, x0, tx1, [&](int z, int y, int x) {
    const long long p = ((long long)z * ny + y) * nx + x;
    gz[p] = pass(z, nz, true, dm, de1, de2, [&](int k) { return sM[L(k, y, x)]; });
    gy[p] = pass(y, ny, false, dm, de1, de2, [&](int k) { return sC[L(z, k, x)]; });
    gx[p] = pass(x, nx, false, dm, de1, de2, [&](int k) { return sB2[L(z, y, k)]; });
  });
}

cudaError_t launch_sobel(const float* m, int nz, int ny, int nx, float* gx, float* gy, float* gz, cudaStream_t s) {
  const dim3 grid((nx + kSbX - 1) / kSbX, (ny + kSbY - 1) / kSbY, (nz + kSbZ - 1) / kSbZ);
  sobel_tiled_kernel<<<grid, 256, 0, s>>>(m, nz, ny, nx, gx, gy, gz);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ conversions ------------------

__global__ void to_bf16_kernel(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

cudaError_t launch_to_bf16(const float* in, __nv_bfloat16* out, long long n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  to_bf16_kernel<<<blocks, 256, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

__global__ void to_quad16_kernel(const float* __restrict__ ref, const float* __restrict__ gx,
                                 const float* __restrict__ gy, const float* __restrict__ gz, long long n,
                                 __nv_bfloat16* __restrict__ q16) {
  const long long groups = (n + 3) / 4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < groups * 16;
       i += (long long)gridDim.x * blockDim.x) {
    const long long g = i >> 4;
    const int k = (int)(i >> 2) & 3, j = (int)i & 3;
    const long long p = 4 * g + j;
    const float* src = k == 0 ? ref : (k == 1 ? gx : (k == 2 ? gy : gz));
    q16[i] = __float2bfloat16_rn(p < n ? src[p] : 0.0f);
  }
}

cudaError_t launch_to_quad16(const float* ref, const float* gx, const float* gy, const float* gz, long long n,
                             __nv_bfloat16* q16, cudaStream_t s) {
  const long long total = (n + 3) / 4 * 16;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  to_quad16_kernel<<<blocks, 256, 0, s>>>(ref, gx, gy, gz, n, q16);
  return cudaGetLastError();
}

__device__ __forceinline__ float load_any(const void* in, int t, long long i) {
  switch (t) {
    case FA_F32: return static_cast<const float*>(in)[i];
    case FA_F16: return __half2float(static_cast<const __half*>(in)[i]);
    case FA_BF16: return __bfloat162float(static_cast<const __nv_bfloat16*>(in)[i]);
    default: return (float)static_cast<const uint16_t*>(in)[i];
  }
}

__global__ void convert_kernel(const void* __restrict__ in, int in_t, void* __restrict__ out, int out_t, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float v = load_any(in, in_t, i);
    if (out_t == FA_F16)
      static_cast<__half*>(out)[i] = __float2half_rn(v);
    else
      static_cast<float*>(out)[i] = v;
  }
}

cudaError_t launch_convert(const void* in, fa_dtype in_type, void* out, fa_dtype out_type, long long n,
                           cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  convert_kernel<<<blocks, 256, 0, s>>>(in, (int)in_type, out, (int)out_type, n);
  return cudaGetLastError();
}

// Raw frame (any dtype) -> warper storage with FrameWarpAligner's +1 offset
// (FrameWarpAligner.cpp:142), converted to float first as the reference does (convertTo CV_32F).
__global__ void offset_convert_kernel(const void* __restrict__ in, int in_t, void* __restrict__ out, int out_t,
                                      long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float v = load_any(in, in_t, i) + 1.0f;
    if (out_t == FA_F16)
      static_cast<__half*>(out)[i] = __float2half_rn(v);
    else
      static_cast<float*>(out)[i] = v;
  }
}

cudaError_t launch_offset_convert(const void* in, fa_dtype in_type, void* out, fa_dtype out_type, long long n,
                                  cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  offset_convert_kernel<<<blocks, 256, 0, s>>>(in, (int)in_type, out, (int)out_type, n);
  return cudaGetLastError();
}

// Raw or converted values into a frame slot's interior (row pitch fpitch, plane stride fplane, out
// pointing at voxel (0,0,0)); add_one applies FrameWarpAligner's +1 (FrameWarpAligner.cpp:142).
__global__ void to_slot_kernel(const void* __restrict__ in, int in_t, void* __restrict__ out, int out_kind, int ny,
                               int nx, int n_rows, int fpitch, long long fplane, int add_one) {
  for (int row = blockIdx.x; row < n_rows; row += gridDim.x) {
    const int y = row % ny, z = row / ny;
    const long long ib = (long long)row * nx;
    const long long ob = (long long)z * fplane + (long long)y * fpitch;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      if (out_kind == kFrameRawU16) {
        // count + 1, saturated (a raw count of 65535 is stored as 65535)
        const unsigned c = static_cast<const unsigned short*>(in)[ib + x] + (add_one ? 1u : 0u);
        static_cast<unsigned short*>(out)[ob + x] = (unsigned short)(c > 65535u ? 65535u : c);
      } else {
        const float v = load_any(in, in_t, ib + x) + (add_one ? 1.0f : 0.0f);
        if (out_kind == kFrameF16)
          static_cast<__half*>(out)[ob + x] = __float2half_rn(v);
        else
          static_cast<float*>(out)[ob + x] = v;
      }
    }
  }
}

// The same conversion 8 elements per thread with 16-byte loads and stores (rows of a multiple of 8
// elements, 16-byte aligned rows on both sides): dense FP32 or uint16 in, slot storage IN_U16 ->
// raw counts (saturated + 1) or FP16 / FP32 values.
template <bool IN_U16, int OUT_KIND>
__global__ void __launch_bounds__(256) to_slot_vec_kernel(const void* __restrict__ in, void* __restrict__ out,
                                                          int nx8, int ny, long long n_chunks, int fpitch,
                                                          long long fplane, int add_one) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n_chunks;
       c += (long long)gridDim.x * blockDim.x) {
    const long long row = c / nx8;
    const int xc = (int)(c - row * nx8);
    const int y = (int)(row % ny);
    const long long z = row / ny;
    const long long ib = c * 8;  // rows are dense: row * nx + 8 * xc
    const long long ob = z * fplane + (long long)y * fpitch + 8 * xc;
    if (OUT_KIND == kFrameRawU16) {
      // count + 1, saturated (a raw count of 65535 is stored as 65535)
      uint4 q = *reinterpret_cast<const uint4*>(static_cast<const unsigned short*>(in) + ib);
      unsigned w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const unsigned lo = min((w[i] & 0xffffu) + (unsigned)add_one, 65535u);
        const unsigned hi = min((w[i] >> 16) + (unsigned)add_one, 65535u);
        w[i] = lo | (hi << 16);
      }
      *reinterpret_cast<uint4*>(static_cast<unsigned short*>(out) + ob) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
      float v[8];
      if (IN_U16) {
        const uint4 q = *reinterpret_cast<const uint4*>(static_cast<const unsigned short*>(in) + ib);
        const unsigned w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
          v[2 * i] = (float)(w[i] & 0xffffu);
          v[2 * i + 1] = (float)(w[i] >> 16);
        }
      } else {
        const float4 a = *reinterpret_cast<const float4*>(static_cast<const float*>(in) + ib);
        const float4 b = *reinterpret_cast<const float4*>(static_cast<const float*>(in) + ib + 4);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
      }
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] = v[i] + (add_one ? 1.0f : 0.0f);
      if (OUT_KIND == kFrameF16) {
        __half2 h[4];
#pragma unroll
        for (int i = 0; i < 4; i++) h[i] = __halves2half2(__float2half_rn(v[2 * i]), __float2half_rn(v[2 * i + 1]));
        *reinterpret_cast<uint4*>(static_cast<__half*>(out) + ob) = *reinterpret_cast<const uint4*>(h);
      } else {
        float* o = static_cast<float*>(out) + ob;
        *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<float4*>(o + 4) = make_float4(v[4], v[5], v[6], v[7]);
      }
    }
  }
}

cudaError_t launch_to_slot(const void* in, fa_dtype in_type, void* out, int out_kind, int nz, int ny, int nx,
                           int fpitch, long long fplane, bool add_one, cudaStream_t s) {
  const int n_rows = nz * ny;
  const size_t out_esz = out_kind == kFrameF32 ? 4 : 2;
  const bool vec = nx % 8 == 0 && (in_type == FA_U16 || in_type == FA_F32) &&
                   (out_kind != kFrameRawU16 || in_type == FA_U16) && reinterpret_cast<uintptr_t>(in) % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(out) % 16 == 0 && (fpitch * out_esz) % 16 == 0 &&
                   (fplane * (long long)out_esz) % 16 == 0;
  if (vec) {
    const long long n_chunks = (long long)n_rows * (nx / 8);
    const int blocks = (int)std::min<long long>((n_chunks + 255) / 256, 148 * 8);
    const int a1 = add_one ? 1 : 0;
    if (in_type == FA_U16) {
      if (out_kind == kFrameRawU16)
        to_slot_vec_kernel<true, kFrameRawU16><<<blocks, 256, 0, s>>>(in, out, nx / 8, ny, n_chunks, fpitch, fplane, a1);
      else if (out_kind == kFrameF16)
        to_slot_vec_kernel<true, kFrameF16><<<blocks, 256, 0, s>>>(in, out, nx / 8, ny, n_chunks, fpitch, fplane, a1);
      else
        to_slot_vec_kernel<true, kFrameF32><<<blocks, 256, 0, s>>>(in, out, nx / 8, ny, n_chunks, fpitch, fplane, a1);
    } else {
      if (out_kind == kFrameF16)
        to_slot_vec_kernel<false, kFrameF16><<<blocks, 256, 0, s>>>(in, out, nx / 8, ny, n_chunks, fpitch, fplane, a1);
      else
        to_slot_vec_kernel<false, kFrameF32><<<blocks, 256, 0, s>>>(in, out, nx / 8, ny, n_chunks, fpitch, fplane, a1);
    }
    return cudaGetLastError();
  }
  int blocks = n_rows < 148 * 16 ? n_rows : 148 * 16;
  to_slot_kernel<<<blocks, 256, 0, s>>>(in, (int)in_type, out, out_kind, ny, nx, n_rows, fpitch, fplane, add_one ? 1 : 0);
  return cudaGetLastError();
}

// downsample (AbstractFrameAligner.cpp:37-56): output (z, y/b, x/b) = float sum of its b x b block,
// accumulated in the reference's loop order (y, then x).
__global__ void downsample_kernel(const void* __restrict__ in, int in_t, int nz, int ny, int nx, int b,
                                  float* __restrict__ out) {
  const int nh = (ny + b - 1) / b, nw = (nx + b - 1) / b;
  const long long n = (long long)nz * nh * nw;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int ox = (int)(o % nw);
    const long long r = o / nw;
    const int oy = (int)(r % nh);
    const int z = (int)(r / nh);
    float acc = 0.0f;
    for (int y = oy * b; y < min(ny, oy * b + b); y++)
      for (int x = ox * b; x < min(nx, ox * b + b); x++)
        acc = __fadd_rn(acc, load_any(in, in_t, ((long long)z * ny + y) * nx + x));
    out[o] = acc;
  }
}

cudaError_t launch_downsample(const void* in, fa_dtype in_type, int nz, int ny, int nx, int b, float* out,
                              cudaStream_t s) {
  long long n = (long long)nz * ((ny + b - 1) / b) * ((nx + b - 1) / b);
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) blocks = 1;
  downsample_kernel<<<blocks, 256, 0, s>>>(in, (int)in_type, nz, ny, nx, b, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ fused evaluation -------------

template <int NDIM, typename FT, typename RT>
__global__ void __launch_bounds__(kEvalThreads) eval_kernel(const Job* __restrict__ jobs) {
  const Job& job = jobs[blockIdx.y];
  if (job.state != nullptr && (job.state->phase == kPhaseDone || job.state->phase == kPhaseWaitWarm)) return;
  const RefDev& R = *job.ref;
  const int tile = blockIdx.x;
  if (tile >= R.n_tiles) return;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  const int row_begin = tile * R.tile_rows;
  const int row_end = min(row_begin + R.tile_rows, R.n_rows);
  const int c0 = R.tile_c0[tile];
  const int cw = max(c0 - 1, 0);
  const bool bidir = R.bidir != 0;
  const float dq = R.dq;

  __shared__ float4 sD[kWin * kDParamF4];
  __shared__ float sred[kEvalWarps][1 + 3 * NDIM];
  for (int i = threadIdx.x; i < kWin * kDParamF4; i += blockDim.x) {
    const int k = cw + i / kDParamF4;
    sD[i] = (k < R.nD) ? job.dparams[k * kDParamF4 + i % kDParamF4] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncthreads();

  const FT* __restrict__ fr = static_cast<const FT*>(job.frame);
  // reference / gradient value k (0: reference, 1..3: gx, gy, gz) of voxel p
  auto refgrad = [&](int k, long long p) -> float {
    if constexpr (sizeof(RT) == 4) {
      const float* planes[4] = {R.ref32, R.gx32, R.gy32, R.gz32};
      return __ldg(planes[k] + p);
    } else {
      return __bfloat162float(__ldg(R.q16 + (p >> 2) * 16 + k * 4 + (p & 3)));
    }
  };

  float af = 0.0f;
  float ag[3][NDIM];
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int k = 0; k < NDIM; k++) ag[s][k] = 0.0f;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int row = row_begin + warp; row < row_end; row += kEvalWarps) {
    const RowDesc rd = R.rows[row];
    const int z = row / ny;
    const int y = row - z * ny;
    const bool flip = bidir && (y & 1);
    const long long rowoff = (long long)row * nx;
    for (int x = lane; x < nx; x += 32) {
      const VoxelModel vm = voxel_model(rd, x, nx, flip, bidir, dq);
      // the host geometry guarantees c0-1 <= di <= c0+2; the clamp only keeps the shared-memory
      // window in bounds
      const int wi = min(max(vm.di - cw, 0), kWin - 2);
      const float v = sample<NDIM, FT>(fr, job.fplane, job.fpitch, sD + wi * kDParamF4, vm.f, x, y, z, nx, ny, nz);
      const long long p = rowoff + x;
      const float t = refgrad(0, p);
      // include iff the interpolated value is positive: CPU rule px == 0 -> -1, then wimg >= 0
      // (FrameWarper.cpp:67, 16-25)
      const float e = (v > 0.0f) ? v - t : 0.0f;
      af = fmaf(e, e, af);
      if (!vm.last) {
        const float e1 = e * vm.f;           // weight of control r+1: Df
        const float e0 = e * (1.0f - vm.f);  // weight of control r:   1 - Df
        float gk[NDIM];
        gk[0] = refgrad(1, p);
        gk[1] = refgrad(2, p);
        if (NDIM == 3) gk[NDIM - 1] = refgrad(3, p);
        if (vm.r == c0) {
#pragma unroll
          for (int k = 0; k < NDIM; k++) {
            ag[0][k] = fmaf(gk[k], e0, ag[0][k]);
            ag[1][k] = fmaf(gk[k], e1, ag[1][k]);
          }
        } else {
#pragma unroll
          for (int k = 0; k < NDIM; k++) {
            ag[1][k] = fmaf(gk[k], e0, ag[1][k]);
            ag[2][k] = fmaf(gk[k], e1, ag[2][k]);
          }
        }
      }
    }
  }

  // FP32 butterfly across the warp, FP64 across warps (fixed order).
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    af += __shfl_xor_sync(0xffffffffu, af, o);
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
      for (int k = 0; k < NDIM; k++) ag[s][k] += __shfl_xor_sync(0xffffffffu, ag[s][k], o);
  }
  if (lane == 0) {
    sred[warp][0] = af;
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
      for (int k = 0; k < NDIM; k++) sred[warp][1 + s * NDIM + k] = ag[s][k];
  }
  __syncthreads();
  double* out = job.partials + (long long)tile * kPartialDoubles;
  if (threadIdx.x < 1 + 3 * NDIM) {
    double acc = 0.0;
    for (int w = 0; w < kEvalWarps; w++) acc += (double)sred[w][threadIdx.x];
    const int i = threadIdx.x;
    if (i == 0) {
      out[0] = acc;
    } else {
      const int s = (i - 1) / NDIM, k = (i - 1) % NDIM;
      out[2 + s * 3 + k] = acc;
    }
  } else if (threadIdx.x == 1 + 3 * NDIM) {
    out[1] = (double)c0;
    if (NDIM == 2) out[2 + 0 * 3 + 2] = out[2 + 1 * 3 + 2] = out[2 + 2 * 3 + 2] = 0.0;
  }
}

cudaError_t launch_eval4(const Job* jobs_dev, int n_jobs, int max_tiles, int n_dim, int frame_kind, bool ref_bf16,
                         int mb, cudaStream_t s);

cudaError_t launch_eval(const Job* jobs_dev, int n_jobs, int max_tiles, int n_dim, int frame_kind, bool ref_bf16,
                        cudaStream_t s, bool rows_multiple_of_4, int mb) {
  if (rows_multiple_of_4) return launch_eval4(jobs_dev, n_jobs, max_tiles, n_dim, frame_kind, ref_bf16, mb, s);
  const dim3 grid(max_tiles, n_jobs);
  return dispatch_cfg(n_dim, frame_kind, ref_bf16, [&](auto c) {
    using C = decltype(c);
    eval_kernel<C::nd, typename C::F, typename C::R><<<grid, kEvalThreads, 0, s>>>(jobs_dev);
    return cudaGetLastError();
  });
}

// ------------------------------------------------------------------ reductions -------------------

__global__ void __launch_bounds__(kSolveThreads) reduce_kernel(const Job* __restrict__ job) {
  const RefDev& R = *job->ref;
  reduce_partials(R, job->partials, job->result, job->result + 1);
}

cudaError_t launch_reduce(const Job* job_dev, const RefDev&, cudaStream_t s) {
  reduce_kernel<<<1, kSolveThreads, 0, s>>>(job_dev);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ warped image -----------------

template <int NDIM, typename FT>
__global__ void __launch_bounds__(256) warp_kernel(const RefDev* __restrict__ Rp, const FT* __restrict__ fr,
                                                   long long fplane, int fpitch, const float4* __restrict__ dparams,
                                                   float invalid_value, float* __restrict__ out) {
  const RefDev& R = *Rp;
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  extern __shared__ float4 sAll[];
  for (int i = threadIdx.x; i < R.nD * kDParamF4; i += blockDim.x) sAll[i] = dparams[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int row = blockIdx.x * nwarps + warp; row < R.n_rows; row += gridDim.x * nwarps) {
    const RowDesc rd = R.rows[row];
    const int z = row / ny;
    const int y = row - z * ny;
    const bool flip = R.bidir && (y & 1);
    for (int x = lane; x < nx; x += 32) {
      const VoxelModel vm = voxel_model(rd, x, nx, flip, R.bidir != 0, R.dq);
      const int di = min(max(vm.di, 0), R.nD - 2);
      float v = sample<NDIM, FT>(fr, fplane, fpitch, sAll + di * kDParamF4, vm.f, x, y, z, nx, ny, nz);
      if (v == 0.0f) v = invalid_value;
      out[(long long)row * nx + x] = v;
    }
  }
}

cudaError_t launch_warp(const RefDev* ref_dev, const RefDev& R, const void* frame, long long fplane, int fpitch,
                        int frame_kind, const float4* dparams, float invalid_value, float* out, cudaStream_t s) {
  int blocks = (R.n_rows + 7) / 8;
  if (blocks > 148 * 8) blocks = 148 * 8;
  const size_t smem = (size_t)R.nD * kDParamF4 * sizeof(float4);
  return dispatch_cfg(R.n_dim, frame_kind, false, [&](auto c) {
    using C = decltype(c);
    auto kern = warp_kernel<C::nd, typename C::F>;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    kern<<<blocks, 256, smem, s>>>(ref_dev, static_cast<const typename C::F*>(frame), fplane, fpitch, dparams,
                                   invalid_value, out);
    return cudaGetLastError();
  });
}

// ------------------------------------------------------------------ Hessian ----------------------

// Per tile and per storage-range slot s (range c0 + s): the 21 (3-D) or 10 (2-D) sums
//   A = sum v0 v0^T (upper), B = sum v1 v1^T (upper), C = sum v1 v0^T
// with v0 = float(grad * float(1 - Df)), v1 = float(grad * Df) and Df exact
// (FrameWarper.cpp:258-259, 319-342), over the voxels of the range that are not its last.
constexpr int kHessTerms = 21;

template <int NDIM>
__global__ void __launch_bounds__(256) hessian_tile_kernel(const RefDev* __restrict__ Rp, double pd, double ild,
                                                           double ifd, double stack, double* __restrict__ parts) {
  const RefDev& R = *Rp;
  const int tile = blockIdx.x;
  const int slot = blockIdx.y;
  const int nx = R.nx, ny = R.ny;
  const int row_begin = tile * R.tile_rows;
  const int row_end = min(row_begin + R.tile_rows, R.n_rows);
  const int c0 = R.tile_c0[tile];
  const double nDm1 = (double)(R.nD - 1);
  constexpr int NU = NDIM * (NDIM + 1) / 2;
  double acc[2 * NU + NDIM * NDIM];
#pragma unroll
  for (int i = 0; i < 2 * NU + NDIM * NDIM; i++) acc[i] = 0.0;
  for (int row = row_begin; row < row_end; row++) {
    const RowDesc rd = R.rows[row];
    const int z = row / ny;
    const int y = row - z * ny;
    const bool flip = R.bidir && (y & 1);
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const int r = R.bidir ? rd.r0 + (x >= rd.xr ? 1 : 0) : rd.di0 + (x >= rd.xdi ? 1 : 0);
      if (r - c0 != slot || x == rd.xlast) continue;
      const int xs = flip ? nx - 1 - x : x;
      // t = z*interframe + y*interline + x*pixel; q = t / stack * (nD - 1) (FrameWarper.cpp:258-259)
      const double t = __dadd_rn(__dadd_rn(__dmul_rn((double)z, ifd), __dmul_rn((double)y, ild)), __dmul_rn((double)xs, pd));
      const double q = __dmul_rn(__ddiv_rn(t, stack), nDm1);
      const float df = (float)(q - floor(q));
      const float w0 = __fsub_rn(1.0f, df);
      const long long p = (long long)row * nx + x;
      float g[NDIM];
      g[0] = R.gx32[p];
      g[1] = R.gy32[p];
      if (NDIM == 3) g[NDIM - 1] = R.gz32[p];
      float v0[NDIM], v1[NDIM];
#pragma unroll
      for (int k = 0; k < NDIM; k++) {
        v0[k] = __fmul_rn(g[k], w0);
        v1[k] = __fmul_rn(g[k], df);
      }
      int u = 0;
#pragma unroll
      for (int a = 0; a < NDIM; a++)
#pragma unroll
        for (int b = a; b < NDIM; b++, u++) {
          acc[u] += (double)__fmul_rn(v0[a], v0[b]);
          acc[NU + u] += (double)__fmul_rn(v1[a], v1[b]);
        }
#pragma unroll
      for (int a = 0; a < NDIM; a++)
#pragma unroll
        for (int b = 0; b < NDIM; b++) acc[2 * NU + a * NDIM + b] += (double)__fmul_rn(v1[a], v0[b]);
    }
  }
  __shared__ double sacc[256];
  double* out = parts + ((long long)tile * 2 + slot) * kHessTerms;
  for (int i = 0; i < 2 * NU + NDIM * NDIM; i++) {
    sacc[threadIdx.x] = acc[i];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sacc[threadIdx.x] += sacc[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = sacc[0];
    __syncthreads();
  }
}

// Hd[c] = sum_t A(t, c - c0_t) + B(t, c - 1 - c0_t);  Hl[c] = sum_t C(t, c - 1 - c0_t).
template <int NDIM>
__global__ void hessian_reduce_kernel(const RefDev* __restrict__ Rp, const double* __restrict__ parts,
                                      double* __restrict__ Hd, double* __restrict__ Hl) {
  const RefDev& R = *Rp;
  constexpr int NU = NDIM * (NDIM + 1) / 2;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R.nD) return;
  double d[NDIM * NDIM], l[NDIM * NDIM];
  for (int i = 0; i < NDIM * NDIM; i++) d[i] = l[i] = 0.0;
  const int t0 = max(0, R.ctrl_tiles[c].x), t1 = R.ctrl_tiles[c].y;
  for (int t = t0; t < t1; t++) {
    const int ct = R.tile_c0[t];
    for (int s = 0; s < 2; s++) {
      const double* pt = parts + ((long long)t * 2 + s) * kHessTerms;
      const int r = ct + s;
      if (r == c) {
        int u = 0;
        for (int a = 0; a < NDIM; a++)
          for (int b = a; b < NDIM; b++, u++) {
            d[a * NDIM + b] += pt[u];
            if (a != b) d[b * NDIM + a] += pt[u];
          }
      }
      if (r + 1 == c) {
        int u = 0;
        for (int a = 0; a < NDIM; a++)
          for (int b = a; b < NDIM; b++, u++) {
            d[a * NDIM + b] += pt[NU + u];
            if (a != b) d[b * NDIM + a] += pt[NU + u];
          }
        for (int a = 0; a < NDIM * NDIM; a++) l[a] += pt[2 * NU + a];
      }
    }
  }
  for (int i = 0; i < NDIM * NDIM; i++) {
    Hd[c * NDIM * NDIM + i] = d[i];
    Hl[c * NDIM * NDIM + i] = l[i];
  }
}

cudaError_t launch_hessian(const RefDev* ref_dev, const RefDev& R, const double* scan4, double* tile_parts, double* Hd,
                           double* Hl, cudaStream_t s) {
  dim3 grid(R.n_tiles, 2);
  if (R.n_dim == 3) {
    hessian_tile_kernel<3><<<grid, 256, 0, s>>>(ref_dev, scan4[0], scan4[1], scan4[2], scan4[3], tile_parts);
    hessian_reduce_kernel<3><<<(R.nD + 127) / 128, 128, 0, s>>>(ref_dev, tile_parts, Hd, Hl);
  } else {
    hessian_tile_kernel<2><<<grid, 256, 0, s>>>(ref_dev, scan4[0], scan4[1], scan4[2], scan4[3], tile_parts);
    hessian_reduce_kernel<2><<<(R.nD + 127) / 128, 128, 0, s>>>(ref_dev, tile_parts, Hd, Hl);
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------------ batched-solve bookkeeping ----

// One block of 1024 threads scans the job table in chunks: ballots give each warp's active / done
// counts, a shuffle scan the tile prefix inside a warp, and thread 0 the per-warp offsets.
__global__ void __launch_bounds__(1024) compact_kernel(const Job* __restrict__ jobs, int n, int* __restrict__ active,
                                                       int* __restrict__ n_active, int* __restrict__ tile_prefix,
                                                       int* __restrict__ busy, int* __restrict__ done_list,
                                                       int* __restrict__ n_done) {
  __shared__ int s_act[32], s_tiles[32], s_done[32];
  __shared__ int base_a, base_t, base_d, tot_a, tot_t, tot_d;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) {
    base_a = 0;
    base_t = 0;
    base_d = busy != nullptr ? *n_done : 0;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int c = 0; c < n; c += blockDim.x) {
    const int i = c + threadIdx.x;
    int phase = i < n ? jobs[i].state->phase : (int)kPhaseDone;
    if (phase == kPhaseWaitWarm) {
      // Resume a frame waiting for its warm start once the earlier frame's solution is written (by a
      // finished solve launch): the fourth starting point x + (warm - x).
      const Job& j = jobs[i];
      FrameState* S = j.state;
      if (*S->warm_seq == S->warm_need) {
        const RefDev& R = *j.ref;
        for (int q = 0; q < R.P; q++) j.p[q] = S->warm[q] - j.x[q];
        write_trial_dparams(j, R, 0, 1);
        S->phase = kPhaseStartLast;
        phase = kPhaseStartLast;
      }
    }
    const bool act = i < n && phase != kPhaseDone && phase != kPhaseWaitWarm;
    const bool fin = i < n && busy != nullptr && phase == kPhaseDone && busy[i] != 0;
    const int tiles = act ? jobs[i].ref->n_tiles * (phase == kPhaseStartPair ? 2 : 1) : 0;
    int incl = tiles;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const unsigned ma = __ballot_sync(0xffffffffu, act), md = __ballot_sync(0xffffffffu, fin);
    if (lane == 31) s_tiles[w] = incl;
    if (lane == 0) {
      s_act[w] = __popc(ma);
      s_done[w] = __popc(md);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int a = 0, t = 0, d = 0;
      for (int k = 0; k < nw; k++) {
        const int va = s_act[k], vt = s_tiles[k], vd = s_done[k];
        s_act[k] = a;
        s_tiles[k] = t;
        s_done[k] = d;
        a += va;
        t += vt;
        d += vd;
      }
      tot_a = a;
      tot_t = t;
      tot_d = d;
    }
    __syncthreads();
    if (act) {
      const int pos = base_a + s_act[w] + __popc(ma & lt);
      active[pos] = i;
      tile_prefix[pos] = base_t + s_tiles[w] + incl - tiles;
    }
    if (fin) {
      done_list[base_d + s_done[w] + __popc(md & lt)] = i;
      busy[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      base_a += tot_a;
      base_t += tot_t;
      base_d += tot_d;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *n_active = base_a;
    tile_prefix[base_a] = base_t;
    if (busy != nullptr) *n_done = base_d;
  }
}

cudaError_t launch_compact(const Job* jobs_dev, int n_jobs, int* active, int* n_active, int* tile_prefix, int* busy,
                           int* done_list, int* n_done, cudaStream_t s) {
  compact_kernel<<<1, 1024, 0, s>>>(jobs_dev, n_jobs, active, n_active, tile_prefix, busy, done_list, n_done);
  return cudaGetLastError();
}

// Last node of the body of a batched solve's device-side loop: counts the rounds and repeats the body
// while a frame is still active and fewer than max_rounds rounds ran.
__global__ void loop_control_kernel(cudaGraphConditionalHandle h, const int* __restrict__ n_active,
                                    int* __restrict__ rounds, int max_rounds) {
  const int r = *rounds + 1;
  *rounds = r;
  cudaGraphSetConditional(h, *n_active > 0 && r < max_rounds ? 1u : 0u);
}

cudaError_t launch_loop_control(cudaGraphConditionalHandle h, const int* n_active, int* rounds, int max_rounds,
                                cudaStream_t s) {
  loop_control_kernel<<<1, 1, 0, s>>>(h, n_active, rounds, max_rounds);
  return cudaGetLastError();
}

// Zero start of a batched solve (the host-side init of the single-frame driver, on the device).
__global__ void activate_kernel(const Job* __restrict__ jobs, const Activation* __restrict__ recs, int* busy) {
  const Activation r = recs[blockIdx.x];
  const Job& j = jobs[r.job];
  const RefDev& R = *j.ref;
  for (int i = threadIdx.x; i < R.P; i += blockDim.x) {
    j.x[i] = 0.0;
    j.g[i] = 0.0;
    j.p[i] = 0.0;
    j.gt[i] = 0.0;
  }
  for (int i = threadIdx.x; i < R.nD * kDParamF4; i += blockDim.x) j.dparams[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  double rigid[3];
  bool nonzero = false;
  for (int c = 0; c < 3; c++) {
    rigid[c] = (c < R.n_dim) ? r.rigid[c] : 0.0;
    nonzero = nonzero || rigid[c] != 0.0;
  }
  const bool pair = r.pair != 0 && nonzero;
  if (pair) write_const_dparams(j.dparams2, R.nD, R.n_dim, rigid, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) {
    FrameState S{};
    S.phase = pair ? kPhaseStartPair : kPhaseStartZero;
    S.max_iter = r.max_iter > 0 ? r.max_iter : 100;
    S.warm = r.warm;
    S.warm_seq = r.warm_seq;
    S.warm_need = r.warm_need;
    S.seq = r.seq;
    S.use_warm = (r.use_warm != 0 && r.warm != nullptr && r.warm_seq != nullptr) ? 1 : 0;
    for (int c = 0; c < 3; c++) S.rigid[c] = r.rigid[c];
    if (R.n_dim == 2) S.rigid[2] = 0.0;
    *j.state = S;
    busy[r.job] = 1;
  }
}

// Start of the aligner's batched solve straight from the phase-correlation peaks in device memory, so
// that the host need not read them first: job i takes peak i (flat index of the correlation surface
// of a cnz x cny x cnx volume), unravels and wraps it like unravel_shift (VolumePhaseCorrelator.cpp:
// 94-103), scales x and y by the binning (FrameWarpAligner.cpp:186-188) and sets the zero start, or the
// paired start when `pair` and the shift is not zero.
__global__ void activate_peaks_kernel(const Job* __restrict__ jobs, const long long* __restrict__ peaks, int cnx,
                                      int cny, int cnz, int binning, int max_iter, int pair) {
  const Job& j = jobs[blockIdx.x];
  const RefDev& R = *j.ref;
  const long long idx = peaks[blockIdx.x];
  long long x = idx % cnx, y = (idx / cnx) % cny, z = idx / ((long long)cnx * cny);
  if (x > cnx / 2) x -= cnx;
  if (y > cny / 2) y -= cny;
  if (z > cnz / 2) z -= cnz;
  double rigid[3] = {(double)x * binning, (double)y * binning, R.n_dim == 3 ? (double)z : 0.0};
  bool nonzero = false;
  for (int c = 0; c < R.n_dim; c++) nonzero = nonzero || rigid[c] != 0.0;
  const bool paired = pair != 0 && nonzero;
  for (int i = threadIdx.x; i < R.P; i += blockDim.x) {
    j.x[i] = 0.0;
    j.g[i] = 0.0;
    j.p[i] = 0.0;
    j.gt[i] = 0.0;
  }
  for (int i = threadIdx.x; i < R.nD * kDParamF4; i += blockDim.x) j.dparams[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (paired) write_const_dparams(j.dparams2, R.nD, R.n_dim, rigid, threadIdx.x, blockDim.x);
  if (threadIdx.x == 0) {
    FrameState S{};
    S.phase = paired ? kPhaseStartPair : kPhaseStartZero;
    S.max_iter = max_iter > 0 ? max_iter : 100;
    for (int c = 0; c < 3; c++) S.rigid[c] = rigid[c];
    *j.state = S;
  }
}

cudaError_t launch_activate_peaks(const Job* jobs_dev, int n, const long long* peaks, int cnx, int cny, int cnz,
                                  int binning, int max_iter, bool pair, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  activate_peaks_kernel<<<n, 128, 0, s>>>(jobs_dev, peaks, cnx, cny, cnz, binning, max_iter, pair ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_activate(const Job* jobs_dev, const Activation* recs, int n, int* busy, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  activate_kernel<<<n, 128, 0, s>>>(jobs_dev, recs, busy);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ smoothStack ------------------

// FrameWarpAligner::smoothStack (FrameWarpAligner.cpp:46-64): per plane, cv::GaussianBlur with sigma
// along x and 1 along y, BORDER_REFLECT_101, float arithmetic (products and sums rounded one by one):
// a row pass summing taps in kernel order, then a column pass in the symmetric form.
__device__ __forceinline__ int reflect101(int p, int n) {
  if (n == 1) return 0;
  while (p < 0 || p >= n) {
    if (p < 0) p = -p;
    if (p >= n) p = 2 * n - 2 - p;
  }
  return p;
}

__global__ void smooth_rows_kernel(const void* __restrict__ in, int in_t, int ny, int nx, long long n,
                                   const float* __restrict__ k, int nk, float* __restrict__ out) {
  const int r = nk / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long row = i - x;
    float s = __fmul_rn(k[0], load_any(in, in_t, row + reflect101(x - r, nx)));
    for (int t = 1; t < nk; t++) s = __fadd_rn(s, __fmul_rn(k[t], load_any(in, in_t, row + reflect101(x + t - r, nx))));
    out[i] = s;
  }
}

__global__ void smooth_cols_kernel(const float* __restrict__ in, int ny, int nx, long long n,
                                   const float* __restrict__ k, int nk, float* __restrict__ out) {
  const int r = nk / 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx);
    const long long py = i / nx;
    const int y = (int)(py % ny);
    const long long plane = (py - y) * nx;
    float s = __fmul_rn(k[r], in[i]);
    for (int t = 1; t <= r; t++) {
      const float a = in[plane + (long long)reflect101(y - t, ny) * nx + x];
      const float b = in[plane + (long long)reflect101(y + t, ny) * nx + x];
      s = __fadd_rn(s, __fmul_rn(k[r + t], __fadd_rn(a, b)));
    }
    out[i] = s;
  }
}

cudaError_t launch_smooth(const void* in, fa_dtype in_type, int nz, int ny, int nx, const float* kx, int nkx,
                          const float* ky, int nky, float* tmp, float* out, cudaStream_t s) {
  const long long n = (long long)nz * ny * nx;
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  smooth_rows_kernel<<<(int)blocks, 256, 0, s>>>(in, (int)in_type, ny, nx, n, kx, nkx, tmp);
  smooth_cols_kernel<<<(int)blocks, 256, 0, s>>>(tmp, ny, nx, n, ky, nky, out);
  return cudaGetLastError();
}

}  // namespace fa
