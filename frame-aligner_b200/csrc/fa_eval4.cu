// fa_eval4.cu -- the fused warp + error + J^T e pass with four consecutive voxels per lane
// (image rows whose length is a multiple of 4).
//
// Same arithmetic contract as eval_kernel (FrameWarper.cpp:4-69,147-176 restated on the device):
// per voxel the scan-time interval and fraction, the displacement d = D[i] + f (D[i+1] - D[i]),
// the zero-padded trilinear sample of the frame at x + d, the masked error, its square, and the
// two control points' J^T e contributions (1 - f) grad e and f grad e.
//
// Why four voxels per lane: along an image row the sample position advances by one voxel plus a
// displacement that changes by ~1e-5 px per voxel, so four neighbours almost always share the
// integer tap offset. They then need only five frame values per tap row, fetched as one aligned
// 8-element window (two 64-bit loads for FP16, two 128-bit loads for FP32) and shifted into place,
// instead of eight gathers per voxel; the reference and gradient values come with two 128-bit
// loads (BF16 groups) or one per plane (FP32). Row segments of 128 voxels that straddle an interval
// boundary, a range end, a change of the integer offset or the volume edge take the per-voxel path.
#include <type_traits>

#include "fa_device.cuh"

namespace fa {

namespace {

// The reference and gradient values of four consecutive voxels starting at a multiple of 4: four
// FP32 planes, or the BF16 groups of RefDev::q16 (two 16-byte loads for all four quantities).
template <typename RT>
struct RefGradSrc;
template <>
struct RefGradSrc<float> {
  const float* r;
  const float* g[3];
  __device__ explicit RefGradSrc(const RefDev& R) : r(R.ref32), g{R.gx32, R.gy32, R.gz32} {}
  // the loads (issued early), then the values
  struct Raw {
    float4 t, g[3];
  };
  template <int NDIM>
  __device__ __forceinline__ Raw load_raw(long long p0) const {
    Raw w;
    w.t = __ldg(reinterpret_cast<const float4*>(r + p0));
#pragma unroll
    for (int k = 0; k < NDIM; k++) w.g[k] = __ldg(reinterpret_cast<const float4*>(g[k] + p0));
    return w;
  }
  template <int NDIM>
  __device__ __forceinline__ static void unpack(const Raw& w, float* t4, float (*g4)[4]) {
    auto put = [](float4 a, float* v) {
      v[0] = a.x;
      v[1] = a.y;
      v[2] = a.z;
      v[3] = a.w;
    };
    put(w.t, t4);
#pragma unroll
    for (int k = 0; k < NDIM; k++) put(w.g[k], g4[k]);
  }
  // one voxel's reference and gradient values
  template <int NDIM>
  __device__ __forceinline__ void load1(long long p, float& t, float* g1) const {
    t = __ldg(r + p);
#pragma unroll
    for (int k = 0; k < NDIM; k++) g1[k] = __ldg(g[k] + p);
  }
};
template <>
struct RefGradSrc<__nv_bfloat16> {
  const __nv_bfloat16* q;
  __device__ explicit RefGradSrc(const RefDev& R) : q(R.q16) {}
  // the loads (issued early), then the values
  struct Raw {
    uint4 a, c;
  };
  template <int NDIM>
  __device__ __forceinline__ Raw load_raw(long long p0) const {
    const uint4* b = reinterpret_cast<const uint4*>(q + (p0 >> 2) * 16);
    return Raw{__ldg(b), __ldg(b + 1)};
  }
  template <int NDIM>
  __device__ __forceinline__ static void unpack(const Raw& w, float* t4, float (*g4)[4]) {
    auto put = [](unsigned lo, unsigned hi, float* v) {
      v[0] = __uint_as_float(lo << 16);
      v[1] = __uint_as_float(lo & 0xffff0000u);
      v[2] = __uint_as_float(hi << 16);
      v[3] = __uint_as_float(hi & 0xffff0000u);
    };
    put(w.a.x, w.a.y, t4);
    put(w.a.z, w.a.w, g4[0]);
    put(w.c.x, w.c.y, g4[1]);
    if (NDIM == 3) put(w.c.z, w.c.w, g4[NDIM == 3 ? 2 : 0]);
  }
  // one voxel's reference and gradient values (element p & 3 of each quantity's four in the group)
  template <int NDIM>
  __device__ __forceinline__ void load1(long long p, float& t, float* g1) const {
    const __nv_bfloat16* b = q + (p >> 2) * 16 + (p & 3);
    t = __bfloat162float(__ldg(b));
#pragma unroll
    for (int k = 0; k < NDIM; k++) g1[k] = __bfloat162float(__ldg(b + 4 * (k + 1)));
  }
};

}  // namespace

// The raw words of one lane's aligned 8-element frame window of one tap row (16 bytes for 16-bit
// samples, 32 for FP32), loaded before they are decoded so that a segment's loads can be issued
// while the previous segment is computed.
template <typename FT>
struct WinRaw {
  uint2 lo, hi;
};
template <>
struct WinRaw<float> {
  float4 lo, hi;
};
template <typename FT>
__device__ __forceinline__ WinRaw<FT> load_win(const FT* p) {
  if constexpr (std::is_same<FT, float>::value)
    return WinRaw<FT>{__ldg(reinterpret_cast<const float4*>(p)), __ldg(reinterpret_cast<const float4*>(p + 4))};
  else
    return WinRaw<FT>{__ldg(reinterpret_cast<const uint2*>(p)), __ldg(reinterpret_cast<const uint2*>(p + 4))};
}

// Frame values v[k] = window[S + k], k = 0..4, for an alignment S that is the same for every lane of
// the warp (known at compile time: no shifts or selects).
template <int S>
__device__ __forceinline__ void window5s(const WinRaw<RawU16>& r, float* v) {
  const unsigned w[4] = {r.lo.x, r.lo.y, r.hi.x, r.hi.y};
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int e = S + k;
    v[k] = __uint_as_float(__byte_perm(w[e >> 1], 0x4B000000u, (e & 1) ? 0x7632 : 0x7610)) - 8388608.0f;
  }
}
template <int S>
__device__ __forceinline__ void window5s(const WinRaw<__half>& r, float* v) {
  const unsigned w[4] = {r.lo.x, r.lo.y, r.hi.x, r.hi.y};
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const int e = S + k;
    const unsigned short h = (unsigned short)((e & 1) ? (w[e >> 1] >> 16) : (w[e >> 1] & 0xffffu));
    v[k] = __half2float(__ushort_as_half(h));
  }
}
template <int S>
__device__ __forceinline__ void window5s(const WinRaw<float>& r, float* v) {
  const float w[8] = {r.lo.x, r.lo.y, r.lo.z, r.lo.w, r.hi.x, r.hi.y, r.hi.z, r.hi.w};
#pragma unroll
  for (int k = 0; k < 5; k++) v[k] = w[S + k];
}

// Everything one lane loads for its four voxels of a uniform segment: the reference / gradient
// group and the windows of the tap rows (y, z), (y+1, z), (y, z+1), (y+1, z+1).
template <int NDIM, typename FT, typename RT>
struct SegLoad {
  typename RefGradSrc<RT>::Raw rg;
  WinRaw<FT> w[NDIM == 3 ? 4 : 2];
};

// Four voxels of a lane in a uniform row segment (see eval4_tile), from the raw windows of its tap
// rows (y, z), (y+1, z), (y, z+1), (y+1, z+1); weights of voxel j are w + j * s per axis, its
// control-point fraction fl + j * fs.
template <int NDIM, int S, typename FT>
__device__ __forceinline__ void uniform4(const WinRaw<FT>* win, const float* t4, const float (*g4)[4], float wxl,
                                         float sx, float wyl, float sy, float wzl, float sz, float fl, float fs,
                                         float& af, float* acc0, float* acc1) {
  float v[NDIM == 3 ? 4 : 2][5];
#pragma unroll
  for (int r = 0; r < (NDIM == 3 ? 4 : 2); r++) window5s<S>(win[r], v[r]);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const float wx = j ? fmaf((float)j, sx, wxl) : wxl;
    const float wy = j ? fmaf((float)j, sy, wyl) : wyl;
    const float c00 = fmaf(wx, v[0][j + 1] - v[0][j], v[0][j]);
    const float c01 = fmaf(wx, v[1][j + 1] - v[1][j], v[1][j]);
    float val = fmaf(wy, c01 - c00, c00);
    if (NDIM == 3) {
      const float wz = j ? fmaf((float)j, sz, wzl) : wzl;
      const float c10 = fmaf(wx, v[NDIM == 3 ? 2 : 0][j + 1] - v[NDIM == 3 ? 2 : 0][j], v[NDIM == 3 ? 2 : 0][j]);
      const float c11 = fmaf(wx, v[NDIM == 3 ? 3 : 1][j + 1] - v[NDIM == 3 ? 3 : 1][j], v[NDIM == 3 ? 3 : 1][j]);
      const float c1 = fmaf(wy, c11 - c10, c10);
      val = fmaf(wz, c1 - val, val);
    }
    const float e = (val > 0.0f) ? val - t4[j] : 0.0f;
    af = fmaf(e, e, af);
    const float fj = j ? fmaf((float)j, fs, fl) : fl;
    const float e1 = e * fj;
    const float e0 = e - e1;
#pragma unroll
    for (int k = 0; k < NDIM; k++) {
      acc0[k] = fmaf(g4[k][j], e0, acc0[k]);
      acc1[k] = fmaf(g4[k][j], e1, acc1[k]);
    }
  }
}

// Per-lane path of eval4_tile for the four voxels x0 .. x0+3 of one image row (row descriptor rd),
// voxel by voxel: interval, fraction and range per voxel, eight zero-padded taps, and the J^T e
// terms added straight into the tile's control-point sums ag (controls c0 .. c0+2). It runs for the
// few segments that are not uniform, so it is written for few live registers rather than speed: the
// whole pass is compiled to the register budget of its busiest point.
template <int NDIM, typename FT, typename RT>
__device__ __forceinline__ void lane_item(const FT* __restrict__ fr, long long plane, int pitch,
                                          const RefGradSrc<RT> src, const RowDesc rd, int x0, int row_here, int nx,
                                          int ny, int nz, bool bidir, float dq, const float4* sD, int cw, int c0,
                                          float& af, float* ag) {
  const bool flip = bidir && (rd.y & 1);
  const long long p0 = (long long)row_here * nx + x0;
#pragma unroll 1
  for (int j = 0; j < 4; j++) {
    const int x = x0 + j;
    const VoxelModel vm = voxel_model(rd, x, nx, flip, bidir, dq);
    const int wi = min(max(vm.di - cw, 0), kWin - 2);
    const float val = sample<NDIM, FT>(fr, plane, pitch, sD + wi * kDParamF4, vm.f, x, rd.y, rd.z, nx, ny, nz);
    float t, g[NDIM];
    src.template load1<NDIM>(p0 + j, t, g);
    const float e = (val > 0.0f) ? val - t : 0.0f;
    af = fmaf(e, e, af);
    if (!vm.last) {
      const float e1 = e * vm.f;
      const float e0 = e * (1.0f - vm.f);
      const bool first = vm.r == c0;  // controls c0, c0+1; else c0+1, c0+2
#pragma unroll
      for (int k = 0; k < NDIM; k++) {
        const float a0 = g[k] * e0, a1 = g[k] * e1;
        ag[(0 * 3 + k) * 32] += first ? a0 : 0.0f;
        ag[(1 * 3 + k) * 32] += first ? a1 : a0;
        ag[(2 * 3 + k) * 32] += first ? 0.0f : a1;
      }
    }
  }
}

// A row segment's parameters, computed by one lane for the whole warp (see eval4_tile).
struct SegParams {
  float w0x, w0y, w0z, f0;  // sample weights and control-point fraction of the segment's first voxel
  float sx, sy, sz, fs;     // their change per voxel along the row
  long long win;            // frame offset of lane 0's window (tap row y, plane z; multiple of 4 in x)
  int p0;                   // reference / gradient offset of the segment's first voxel
  int meta;                 // bit 0: uniform; bits 1-2: window alignment; bits 3..: storage range
  int xa;                   // x of the segment's first voxel
  int row;                  // image row (z * ny + y)
};
constexpr int kSegBatch = 32;  // segments classified per round, one per lane
constexpr int kSegLen = 128;   // voxels per segment: four per lane

// One tile of one frame, processed by one warp on its own: its control-point window sD (the warp's
// slice of shared memory), its row segments, and its partial sums. No CTA barrier is involved, so
// the warps of a CTA drift apart and hide each other's load latency.
//
// A row segment is kSegLen consecutive voxels of an image row, four per lane.
// Almost every segment is uniform: its voxels share one displacement interval and one storage range,
// contain no range end, and their sample positions x + d(x) share one integer offset per axis,
// because the displacement changes by ~1e-5 px per voxel along a row. Whether it is, and its weights, slopes and window
// offsets, follow from the row descriptor and the segment's two ends (the position is monotone in x
// within an interval). The warp first classifies 32 segments at once, one per lane, into shared
// memory, then walks them: a uniform segment needs no per-lane interval, range or offset logic, its
// frame windows share one compile-time alignment, and its J^T e terms go to one pair of running sums
// that are added to the tile's control points only when the range changes. Other segments take the
// per-lane path (lane_item), which handles every case voxel by voxel where needed.
//
// PIPE: the uniform walk is software-pipelined, the loads of the next uniform segment issued before
// the current one is computed (two segments' loads live at once: only with 16-bit storage and the
// largest register budget, 2 CTAs per SM); without it each segment's loads are followed by its
// arithmetic.
template <int NDIM, typename FT, typename RT, bool PIPE>
__device__ __forceinline__ void eval4_tile(const Job& job, const RefDev& R, const int tile, float4* sD,
                                           SegParams* sp, float* sg, const float4* __restrict__ dparams,
                                           double* __restrict__ partials) {
  const int nx = R.nx, ny = R.ny, nz = R.nz;
  const int row_begin = tile * R.tile_rows;
  const int row_end = min(row_begin + R.tile_rows, R.n_rows);
  const int c0 = R.tile_c0[tile];
  const int cw = max(c0 - 1, 0);
  const bool bidir = R.bidir != 0;
  const float dq = R.dq;
  const int lane = threadIdx.x & 31;

  __syncwarp();  // the previous tile's readers of sD and sp are done
  if (lane < kWin * kDParamF4) {
    const int k = cw + lane / kDParamF4;
    sD[lane] = (k < R.nD) ? dparams[k * kDParamF4 + lane % kDParamF4] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  __syncwarp();

  const FT* __restrict__ fr = static_cast<const FT*>(job.frame);
  const RefGradSrc<RT> src(R);

  float af = 0.0f;
  // the lane's J^T e sums of controls c0 .. c0+2, entry (s * 3 + k) * 32 (shared memory: they change
  // only when a range ends and on the per-lane path)
  float* ag = sg + lane;
#pragma unroll
  for (int i = 0; i < 9; i++) ag[i * 32] = 0.0f;
  // running J^T e sums of uniform segments, for controls ur and ur + 1 (ur: their storage range)
  float ua0[NDIM], ua1[NDIM];
#pragma unroll
  for (int k = 0; k < NDIM; k++) ua0[k] = ua1[k] = 0.0f;
  int ur = -1;
  auto flush_uniform = [&]() {
    if (ur == c0) {
#pragma unroll
      for (int k = 0; k < NDIM; k++) {
        ag[(0 * 3 + k) * 32] += ua0[k];
        ag[(1 * 3 + k) * 32] += ua1[k];
      }
    } else if (ur >= 0) {
#pragma unroll
      for (int k = 0; k < NDIM; k++) {
        ag[(1 * 3 + k) * 32] += ua0[k];
        ag[(2 * 3 + k) * 32] += ua1[k];
      }
    }
#pragma unroll
    for (int k = 0; k < NDIM; k++) ua0[k] = ua1[k] = 0.0f;
  };
  const float lane_u = (float)(lane * 4);  // x - (segment start) of the lane's first voxel

  // segments of the tile's rows
  const int segs = (nx + kSegLen - 1) / kSegLen;
  const int n_items = (row_end - row_begin) * segs;
  const long long plane = job.fplane;
  const int pitch = job.fpitch;
  const bool padded = job.fpad != 0;
  for (int base = 0; base < n_items; base += kSegBatch) {
    // ---- classify segments base .. base + 31, segment base + lane by this lane ----
    if (base + lane < n_items) {
      const int it = base + lane;
      const int row = row_begin + it / segs;
      const int xa = (it - (row - row_begin) * segs) * kSegLen;
      const RowDesc rd = R.rows[row];
      const bool flip = bidir && (rd.y & 1);
      const int xb = min(xa + kSegLen - 1, nx - 1);
      const int xsa = flip ? nx - 1 - xa : xa, xsb = flip ? nx - 1 - xb : xb;
      const int dia = rd.di0 + (xsa >= rd.xdi ? 1 : 0);
      const int dib = rd.di0 + (xsb >= rd.xdi ? 1 : 0);
      const int ra = bidir ? rd.r0 + (xa >= rd.xr ? 1 : 0) : dia;
      const int rb = bidir ? rd.r0 + (xb >= rd.xr ? 1 : 0) : dib;
      bool uni = dia == dib && ra == rb && (rd.xlast < xa || rd.xlast > xb);
      const float4* Pa = sD + min(max(dia - cw, 0), kWin - 2) * kDParamF4;
      const float fsa = fmaf((float)xsa, dq, rd.qbase) - (float)(dia - rd.di0);
      const float fs = flip ? -dq : dq;
      const float span = (float)(xb - xa);
      const float4 na = Pa[0], pha = Pa[1], dda = Pa[2];
      const float sx = fs * dda.x, sy = fs * dda.y, sz = NDIM == 3 ? fs * dda.z : 0.0f;
      const float tax = fmaf(fsa, dda.x, pha.x), tay = fmaf(fsa, dda.y, pha.y);
      const float flx = floorf(tax), fly = floorf(tay);
      uni = uni && floorf(fmaf(span, sx, tax)) == flx && floorf(fmaf(span, sy, tay)) == fly;
      float taz = 0.f, flz = 0.f;
      if (NDIM == 3) {
        taz = fmaf(fsa, dda.z, pha.z);
        flz = floorf(taz);
        uni = uni && floorf(fmaf(span, sz, taz)) == flz;
      }
      const int ox = (int)na.x + (int)flx;
      const int iy = rd.y + (int)na.y + (int)fly;
      const int iz = NDIM == 3 ? rd.z + (int)na.z + (int)flz : 0;
      const int ab = ox & ~3;                   // window start relative to x0 (multiple of 4)
      const int x_last = min(xa + kSegLen - 4, nx - 4);  // first voxel of the segment's last active lane
      int cy, cz;
      if (padded) {
        // windows inside the row's zero halo; tap rows / planes wholly outside read halo zeros
        uni = uni && xa + ab >= -kHaloX && x_last + ab + 7 <= nx - 1 + kHaloX;
        cy = min(max(iy, -kHaloY), ny + kHaloY - 2);
        cz = NDIM == 3 ? min(max(iz, -kHaloZ), nz + kHaloZ - 2) : 0;
      } else {
        uni = uni && xa + ab >= 0 && x_last + ab + 7 <= nx - 1 && iy >= 0 && iy + 1 <= ny - 1 &&
              (NDIM == 2 || (iz >= 0 && iz + 1 <= nz - 1));
        cy = iy;
        cz = iz;
      }
      SegParams q;
      q.w0x = tax - flx;
      q.w0y = tay - fly;
      q.w0z = taz - flz;
      q.f0 = fsa;
      q.sx = sx;
      q.sy = sy;
      q.sz = sz;
      q.fs = fs;
      q.win = (long long)cz * plane + (long long)cy * pitch + xa + ab;
      q.p0 = row * nx + xa;
      q.xa = xa;
      q.row = row;
      q.meta = (uni ? 1 : 0) | ((ox & 3) << 1) | (ra << 3);
      sp[lane] = q;
    }
    __syncwarp();
    // ---- walk the uniform ones, in order ----
    const int cnt = min(kSegBatch, n_items - base);
    unsigned umask = __ballot_sync(0xffffffffu, lane < cnt && (sp[lane].meta & 1) != 0);
    // the loads of one lane for segment P (lanes past the row end load nothing)
    auto seg_load = [&](const SegParams& P, SegLoad<NDIM, FT, RT>& L) {
      if (P.xa + lane * 4 < nx) {
        L.rg = src.template load_raw<NDIM>(P.p0 + lane * 4);
        const FT* wp = fr + (P.win + lane * 4);
        L.w[0] = load_win(wp);
        L.w[1] = load_win(wp + pitch);
        if (NDIM == 3) {
          L.w[NDIM == 3 ? 2 : 0] = load_win(wp + plane);
          L.w[NDIM == 3 ? 3 : 1] = load_win(wp + plane + pitch);
        }
      }
    };
    // a segment's range: the running sums are flushed when it changes
    auto seg_range = [&](const SegParams& P) {
      const int ra = P.meta >> 3;
      if (ra != ur) {
        flush_uniform();
        ur = ra;
      }
    };
    // the arithmetic of segment P on loaded values (lanes inside the row)
    auto seg_math = [&](const SegParams& P, const SegLoad<NDIM, FT, RT>& L) {
      {
        float t4[4], g4[NDIM][4];
        RefGradSrc<RT>::template unpack<NDIM>(L.rg, t4, g4);
        const float wxl = fmaf(lane_u, P.sx, P.w0x);
        const float wyl = fmaf(lane_u, P.sy, P.w0y);
        const float wzl = NDIM == 3 ? fmaf(lane_u, P.sz, P.w0z) : 0.0f;
        const float fl = fmaf(lane_u, P.fs, P.f0);
        switch ((P.meta >> 1) & 3) {
          case 0:
            uniform4<NDIM, 0, FT>(L.w, t4, g4, wxl, P.sx, wyl, P.sy, wzl, P.sz, fl, P.fs, af, ua0, ua1);
            break;
          case 1:
            uniform4<NDIM, 1, FT>(L.w, t4, g4, wxl, P.sx, wyl, P.sy, wzl, P.sz, fl, P.fs, af, ua0, ua1);
            break;
          case 2:
            uniform4<NDIM, 2, FT>(L.w, t4, g4, wxl, P.sx, wyl, P.sy, wzl, P.sz, fl, P.fs, af, ua0, ua1);
            break;
          default:
            uniform4<NDIM, 3, FT>(L.w, t4, g4, wxl, P.sx, wyl, P.sy, wzl, P.sz, fl, P.fs, af, ua0, ua1);
            break;
        }
      }
    };
    auto seg_compute = [&](const SegParams& P, const SegLoad<NDIM, FT, RT>& L) {
      seg_range(P);
      if (P.xa + lane * 4 < nx) seg_math(P, L);
      __syncwarp();  // lanes past the row end rejoin here
    };
    // next uniform segment of the batch (-1: none), taken off the mask
    auto next_uniform = [&]() {
      if (umask == 0u) return -1;
      const int q = __ffs(umask) - 1;
      umask &= umask - 1u;
      return q;
    };
    if constexpr (PIPE) {
      // two load buffers, alternating: A holds segment q while B receives the one after it
      SegLoad<NDIM, FT, RT> A, B;
      int q = next_uniform();
      if (q >= 0) seg_load(sp[q], A);
      while (q >= 0) {
        int qn = next_uniform();
        if (qn >= 0) seg_load(sp[qn], B);
        seg_compute(sp[q], A);
        q = qn;
        if (q < 0) break;
        qn = next_uniform();
        if (qn >= 0) seg_load(sp[qn], A);
        seg_compute(sp[q], B);
        q = qn;
      }
    } else {
      for (int q = next_uniform(); q >= 0; q = next_uniform()) {
        const SegParams& P = sp[q];
        seg_range(P);
        if (P.xa + lane * 4 < nx) {
          SegLoad<NDIM, FT, RT> L;
          seg_load(P, L);
          seg_math(P, L);
        }
        __syncwarp();  // lanes past the row end rejoin here
      }
    }
    // the batch's other segments, lane by lane (after the uniform walk, so that its registers are
    // free for the per-lane path)
    for (int q = 0; q < cnt; q++) {
      if (sp[q].meta & 1) continue;
      const int x0 = sp[q].xa + lane * 4;
      if (x0 < nx) {
        const int row = sp[q].row;
        lane_item<NDIM, FT, RT>(fr, plane, pitch, src, R.rows[row], x0, row, nx, ny, nz, bidir, dq, sD, cw, c0, af,
                                ag);
      }
      // Explicit reconvergence point: the per-lane branches above must not leave the warp split
      // into groups that then run the rest of the loop one after the other.
      __syncwarp();
    }
    __syncwarp();  // every lane is done reading this batch's parameters
  }
  flush_uniform();
  float g9[3][NDIM];
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int k = 0; k < NDIM; k++) g9[s][k] = ag[(s * 3 + k) * 32];
  __syncwarp();  // sg is free for the next tile
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    af += __shfl_xor_sync(0xffffffffu, af, o);
#pragma unroll
    for (int s = 0; s < 3; s++)
#pragma unroll
      for (int k = 0; k < NDIM; k++) g9[s][k] += __shfl_xor_sync(0xffffffffu, g9[s][k], o);
  }
  // Lane i < 11 writes entry i of the tile's partial sums [f, c0, g(3 x 3)] (every lane holds the
  // totals; the value is picked with selects so that the warp does not branch).
  float pick = af;
#pragma unroll
  for (int s = 0; s < 3; s++)
#pragma unroll
    for (int k = 0; k < 3; k++) pick = (lane == 2 + s * 3 + k) ? (k < NDIM ? g9[s][k < NDIM ? k : 0] : 0.0f) : pick;
  double* out = partials + (long long)tile * kPartialDoubles;
  if (lane < 11) out[lane] = lane == 1 ? (double)c0 : (double)pick;
  __syncwarp();
}

// Whether eval4_tile pipelines its uniform walk for this storage and register budget.
template <typename FT, typename RT, int MB>
constexpr bool kPipe = MB == 2 && sizeof(FT) == 2 && sizeof(RT) == 2;

// One grid per launch: CTA x of job y covers tiles 8x .. 8x+7, one per warp.
template <int NDIM, typename FT, typename RT, int MB>
__global__ void __launch_bounds__(kEvalThreads, MB) eval4_kernel(const Job* __restrict__ jobs) {
  __shared__ float4 sD[kEvalWarps][kWin * kDParamF4];
  __shared__ SegParams sp[kEvalWarps][kSegBatch];
  __shared__ float sg[kEvalWarps][9 * 32];
  const Job& job = jobs[blockIdx.y];
  if (job.state != nullptr && (job.state->phase == kPhaseDone || job.state->phase == kPhaseWaitWarm)) return;
  const RefDev& R = *job.ref;
  const int warp = threadIdx.x >> 5;
  const int tile = blockIdx.x * kEvalWarps + warp;
  if (tile >= R.n_tiles) return;
  eval4_tile<NDIM, FT, RT, kPipe<FT, RT, MB>>(job, R, tile, sD[warp], sp[warp], sg[warp], job.dparams, job.partials);
}

// Persistent form for batched solves: the grid's warps walk the (active frame, tile) items of the
// compacted active list, item = tile_prefix[a] + tile, so frames that have converged cost nothing and
// frames of different sizes share the launch. Each warp's items increase, so its frame index only
// moves forward (binary search over the remaining prefix).
template <int NDIM, typename FT, typename RT, int MB>
__global__ void __launch_bounds__(kEvalThreads, MB) eval4_active_kernel(const Job* __restrict__ jobs,
                                                                     const int* __restrict__ active,
                                                                     const int* __restrict__ n_active,
                                                                     const int* __restrict__ tile_prefix) {
  __shared__ float4 sD[kEvalWarps][kWin * kDParamF4];
  __shared__ SegParams sp[kEvalWarps][kSegBatch];
  __shared__ float sg[kEvalWarps][9 * 32];
  const int na = *n_active;
  const int n_items = tile_prefix[na];
  const int warp = threadIdx.x >> 5;
  const int stride = gridDim.x * kEvalWarps;
  int a = 0;
  for (int item = blockIdx.x * kEvalWarps + warp; item < n_items; item += stride) {
    int hi = na - 1;
    while (a < hi) {  // last a with tile_prefix[a] <= item
      const int mid = (a + hi + 1) >> 1;
      if (tile_prefix[mid] <= item)
        a = mid;
      else
        hi = mid - 1;
    }
    int tile = item - tile_prefix[a];
    const Job& job = jobs[active[a]];
    const RefDev& R = *job.ref;
    // a frame in the paired start phase has two items per tile: the zero start, then the rigid one
    const bool second = tile >= R.n_tiles;
    if (second) tile -= R.n_tiles;
    eval4_tile<NDIM, FT, RT, kPipe<FT, RT, MB>>(job, R, tile, sD[warp], sp[warp], sg[warp], second ? job.dparams2 : job.dparams,
                             second ? job.partials2 : job.partials);
  }
}

template <typename Fn>
inline cudaError_t dispatch_mb(int mb, Fn&& f) {
  if (mb >= 4) return f(std::integral_constant<int, 4>{});
  if (mb == 3) return f(std::integral_constant<int, 3>{});
  return f(std::integral_constant<int, 2>{});
}

cudaError_t launch_eval4(const Job* jobs_dev, int n_jobs, int max_tiles, int n_dim, int frame_kind, bool ref_bf16,
                         int mb, cudaStream_t s) {
  const dim3 grid((max_tiles + kEvalWarps - 1) / kEvalWarps, n_jobs);
  return dispatch_cfg(n_dim, frame_kind, ref_bf16, [&](auto c) {
    using C = decltype(c);
    return dispatch_mb(mb, [&](auto m) {
      eval4_kernel<C::nd, typename C::F, typename C::R, decltype(m)::value><<<grid, kEvalThreads, 0, s>>>(jobs_dev);
      return cudaGetLastError();
    });
  });
}

size_t eval4_active_local_bytes(int n_dim, int frame_kind, bool ref_bf16, int mb) {
  size_t bytes = 0;
  dispatch_cfg(n_dim, frame_kind, ref_bf16, [&](auto c) {
    using C = decltype(c);
    return dispatch_mb(mb, [&](auto m) {
      cudaFuncAttributes a{};
      const cudaError_t e =
          cudaFuncGetAttributes(&a, eval4_active_kernel<C::nd, typename C::F, typename C::R, decltype(m)::value>);
      bytes = e == cudaSuccess ? a.localSizeBytes : 0;
      return e;
    });
  });
  return bytes;
}

cudaError_t launch_eval4_active(const Job* jobs_dev, const int* active, const int* n_active, const int* tile_prefix,
                                long long most_items, int n_dim, int frame_kind, bool ref_bf16, int mb, int grid,
                                cudaStream_t s) {
  const long long most_ctas = (most_items + kEvalWarps - 1) / kEvalWarps;
  const int g = (int)(most_ctas < grid ? (most_ctas < 1 ? 1 : most_ctas) : grid);
  return dispatch_cfg(n_dim, frame_kind, ref_bf16, [&](auto c) {
    using C = decltype(c);
    return dispatch_mb(mb, [&](auto m) {
      eval4_active_kernel<C::nd, typename C::F, typename C::R, decltype(m)::value>
          <<<g, kEvalThreads, 0, s>>>(jobs_dev, active, n_active, tile_prefix);
      return cudaGetLastError();
    });
  });
}

}  // namespace fa
