// fa_api.cu -- host runtime behind the C ABI (include/fa_b200.h): device memory under a budget,
// reference set-up (exact scan geometry, Sobel, Hessian), frame slots, fused evaluations, the
// single-frame and batched trust-region drivers, and the phase correlator.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>

#include "fa_runtime.h"

using fa::Job;
using fa::RefDev;
using fa::RowDesc;
using namespace fa_rt;

// ================================================================== runtime helpers ================

namespace fa_rt {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

fa_status fail(fa_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

fa_status dalloc(fa_context* ctx, size_t bytes, void** out, std::vector<Alloc>& owner) {
  if (bytes == 0) bytes = 16;
  size_t prev = ctx->used.fetch_add(bytes);
  if (ctx->budget && prev + bytes > ctx->budget) {
    ctx->used.fetch_sub(bytes);
    return fail(FA_ERR_OOM, "memory budget exhausted (" + std::to_string(prev + bytes) + " > " +
                                std::to_string(ctx->budget) + " bytes)");
  }
  cudaError_t e = cudaMalloc(out, bytes);
  if (e != cudaSuccess) {
    ctx->used.fetch_sub(bytes);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? FA_ERR_OOM : FA_ERR_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  owner.push_back({*out, bytes});
  return FA_OK;
}

void dfree_all(fa_context* ctx, std::vector<Alloc>& owner) {
  for (auto& a : owner) {
    cudaFree(a.p);
    ctx->used.fetch_sub(a.n);
  }
  owner.clear();
}

}  // namespace fa_rt

namespace fa_rt {

// ImageScanParameters fields after AbstractFrameWarper::processScanParameters
// (FrameWarper.cpp:223-236).
fa_scan_params process_scan(const fa_scan_params& in, int nz, int nD) {
  fa_scan_params out = in;
  double frame_interval_max = nz * in.frame_duration / (nD - nz);
  if ((in.interframe_duration - in.frame_duration) > frame_interval_max) {
    out.interframe_duration = out.frame_duration + frame_interval_max;
    out.stack_duration = (nz - 1) * out.interframe_duration + out.frame_duration;
  }
  return out;
}

}  // namespace fa_rt

namespace {


struct ScanEval {
  fa_scan_params p;
  int ny, nx, nD;
  double q(long long s) const {
    const long long plane = (long long)ny * nx;
    int z = (int)(s / plane);
    int y = (int)((s / nx) % ny);
    int x = (int)(s % nx);
    double t = z * p.interframe_duration + y * p.interline_duration + x * p.pixel_duration;
    return t / p.stack_duration * (nD - 1);
  }
  int i(long long s) const {
    double ip;
    modf(q(s), &ip);
    return (int)ip;
  }
};

// Tiles of whole rows, about target_tile_voxels each, never longer than the shortest storage range
// (so a tile meets at most two ranges); per tile its first range, per control point its tile span.
void assign_tiles(Geometry& G, int target_tile_voxels) {
  const int nx = G.nx, nD = G.nD;
  int tr = std::max(1, target_tile_voxels / nx);
  tr = (int)std::min<long long>(tr, std::max<long long>(1, G.lmin / nx));
  G.tile_rows = tr;
  G.n_tiles = (G.n_rows + tr - 1) / tr;
  G.tile_c0.resize(G.n_tiles);
  for (int t = 0; t < G.n_tiles; t++) G.tile_c0[t] = G.rows[(size_t)t * tr].r0;
  G.ctrl_tiles.resize(nD);
  for (int c = 0; c < nD; c++) {
    int a = (int)(std::lower_bound(G.tile_c0.begin(), G.tile_c0.end(), c - 2) - G.tile_c0.begin());
    int b = (int)(std::upper_bound(G.tile_c0.begin(), G.tile_c0.end(), c) - G.tile_c0.begin());
    G.ctrl_tiles[c] = make_int2(a, b);
  }
}

fa_status build_geometry(const fa_scan_params& scan, int nz, int ny, int nx, int nD, int target_tile_voxels,
                         Geometry& G) {
  if (nx < 2 || ny < 2 || nz < 1 || nD < 2)
    return fail(FA_ERR_BAD_ARG, "need nx >= 2, ny >= 2, nz >= 1 and nD >= 2 (the Sobel edge filters read two "
                                "samples per axis)");
  const long long N = (long long)nz * ny * nx;
  if (N >= (1LL << 31)) return fail(FA_ERR_UNSUPPORTED, "volume larger than 2^31 voxels");
  const fa_scan_params p = process_scan(scan, nz, nD);
  if (!(p.pixel_duration > 0) || !(p.stack_duration > 0) || !std::isfinite(p.stack_duration) ||
      !std::isfinite(p.interframe_duration) || !std::isfinite(p.interline_duration))
    return fail(FA_ERR_BAD_ARG, "scan durations must be finite and positive");
  ScanEval S{p, ny, nx, nD};
  G.nz = nz;
  G.ny = ny;
  G.nx = nx;
  G.nD = nD;
  G.N = N;
  G.n_rows = nz * ny;
  // The scan time must increase along the scan so that interval boundaries are single points.
  for (int r = 0; r + 1 < G.n_rows; r++)
    if (S.q((long long)r * nx + nx - 1) > S.q((long long)(r + 1) * nx))
      return fail(FA_ERR_UNSUPPORTED, "scan time decreases between lines or planes (interframe or interline "
                                      "duration shorter than the line/frame it follows)");
  if ((long long)S.i(N - 1) != (long long)nD - 2) return fail(FA_ERR_BAD_ARG, "Something went wrong");
  G.scan_begin.assign(nD - 1, 0);
  for (int k = 1; k <= nD - 2; k++) {
    long long lo = G.scan_begin[k - 1], hi = N - 1;
    while (lo < hi) {
      long long mid = lo + (hi - lo) / 2;
      if (S.i(mid) >= k)
        hi = mid;
      else
        lo = mid + 1;
    }
    if (S.i(lo) != k) return fail(FA_ERR_UNSUPPORTED, "a control interval is skipped by the scan");
    G.scan_begin[k] = lo;
  }
  auto storage_of = [&](long long s) {
    long long row = s / nx;
    int xs = (int)(s % nx);
    int y = (int)(row % ny);
    int xt = (scan.bidirectional && (y % 2 == 1)) ? nx - 1 - xs : xs;
    return row * nx + xt;
  };
  G.begin.assign(nD, 0);
  G.end.assign(nD, 0);
  for (int k = 0; k <= nD - 2; k++) G.begin[k] = (int)storage_of(G.scan_begin[k]);
  for (int k = 1; k <= nD - 2; k++)
    if (G.begin[k] <= G.begin[k - 1])
      return fail(FA_ERR_UNSUPPORTED, "bidirectional ranges are not increasing in storage order");
  for (int k = 0; k < nD - 2; k++) G.end[k] = G.begin[k + 1] - 1;
  G.end[nD - 2] = (int)(N - 1);
  long long lmin = N;
  for (int k = 0; k <= nD - 2; k++) {
    lmin = std::min<long long>(lmin, (long long)G.end[k] - G.begin[k] + 1);
    long long send = (k < nD - 2) ? G.scan_begin[k + 1] : N;
    lmin = std::min<long long>(lmin, send - G.scan_begin[k]);
  }
  if (lmin < nx)
    return fail(FA_ERR_UNSUPPORTED, "a control interval is shorter than one image row (" + std::to_string(lmin) +
                                        " < " + std::to_string(nx) + " voxels)");
  G.dq = (float)(p.pixel_duration / p.stack_duration * (nD - 1));
  G.rows.resize(G.n_rows);
  int r0 = 0;
  for (int row = 0; row < G.n_rows; row++) {
    RowDesc d{};
    const long long s0 = (long long)row * nx;
    d.di0 = S.i(s0);
    d.qbase = (float)(S.q(s0) - d.di0);
    d.xdi = nx;
    if (d.di0 + 1 <= nD - 2 && G.scan_begin[d.di0 + 1] < s0 + nx) d.xdi = (int)(G.scan_begin[d.di0 + 1] - s0);
    while (r0 + 1 <= nD - 2 && G.begin[r0 + 1] <= s0) r0++;
    d.r0 = r0;
    d.xr = nx;
    if (r0 + 1 <= nD - 2 && G.begin[r0 + 1] < s0 + nx) d.xr = (int)(G.begin[r0 + 1] - s0);
    d.xlast = -1;
    d.y = row % ny;
    d.z = row / ny;
    const long long e = G.end[r0];
    if (e >= s0 && e < s0 + nx) d.xlast = (int)(e - s0);
    G.rows[row] = d;
  }
  G.lmin = lmin;
  assign_tiles(G, target_tile_voxels);
  return FA_OK;
}

}  // namespace

namespace fa_rt {

// Control-point parameters of the fused pass from a host displacement set (see kDParamF4).
void make_dparams(const double* D, int nD, int n_dim, float4* out) {
  for (int k = 0; k < nD; k++) {
    double d[3], dn[3];
    for (int c = 0; c < 3; c++) {
      d[c] = c < n_dim ? D[3 * k + c] : 0.0;
      dn[c] = (c < n_dim && k + 1 < nD) ? D[3 * (k + 1) + c] : d[c];
    }
    const double f0 = std::floor(d[0]), f1 = std::floor(d[1]), f2 = std::floor(d[2]);
    out[3 * k + 0] = make_float4((float)f0, (float)f1, (float)f2, 0.f);
    out[3 * k + 1] = make_float4((float)(d[0] - f0), (float)(d[1] - f1), (float)(d[2] - f2), 0.f);
    out[3 * k + 2] = make_float4((float)(dn[0] - d[0]), (float)(dn[1] - d[1]), (float)(dn[2] - d[2]), 0.f);
  }
}

}  // namespace fa_rt

namespace {


}  // namespace

namespace fa_rt {

bool finite_all(const double* v, size_t n) {
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(v[i])) return false;
  return true;
}

}  // namespace fa_rt

namespace {


}  // namespace

// ================================================================== context ========================

extern "C" const char* fa_last_error(void) { return g_err.c_str(); }

extern "C" const char* fa_status_string(fa_status s) {
  switch (s) {
    case FA_OK: return "ok";
    case FA_ERR_BAD_ARG: return "bad argument";
    case FA_ERR_OOM: return "out of memory";
    case FA_ERR_CUDA: return "CUDA error";
    case FA_ERR_TIMEOUT: return "timeout";
    case FA_ERR_UNSUPPORTED: return "unsupported";
    case FA_ERR_NOT_FOUND: return "not found";
    case FA_ERR_STATE: return "bad state";
    case FA_ERR_BUSY: return "busy";
  }
  return "unknown";
}

extern "C" fa_status fa_gpu_support(int* supported, char* message, size_t message_len) {
  if (!supported) return fail(FA_ERR_BAD_ARG, "supported is NULL");
  *supported = 0;
  auto msg = [&](const char* m) {
    if (message && message_len) {
      std::snprintf(message, message_len, "%s", m);
    }
  };
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    msg(e == cudaErrorInsufficientDriver ? "Insufficient Driver" : "No compatible GPU");
    return FA_OK;
  }
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) {
    msg("No compatible GPU (this build targets sm_100a)");
    return FA_OK;
  }
  *supported = 1;
  msg("");
  return FA_OK;
}

extern "C" fa_status fa_create(const fa_config* cfg, fa_context** out) {
  if (!out) return fail(FA_ERR_BAD_ARG, "out is NULL");
  int dev = cfg ? cfg->device : 0;
  FA_CU(cudaSetDevice(dev));
  size_t free_b = 0, total_b = 0;
  FA_CU(cudaMemGetInfo(&free_b, &total_b));
  fa_context* c = new fa_context;
  c->device = dev;
  c->budget = (cfg && cfg->memory_budget) ? cfg->memory_budget : (size_t)(0.9 * (double)free_b);
  c->autotune = cfg ? cfg->autotune : 0;
  *out = c;
  return FA_OK;
}

extern "C" fa_status fa_destroy(fa_context* ctx) {
  if (!ctx) return fail(FA_ERR_BAD_ARG, "ctx is NULL");
  delete ctx;
  return FA_OK;
}

extern "C" fa_status fa_scan_params_init(double line_duration, double interline_duration, double interframe_duration,
                                         int n_x, int n_y, int n_z, int bidirectional, fa_scan_params* s) {
  if (!s) return fail(FA_ERR_BAD_ARG, "out is NULL");
  s->line_duration = line_duration;
  s->interline_duration = interline_duration;
  s->interframe_duration = interframe_duration;
  s->n_x = std::max(n_x, 1);
  s->n_y = std::max(n_y, 1);
  s->n_z = n_z;
  if (s->interline_duration < s->line_duration) s->interline_duration = 1.01 * s->line_duration;
  s->pixel_duration = s->line_duration / s->n_x;
  s->frame_duration = s->n_y * s->interline_duration;
  s->stack_duration = (s->n_z - 1) * s->interframe_duration + s->frame_duration;
  s->bidirectional = bidirectional ? 1 : 0;
  return FA_OK;
}

// ================================================================== reference ======================

namespace {

// Re-tiles a reference for a new target tile size and uploads the tables and RefDev.
fa_status retile(fa_reference* R, int target_tile_voxels) {
  assign_tiles(R->G, target_tile_voxels);
  R->host.tile_rows = R->G.tile_rows;
  R->host.n_tiles = R->G.n_tiles;
  cudaStream_t s = R->stream;
  FA_CU(cudaMemcpyAsync(R->tile_c0_dev, R->G.tile_c0.data(), R->G.tile_c0.size() * sizeof(int),
                        cudaMemcpyHostToDevice, s));
  FA_CU(cudaMemcpyAsync(R->ctrl_dev, R->G.ctrl_tiles.data(), R->G.ctrl_tiles.size() * sizeof(int2),
                        cudaMemcpyHostToDevice, s));
  FA_CU(cudaMemcpyAsync(R->dev, &R->host, sizeof(RefDev), cudaMemcpyHostToDevice, s));
  FA_CU(cudaStreamSynchronize(s));
  return FA_OK;
}

// Launches of at least this many frames use the register budget tuned for many frames.
constexpr int kManyFrames = 4;

struct TuneResult {
  int target, mb, grid_mult, mb_small;
  double ms;
};
std::mutex g_tune_mu;
std::map<std::string, TuneResult> g_tune_cache;

// The project's autotuner for the fused pass: times each (tile size, CTAs per SM) candidate with the
// persistent kernel the batched solver uses, on a launch of K distinct synthetic frames (copies of the
// reference, slightly displaced; K up to 16, as many as fit in 256 MB, so that the frames do not all
// stay in L2 as a real batch's do not) and on a launch of one. The tile size and the budget for
// launches of many frames are those of the lowest per-frame time of the K-frame launch; at that tile
// size the budget for launches of a few frames (single-frame path, static-scratch entry, serving loop)
// is the fastest one-frame one. The choice is cached
// per volume shape, control-point count and precision for the life of the process. Register budgets
// under which the kernel spills more than 128 bytes are skipped (the largest budget is always a
// candidate).
fa_status autotune(fa_reference* R) {
  char keyb[128];
  std::snprintf(keyb, sizeof(keyb), "%d,%d,%d,%d,%d,%d", R->nz, R->ny, R->nx, R->nD, (int)R->prec,
                R->scan.bidirectional);
  const std::string key(keyb);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      R->host.tune_mb = it->second.mb;
      R->host.tune_grid_mult = it->second.grid_mult;
      R->host.tune_mb_small = it->second.mb_small;
      return retile(R, it->second.target);
    }
  }
  fa_context* ctx = R->ctx;
  const int kind = R->prec == FA_PREC_MIXED ? fa::kFrameF16 : fa::kFrameF32;
  std::vector<Alloc> tmp;
  auto done = [&](fa_status st) {
    std::string keep = g_err;
    cudaStreamSynchronize(R->stream);
    dfree_all(ctx, tmp);
    g_err = keep;
    return st;
  };
  void* frame;
  float4* dp;
  double* parts;
  Job* jobs_dev;
  int *list, *cnt, *prefix;
  const int hz = R->nz > 1 ? fa::kHaloZ : 0;
  const int pitch = R->nx + 2 * fa::kHaloX;
  const long long plane = (long long)pitch * (R->ny + 2 * fa::kHaloY);
  const size_t esz = kind == fa::kFrameF16 ? 2 : 4;
  const size_t elems = (size_t)plane * (R->nz + 2 * hz);
  const int K = (int)std::max<size_t>(2, std::min<size_t>(16, ((size_t)256 << 20) / (elems * esz)));
  fa_status st = dalloc(ctx, (size_t)K * elems * esz, &frame, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, (size_t)R->nD * fa::kDParamF4, &dp, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, (size_t)K * R->G.n_rows * fa::kPartialDoubles, &parts, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, (size_t)K, &jobs_dev, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, (size_t)K, &list, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, 1, &cnt, tmp);
  if (st == FA_OK) st = dalloc_t(ctx, (size_t)K + 1, &prefix, tmp);
  if (st != FA_OK) return done(st);
  cudaStream_t s = R->stream;
  void* interior = static_cast<char*>(frame) + ((long long)hz * plane + (long long)fa::kHaloY * pitch + fa::kHaloX) * esz;
  cudaError_t e = cudaMemsetAsync(frame, 0, elems * esz, s);
  if (e == cudaSuccess)
    e = fa::launch_to_slot(R->host.ref32, FA_F32, interior, kind, R->nz, R->ny, R->nx, pitch, plane, false, s);
  for (int i = 1; i < K && e == cudaSuccess; i++)
    e = cudaMemcpyAsync(static_cast<char*>(frame) + (size_t)i * elems * esz, frame, elems * esz,
                        cudaMemcpyDeviceToDevice, s);
  std::vector<double> D((size_t)R->nD * 3);
  for (int k = 0; k < R->nD; k++) {
    D[3 * k] = 0.3 + 0.01 * k;
    D[3 * k + 1] = -0.2;
    D[3 * k + 2] = R->n_dim == 3 ? 0.1 : 0.0;
  }
  std::vector<float4> hdp((size_t)R->nD * fa::kDParamF4);
  make_dparams(D.data(), R->nD, R->n_dim, hdp.data());
  std::vector<Job> jobs(K);
  std::vector<int> all(K);
  for (int i = 0; i < K; i++) {
    Job j{};
    j.ref = R->dev;
    j.frame = static_cast<char*>(interior) + (size_t)i * elems * esz;
    j.fplane = plane;
    j.fpitch = pitch;
    j.fpad = 1;
    j.dparams = dp;
    j.partials = parts + (size_t)i * R->G.n_rows * fa::kPartialDoubles;
    jobs[i] = j;
    all[i] = i;
  }
  const int kcount = K, kone = 1;
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, hdp.data(), hdp.size() * sizeof(float4), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(jobs_dev, jobs.data(), K * sizeof(Job), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(list, all.data(), K * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, &kcount, sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("autotune set-up: ") + cudaGetErrorString(e)));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  TuneResult best{4096, 2, 2, 2, 1e30};
  const int targets[] = {1024, 2048, 4096, 8192, 16384};
  const int mbs[] = {2, 3, 4};
  // per-frame time of the K-frame launch and time of the one-frame launch per (tile size, budget);
  // 0 = not a candidate
  double many[5][3], one[5][3];
  for (int ti = 0; ti < 5; ti++)
    for (int mi = 0; mi < 3; mi++) many[ti][mi] = one[ti][mi] = 0.0;
  std::vector<int> hprefix(K + 1);
  for (int ti = 0; ti < 5; ti++) {
    const int target = targets[ti];
    if (retile(R, target) != FA_OK) break;
    for (int i = 0; i <= K; i++) hprefix[i] = i * R->G.n_tiles;
    e = cudaMemcpyAsync(prefix, hprefix.data(), (K + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) break;
    for (int mi = 0; mi < 3; mi++) {
      const int mb = mbs[mi];
      const bool mixed = R->prec == FA_PREC_MIXED;
      // register budgets under which the kernel spills more than a few values are not candidates
      if (mb != mbs[0] && fa::eval4_active_local_bytes(R->n_dim, kind, mixed, mb) > 128) continue;
      auto launch = [&]() {
        return fa::launch_eval4_active(jobs_dev, list, cnt, prefix, (long long)K * R->G.n_tiles, R->n_dim, kind, mixed,
                                       mb, mb * sms, s);
      };
      double per_frame[2] = {0.0, 0.0};  // K frames, one frame
      for (int c = 0; c < 2; c++) {
        const int count = c == 0 ? K : 1;
        e = cudaMemcpyAsync(cnt, count == K ? &kcount : &kone, sizeof(int), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e0, s);
        for (int r = 0; r < 3 && e == cudaSuccess; r++) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(e1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        g_launches += 4;
        if (e != cudaSuccess) break;
        per_frame[c] = ms / count;
      }
      if (e != cudaSuccess) break;
      many[ti][mi] = per_frame[0];
      one[ti][mi] = per_frame[1];
    }
    if (e != cudaSuccess) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(e)));
  for (int ti = 0; ti < 5; ti++) {
    double tk = 1e30, t1 = 1e30;
    int mb_k = 2, mb_1 = 2;
    for (int mi = 0; mi < 3; mi++) {
      if (many[ti][mi] > 0.0 && many[ti][mi] < tk) {
        tk = many[ti][mi];
        mb_k = mbs[mi];
      }
      if (one[ti][mi] > 0.0 && one[ti][mi] < t1) {
        t1 = one[ti][mi];
        mb_1 = mbs[mi];
      }
    }
    if (tk < 1e30 && t1 < 1e30 && tk < best.ms) best = TuneResult{targets[ti], mb_k, mb_k, mb_1, tk};
  }
  R->host.tune_mb = best.mb;
  R->host.tune_grid_mult = best.grid_mult;
  R->host.tune_mb_small = best.mb_small;
  fa_status r = retile(R, best.target);
  if (r == FA_OK) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
  }
  return done(r);
}

fa_status reference_setup(fa_reference* R, const float* src, bool src_device) {
  fa_context* ctx = R->ctx;
  Geometry& G = R->G;
  const long long N = R->N;
  FA_CU(cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking));
  RefDev& h = R->host;
  h.nz = R->nz;
  h.ny = R->ny;
  h.nx = R->nx;
  h.nD = R->nD;
  h.n_dim = R->n_dim;
  h.n_rows = G.n_rows;
  h.N = N;
  h.bidir = R->scan.bidirectional;
  h.dq = G.dq;
  h.tile_rows = G.tile_rows;
  h.n_tiles = G.n_tiles;
  h.P = R->P;
  h.tune_mb = 2;
  h.tune_grid_mult = 2;
  h.tune_mb_small = 2;
  RowDesc* rows;
  int* tile_c0;
  int2* ctrl;
  float *ref32, *gx, *gy, *gz;
  double *Hd, *Hl, *tparts, *scan_dev;
  FA_TRY(dalloc_t(ctx, G.rows.size(), &rows, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)G.n_rows, &tile_c0, R->allocs));  // room for any tile size
  FA_TRY(dalloc_t(ctx, G.ctrl_tiles.size(), &ctrl, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)N, &ref32, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)N, &gx, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)N, &gy, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)N, &gz, R->allocs));
  const int nn = R->n_dim * R->n_dim;
  FA_TRY(dalloc_t(ctx, (size_t)R->nD * nn, &Hd, R->allocs));
  FA_TRY(dalloc_t(ctx, (size_t)R->nD * nn, &Hl, R->allocs));
  FA_TRY(dalloc_t(ctx, 4, &scan_dev, R->allocs));
  FA_TRY(dalloc_t(ctx, 1, &R->dev, R->allocs));
  std::vector<Alloc> tmp;
  fa_status st = dalloc_t(ctx, (size_t)G.n_tiles * 2 * 21, &tparts, tmp);
  R->tile_c0_dev = tile_c0;
  R->ctrl_dev = ctrl;
  if (st != FA_OK) return st;
  cudaStream_t s = R->stream;
  FA_CU(cudaMemcpyAsync(rows, G.rows.data(), G.rows.size() * sizeof(RowDesc), cudaMemcpyHostToDevice, s));
  FA_CU(cudaMemcpyAsync(tile_c0, G.tile_c0.data(), G.tile_c0.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  FA_CU(cudaMemcpyAsync(ctrl, G.ctrl_tiles.data(), G.ctrl_tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, s));
  FA_CU(cudaMemcpyAsync(ref32, src, (size_t)N * sizeof(float), src_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  FA_CU(fa::launch_sobel(ref32, R->nz, R->ny, R->nx, gx, gy, gz, s));
  h.rows = rows;
  h.tile_c0 = tile_c0;
  h.ctrl_tiles = ctrl;
  h.ref32 = ref32;
  h.gx32 = gx;
  h.gy32 = gy;
  h.gz32 = gz;
  h.Hd = Hd;
  h.Hl = Hl;
  if (R->prec == FA_PREC_MIXED) {
    __nv_bfloat16* q16;
    FA_TRY(dalloc_t(ctx, (size_t)((N + 3) / 4) * 16, &q16, R->allocs));
    FA_CU(fa::launch_to_quad16(ref32, gx, gy, gz, N, q16, s));
    h.q16 = q16;
  }
  FA_CU(cudaMemcpyAsync(R->dev, &h, sizeof(RefDev), cudaMemcpyHostToDevice, s));
  const fa_scan_params p = process_scan(R->scan, R->nz, R->nD);
  double scan4[4] = {p.pixel_duration, p.interline_duration, p.interframe_duration, p.stack_duration};
  FA_CU(fa::launch_hessian(R->dev, h, scan4, tparts, Hd, Hl, s));
  R->hd.assign((size_t)R->nD * nn, 0.0);
  R->hl.assign((size_t)R->nD * nn, 0.0);
  FA_CU(cudaMemcpyAsync(R->hd.data(), Hd, R->hd.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  FA_CU(cudaMemcpyAsync(R->hl.data(), Hl, R->hl.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  FA_CU(cudaStreamSynchronize(s));
  fa::band_bounds(R->hd.data(), R->hl.data(), R->nD, R->n_dim, &h.h_inf, &h.h_mindiag);
  {
    double *L0, *inv0;
    int* ok_dev;
    FA_TRY(dalloc_t(ctx, (size_t)R->P * 2 * R->n_dim, &L0, R->allocs));
    FA_TRY(dalloc_t(ctx, (size_t)R->P, &inv0, R->allocs));
    FA_TRY(dalloc_t(ctx, 1, &ok_dev, tmp));
    FA_CU(fa::launch_chol0(Hd, Hl, R->nD, R->n_dim, L0, inv0, ok_dev, s));
    int ok = 0;
    FA_CU(cudaMemcpyAsync(&ok, ok_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
    FA_CU(cudaStreamSynchronize(s));
    h.L0 = L0;
    h.inv0 = inv0;
    h.chol0_ok = ok;
  }
  FA_CU(cudaMemcpyAsync(R->dev, &h, sizeof(RefDev), cudaMemcpyHostToDevice, s));
  FA_CU(cudaStreamSynchronize(s));
  dfree_all(ctx, tmp);
  if (ctx->autotune && R->nx % 4 == 0) FA_TRY(autotune(R));
  return FA_OK;
}

fa_status set_reference_impl(fa_context* ctx, const float* src, bool src_device, int nz, int ny, int nx, int nD,
                             const fa_scan_params* scan, fa_precision precision, fa_reference** out) {
  if (!ctx || !src || !scan || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (precision != FA_PREC_F32 && precision != FA_PREC_MIXED) return fail(FA_ERR_BAD_ARG, "unknown precision");
  FA_CU(cudaSetDevice(ctx->device));
  fa_reference* R = new fa_reference;
  R->ctx = ctx;
  R->nz = nz;
  R->ny = ny;
  R->nx = nx;
  R->nD = nD;
  R->n_dim = nz > 1 ? 3 : 2;
  R->P = nD * R->n_dim;
  R->N = (long long)nz * ny * nx;
  R->prec = precision;
  R->scan = *scan;
  fa_status st = build_geometry(*scan, nz, ny, nx, nD, 4096, R->G);
  if (st == FA_OK) st = reference_setup(R, src, src_device);
  if (st != FA_OK) {
    std::string keep = g_err;
    if (R->stream) cudaStreamDestroy(R->stream);
    dfree_all(ctx, R->allocs);
    delete R;
    g_err = keep;
    return st;
  }
  *out = R;
  return FA_OK;
}

}  // namespace

extern "C" fa_status fa_set_reference(fa_context* ctx, const float* reference, int nz, int ny, int nx, int nD,
                                      const fa_scan_params* scan, fa_precision precision, fa_reference** out) {
  return set_reference_impl(ctx, reference, false, nz, ny, nx, nD, scan, precision, out);
}

extern "C" fa_status fa_set_reference_device(fa_context* ctx, const float* reference_device, int nz, int ny, int nx,
                                             int nD, const fa_scan_params* scan, fa_precision precision,
                                             fa_reference** out) {
  return set_reference_impl(ctx, reference_device, true, nz, ny, nx, nD, scan, precision, out);
}

extern "C" fa_status fa_reference_destroy(fa_reference* R) {
  if (!R) return fail(FA_ERR_BAD_ARG, "ref is NULL");
  if (R->n_frames.load() != 0) return fail(FA_ERR_STATE, "frames of this reference are still registered");
  cudaSetDevice(R->ctx->device);
  if (R->stream) cudaStreamDestroy(R->stream);
  dfree_all(R->ctx, R->allocs);
  delete R;
  return FA_OK;
}

extern "C" fa_status fa_reference_tuning(const fa_reference* R, int* tile_voxels, int* ctas_per_sm) {
  if (!R) return fail(FA_ERR_BAD_ARG, "ref is NULL");
  if (tile_voxels) *tile_voxels = R->G.tile_rows * R->nx;
  if (ctas_per_sm) *ctas_per_sm = R->host.tune_mb;
  return FA_OK;
}

extern "C" fa_status fa_reference_retune(fa_reference* R, int tile_voxels, int ctas_per_sm) {
  if (!R || tile_voxels < 1 || ctas_per_sm < 2 || ctas_per_sm > 4) return fail(FA_ERR_BAD_ARG, "bad arguments");
  if (R->n_frames.load() != 0) return fail(FA_ERR_STATE, "frames of this reference are registered");
  FA_CU(cudaSetDevice(R->ctx->device));
  R->host.tune_mb = ctas_per_sm;
  R->host.tune_grid_mult = ctas_per_sm;
  R->host.tune_mb_small = ctas_per_sm;
  return retile(R, tile_voxels);
}

extern "C" fa_status fa_reference_info(const fa_reference* R, int* n_dim, int* n_params) {
  if (!R) return fail(FA_ERR_BAD_ARG, "ref is NULL");
  if (n_dim) *n_dim = R->n_dim;
  if (n_params) *n_params = R->P;
  return FA_OK;
}

extern "C" fa_status fa_get_hessian(const fa_reference* R, double* H) {
  if (!R || !H) return fail(FA_ERR_BAD_ARG, "NULL argument");
  const int P = R->P, nd = R->n_dim, nn = nd * nd;
  for (int i = 0; i < P; i++)
    for (int j = 0; j < P; j++) {
      const int bi = i / nd, bj = j / nd, a = i % nd, b = j % nd;
      double v = 0;
      if (bi == bj)
        v = R->hd[(size_t)bi * nn + a * nd + b];
      else if (bi == bj + 1)
        v = R->hl[(size_t)bi * nn + a * nd + b];
      else if (bj == bi + 1)
        v = R->hl[(size_t)bj * nn + b * nd + a];
      H[(size_t)i * P + j] = v;
    }
  return FA_OK;
}

extern "C" fa_status fa_get_gradient(const fa_reference* R, float* gx, float* gy, float* gz) {
  if (!R) return fail(FA_ERR_BAD_ARG, "ref is NULL");
  FA_CU(cudaSetDevice(R->ctx->device));
  size_t n = (size_t)R->N * sizeof(float);
  if (gx) FA_CU(cudaMemcpy(gx, R->host.gx32, n, cudaMemcpyDeviceToHost));
  if (gy) FA_CU(cudaMemcpy(gy, R->host.gy32, n, cudaMemcpyDeviceToHost));
  if (gz) FA_CU(cudaMemcpy(gz, R->host.gz32, n, cudaMemcpyDeviceToHost));
  return FA_OK;
}

extern "C" fa_status fa_get_ranges(const fa_reference* R, int* ranges) {
  if (!R || !ranges) return fail(FA_ERR_BAD_ARG, "NULL argument");
  for (int k = 0; k < R->nD; k++) {
    ranges[2 * k] = (k <= R->nD - 2) ? R->G.begin[k] : 0;
    ranges[2 * k + 1] = (k <= R->nD - 2) ? R->G.end[k] : 0;
  }
  return FA_OK;
}

// ================================================================== frames =========================

namespace {

size_t work_doubles(const fa_reference* R) { return (size_t)R->P * (2 * R->n_dim) + 3 * (size_t)R->P; }

int default_kind(const fa_reference* R) { return R->prec == FA_PREC_MIXED ? fa::kFrameF16 : fa::kFrameF32; }

}  // namespace

namespace fa_rt {

fa_status frame_alloc(fa_reference* R, int kind, fa_frame** out) {
  fa_context* ctx = R->ctx;
  fa_frame* F = new fa_frame;
  F->ref = R;
  F->kind = kind;
  auto cleanup = [&](fa_status st) {
    std::string keep = g_err;
    if (F->stream) cudaStreamDestroy(F->stream);
    if (F->h_result) cudaFreeHost(F->h_result);
    if (F->h_dparams) cudaFreeHost(F->h_dparams);
    if (F->h_x) cudaFreeHost(F->h_x);
    if (F->h_state) cudaFreeHost(F->h_state);
    dfree_all(ctx, F->allocs);
    delete F;
    g_err = keep;
    return st;
  };
  if (cudaStreamCreateWithFlags(&F->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "cudaStreamCreate failed"));
  const size_t P = (size_t)R->P;
  fa_status st;
  void* data;
  // Frame slot with a zero halo (kHaloX columns, kHaloY rows, kHaloZ planes on each side).
  const int hz = R->nz > 1 ? fa::kHaloZ : 0;
  const int pitch = R->nx + 2 * fa::kHaloX;
  const long long plane = (long long)pitch * (R->ny + 2 * fa::kHaloY);
  const size_t esz = kind == fa::kFrameF32 ? 4 : 2;
  const size_t elems = (size_t)plane * (R->nz + 2 * hz);
  if ((st = dalloc(ctx, elems * esz, &data, F->allocs)) != FA_OK) return cleanup(st);
  if (cudaMemsetAsync(data, 0, elems * esz, F->stream) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "halo clear failed"));
  const long long origin = (long long)hz * plane + (long long)fa::kHaloY * pitch + fa::kHaloX;
  F->data = static_cast<char*>(data) + origin * esz;  // voxel (0, 0, 0)
  Job& j = F->job;
  j.ref = R->dev;
  j.frame = F->data;
  j.fplane = plane;
  j.fpitch = pitch;
  j.fpad = 1;
  if ((st = dalloc_t(ctx, (size_t)R->nD * fa::kDParamF4 * 2, &j.dparams, F->allocs)) != FA_OK) return cleanup(st);
  j.dparams2 = j.dparams + (size_t)R->nD * fa::kDParamF4;
  if ((st = dalloc_t(ctx, (size_t)R->G.n_tiles * fa::kPartialDoubles * 2, &j.partials, F->allocs)) != FA_OK)
    return cleanup(st);
  j.partials2 = j.partials + (size_t)R->G.n_tiles * fa::kPartialDoubles;
  if ((st = dalloc_t(ctx, 1, &F->state, F->allocs)) != FA_OK) return cleanup(st);
  double* pool;
  size_t nd = 4 * P + work_doubles(R) + 1 + P;
  if ((st = dalloc_t(ctx, nd, &pool, F->allocs)) != FA_OK) return cleanup(st);
  j.x = pool;
  j.g = pool + P;
  j.p = pool + 2 * P;
  j.gt = pool + 3 * P;
  j.work = pool + 4 * P;
  j.result = j.work + work_doubles(R);
  j.state = nullptr;
  if ((st = dalloc_t(ctx, 1, &F->job_dev, F->allocs)) != FA_OK) return cleanup(st);
  if (cudaMallocHost(&F->h_result, (1 + P) * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&F->h_dparams, (size_t)R->nD * fa::kDParamF4 * sizeof(float4)) != cudaSuccess ||
      cudaMallocHost(&F->h_x, P * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&F->h_state, sizeof(fa::FrameState)) != cudaSuccess)
    return cleanup(fail(FA_ERR_OOM, "cudaMallocHost failed"));
  if (cudaMemcpyAsync(F->job_dev, &F->job, sizeof(Job), cudaMemcpyHostToDevice, F->stream) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "job upload failed"));
  R->n_frames++;
  *out = F;
  return FA_OK;
}

}  // namespace fa_rt

namespace {

// Copies a dense frame (host or device, any dtype, values as stored: the +1 offset already applied)
// into the slot's interior.
fa_status frame_fill(fa_frame* F, const void* src, fa_dtype dtype, bool src_device) {
  fa_reference* R = F->ref;
  const long long N = R->N;
  const size_t esz = (dtype == FA_F32) ? 4 : 2;
  std::vector<Alloc> tmp;
  const void* dense = src;
  if (!src_device) {
    void* stage;
    FA_TRY(dalloc(R->ctx, (size_t)N * esz, &stage, tmp));
    cudaError_t e = cudaMemcpyAsync(stage, src, (size_t)N * esz, cudaMemcpyHostToDevice, F->stream);
    if (e != cudaSuccess) {
      dfree_all(R->ctx, tmp);
      return fail(FA_ERR_CUDA, std::string("frame upload: ") + cudaGetErrorString(e));
    }
    dense = stage;
  }
  cudaError_t e = fa::launch_to_slot(dense, dtype, F->data, F->kind, R->nz, R->ny, R->nx, F->job.fpitch, F->job.fplane,
                                     false, F->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(F->stream);
  dfree_all(R->ctx, tmp);
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("frame upload: ") + cudaGetErrorString(e));
  F->have_last = false;
  return FA_OK;
}

fa_status register_impl(fa_reference* R, const void* data, fa_dtype dtype, bool dev, fa_frame** out) {
  if (!R || !data || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (dtype < FA_F32 || dtype > FA_U16) return fail(FA_ERR_BAD_ARG, "unknown dtype");
  FA_CU(cudaSetDevice(R->ctx->device));
  fa_frame* F = nullptr;
  FA_TRY(frame_alloc(R, default_kind(R), &F));
  fa_status st = frame_fill(F, data, dtype, dev);
  if (st != FA_OK) {
    std::string keep = g_err;
    fa_deregister_frame(F);
    g_err = keep;
    return st;
  }
  *out = F;
  return FA_OK;
}

}  // namespace

extern "C" fa_status fa_register_frame(fa_reference* R, const void* data, fa_dtype dtype, fa_frame** out) {
  return register_impl(R, data, dtype, false, out);
}

extern "C" fa_status fa_register_frame_device(fa_reference* R, const void* data, fa_dtype dtype, fa_frame** out) {
  return register_impl(R, data, dtype, true, out);
}

extern "C" fa_status fa_update_frame(fa_frame* F, const void* data, fa_dtype dtype) {
  if (!F || !data) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(F->mu);
  FA_CU(cudaSetDevice(F->ref->ctx->device));
  return frame_fill(F, data, dtype, false);
}

extern "C" fa_status fa_deregister_frame(fa_frame* F) {
  if (!F) return fail(FA_ERR_BAD_ARG, "frame is NULL");
  cudaSetDevice(F->ref->ctx->device);
  if (F->stream) {
    cudaStreamSynchronize(F->stream);
    cudaStreamDestroy(F->stream);
  }
  if (F->h_result) cudaFreeHost(F->h_result);
  if (F->h_dparams) cudaFreeHost(F->h_dparams);
  if (F->h_x) cudaFreeHost(F->h_x);
  if (F->h_state) cudaFreeHost(F->h_state);
  F->ref->n_frames--;
  dfree_all(F->ref->ctx, F->allocs);
  delete F;
  return FA_OK;
}

// ================================================================== evaluation =====================

namespace {

fa_status evaluate(fa_frame* F, const double* D) {
  fa_reference* R = F->ref;
  if (!finite_all(D, (size_t)R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  FA_CU(cudaSetDevice(R->ctx->device));
  make_dparams(D, R->nD, R->n_dim, F->h_dparams);
  const size_t np = (size_t)R->nD * fa::kDParamF4 * sizeof(float4);
  FA_CU(cudaMemcpyAsync(F->job.dparams, F->h_dparams, np, cudaMemcpyHostToDevice, F->stream));
  FA_CU(fa::launch_eval(F->job_dev, 1, R->G.n_tiles, R->n_dim, F->kind, R->prec == FA_PREC_MIXED, F->stream,
                          R->nx % 4 == 0, R->host.tune_mb_small));
  FA_CU(fa::launch_reduce(F->job_dev, R->host, F->stream));
  g_launches += 2;
  FA_CU(cudaMemcpyAsync(F->h_result, F->job.result, (1 + R->P) * sizeof(double), cudaMemcpyDeviceToHost, F->stream));
  FA_CU(cudaStreamSynchronize(F->stream));
  F->last_f = F->h_result[0];
  F->last_g.assign(F->h_result + 1, F->h_result + 1 + R->P);
  F->lastD.assign(D, D + (size_t)R->nD * 3);
  F->have_last = true;
  return FA_OK;
}

}  // namespace

extern "C" fa_status fa_get_error(fa_frame* F, const double* D, double* f) {
  if (!F || !D || !f) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(F->mu);
  FA_TRY(evaluate(F, D));
  *f = F->last_f;
  return FA_OK;
}

extern "C" fa_status fa_get_jacobian(fa_frame* F, const double* D, double* jac) {
  if (!F || !D || !jac) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(F->mu);
  const size_t n = (size_t)F->ref->nD * 3;
  if (!F->have_last || std::memcmp(F->lastD.data(), D, n * sizeof(double)) != 0) FA_TRY(evaluate(F, D));
  std::memcpy(jac, F->last_g.data(), F->last_g.size() * sizeof(double));
  return FA_OK;
}

extern "C" fa_status fa_warp(fa_frame* F, const double* D, float invalid_value, float* out) {
  if (!F || !D || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(F->mu);
  fa_reference* R = F->ref;
  if (!finite_all(D, (size_t)R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  FA_CU(cudaSetDevice(R->ctx->device));
  if (!F->warp_out) {
    void* p;
    FA_TRY(dalloc(R->ctx, (size_t)R->N * sizeof(float), &p, F->allocs));
    F->warp_out = static_cast<float*>(p);
  }
  make_dparams(D, R->nD, R->n_dim, F->h_dparams);
  const size_t np = (size_t)R->nD * fa::kDParamF4 * sizeof(float4);
  FA_CU(cudaMemcpyAsync(F->job.dparams, F->h_dparams, np, cudaMemcpyHostToDevice, F->stream));
  FA_CU(fa::launch_warp(R->dev, R->host, F->data, F->job.fplane, F->job.fpitch, F->kind, F->job.dparams, invalid_value,
                        F->warp_out, F->stream));
  g_launches += 1;
  FA_CU(cudaMemcpyAsync(out, F->warp_out, (size_t)R->N * sizeof(float), cudaMemcpyDeviceToHost, F->stream));
  FA_CU(cudaStreamSynchronize(F->stream));
  F->have_last = false;  // dparams now hold D of the warp, not of the cached evaluation
  return FA_OK;
}

// ================================================================== alignment ======================

namespace {

fa_status init_solve(fa_frame* F, const double* rigid, int max_iterations, bool pair) {
  fa_reference* R = F->ref;
  fa::FrameState& S = *F->h_state;
  std::memset(&S, 0, sizeof(S));
  S.phase = fa::kPhaseStartZero;
  S.max_iter = max_iterations > 0 ? max_iterations : 100;
  for (int c = 0; c < 3; c++) S.rigid[c] = rigid ? rigid[c] : 0.0;
  if (R->n_dim == 2) S.rigid[2] = 0.0;
  bool nonzero = false;
  for (int c = 0; c < R->n_dim; c++) nonzero = nonzero || S.rigid[c] != 0.0;
  Job j = F->job;
  j.state = F->state;
  if (pair && nonzero) {
    // both cold starting points in the first pass: the rigid shift's parameters go to dparams2
    S.phase = fa::kPhaseStartPair;
    std::vector<double> D((size_t)R->nD * 3);
    for (int k = 0; k < R->nD; k++)
      for (int c = 0; c < 3; c++) D[(size_t)3 * k + c] = S.rigid[c];
    make_dparams(D.data(), R->nD, R->n_dim, F->h_dparams);
    FA_CU(cudaMemcpyAsync(j.dparams2, F->h_dparams, (size_t)R->nD * fa::kDParamF4 * sizeof(float4),
                          cudaMemcpyHostToDevice, F->stream));
  }
  FA_CU(cudaMemcpyAsync(F->state, &S, sizeof(S), cudaMemcpyHostToDevice, F->stream));
  FA_CU(cudaMemsetAsync(j.x, 0, 4 * (size_t)R->P * sizeof(double), F->stream));
  FA_CU(cudaMemsetAsync(j.dparams, 0, (size_t)R->nD * fa::kDParamF4 * sizeof(float4), F->stream));
  return FA_OK;
}

// Queues the copies of a solved frame's x and state into its pinned buffers on stream s.
fa_status finish_solve_enqueue(fa_frame* F, cudaStream_t s) {
  FA_CU(cudaMemcpyAsync(F->h_x, F->job.x, (size_t)F->ref->P * sizeof(double), cudaMemcpyDeviceToHost, s));
  FA_CU(cudaMemcpyAsync(F->h_state, F->state, sizeof(fa::FrameState), cudaMemcpyDeviceToHost, s));
  return FA_OK;
}

// D (and the statistics) from the copies finish_solve_enqueue queued, once they completed.
void finish_solve_read(fa_frame* F, double* D_out, fa_align_stats* stats) {
  fa_reference* R = F->ref;
  const int nd = R->n_dim;
  for (int k = 0; k < R->nD; k++) {
    D_out[3 * k] = F->h_x[k * nd];
    D_out[3 * k + 1] = F->h_x[k * nd + 1];
    D_out[3 * k + 2] = nd == 3 ? F->h_x[k * nd + 2] : 0.0;
  }
  if (stats) {
    const fa::FrameState& S = *F->h_state;
    stats->iterations = S.iter;
    stats->evaluations = S.evaluations;
    stats->accepted = S.accepted;
    stats->status = S.hit_max ? 1 : 0;
    stats->f_final = S.f;
    stats->radius_final = S.radius;
  }
}

fa_status finish_solve(fa_frame* F, double* D_out, fa_align_stats* stats) {
  FA_TRY(finish_solve_enqueue(F, F->stream));
  FA_CU(cudaStreamSynchronize(F->stream));
  finish_solve_read(F, D_out, stats);
  return FA_OK;
}

}  // namespace

extern "C" fa_status fa_align_frame(fa_frame* F, const double* rigid_shift, int max_iterations, double* D_out,
                                    fa_align_stats* stats) {
  if (!F || !D_out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (rigid_shift && !finite_all(rigid_shift, 3)) return fail(FA_ERR_BAD_ARG, "rigid shift is not finite");
  std::lock_guard<std::mutex> lk(F->mu);
  fa_reference* R = F->ref;
  FA_CU(cudaSetDevice(R->ctx->device));
  FA_TRY(init_solve(F, rigid_shift, max_iterations, false));
  Job j = F->job;
  j.state = F->state;
  FA_CU(cudaMemcpyAsync(F->job_dev, &j, sizeof(Job), cudaMemcpyHostToDevice, F->stream));
  const int max_steps = (max_iterations > 0 ? max_iterations : 100) + 4;
  int phase = fa::kPhaseStartZero;
  for (int step = 0; step < max_steps && phase != fa::kPhaseDone; step++) {
    FA_CU(fa::launch_eval(F->job_dev, 1, R->G.n_tiles, R->n_dim, F->kind, R->prec == FA_PREC_MIXED, F->stream,
                          R->nx % 4 == 0, R->host.tune_mb_small));
    FA_CU(fa::launch_solve(F->job_dev, 1, R->nD, R->n_dim, F->stream));
    g_launches += 2;
    FA_CU(cudaMemcpyAsync(&F->h_state->phase, &F->state->phase, sizeof(int), cudaMemcpyDeviceToHost, F->stream));
    FA_CU(cudaStreamSynchronize(F->stream));
    phase = F->h_state->phase;
  }
  F->have_last = false;
  FA_TRY(finish_solve(F, D_out, stats));
  Job j0 = F->job;
  FA_CU(cudaMemcpyAsync(F->job_dev, &j0, sizeof(Job), cudaMemcpyHostToDevice, F->stream));
  FA_CU(cudaStreamSynchronize(F->stream));
  return FA_OK;
}

namespace {

// Rigid starts of a batched solve taken on the device from phase-correlation peaks: frame i starts
// from peaks[i] (flat index into a cnz x cny x cnx correlation surface, x and y scaled by binning),
// once `ready` (recorded after the peaks were written) has completed.
struct PeakStart {
  const long long* peaks;
  int cnx, cny, cnz, binning;
  cudaEvent_t ready;
};

// Queues a batched solve of n frames on frames[0]'s stream: the starting states, one launch of the
// cached solve graph, and the copies of every frame's x and state into its pinned buffers; the
// caller's align_batch_finish waits for them. frame_data (optional) replaces each frame's own device
// data pointer for this call. bc keeps the buffers and the graph for the next call on the same
// frames. With `peak_start` the rigid starts come from device peaks (rigid_shifts is ignored) and the
// states are set up on the device, so the host neither waits for the peaks nor copies a state.
//
// The graph holds one while-conditional node whose body is kGraphIters x (fused pass, solve step,
// active-list compaction) and a loop-control kernel: the body repeats on the device until no frame is
// active or the iteration limit is reached, with no host round trip between rounds.
fa_status align_batch_enqueue(fa_frame* const* frames, int n, const double* rigid_shifts, int max_iterations,
                              const void* const* frame_data, BatchCache* bc, const PeakStart* peak_start) {
  if (!frames || n <= 0 || !bc) return fail(FA_ERR_BAD_ARG, "bad arguments");
  for (int i = 0; i < n; i++)
    if (!frames[i]) return fail(FA_ERR_BAD_ARG, "NULL frame");
  fa_reference* R0 = frames[0]->ref;
  for (int i = 0; i < n; i++) {
    if (frames[i]->ref->n_dim != R0->n_dim || frames[i]->ref->prec != R0->prec || frames[i]->ref->ctx != R0->ctx ||
        frames[i]->kind != frames[0]->kind)
      return fail(FA_ERR_BAD_ARG, "batched frames must share dimensionality, precision, storage and context");
  }
  if (rigid_shifts && !finite_all(rigid_shifts, (size_t)3 * n)) return fail(FA_ERR_BAD_ARG, "rigid shift not finite");
  fa_context* ctx = R0->ctx;
  FA_CU(cudaSetDevice(ctx->device));
  cudaStream_t s = frames[0]->stream;
  int max_tiles = 0, max_nD = 0;
  bool vec4 = true;
  for (int i = 0; i < n; i++) vec4 = vec4 && (frames[i]->ref->nx % 4 == 0);
  // the persistent pass evaluates both cold starting points of a frame in its first launch
  const bool vec4_all = vec4;
  std::vector<Job> jobs(n);
  // most work items of one pass: a frame in the paired start phase has two items per tile
  long long most_items = 0;
  for (int i = 0; i < n; i++) {
    fa_frame* F = frames[i];
    if (!peak_start) FA_TRY(init_solve(F, rigid_shifts ? rigid_shifts + 3 * i : nullptr, max_iterations, vec4_all));
    jobs[i] = F->job;
    jobs[i].state = F->state;
    if (frame_data) jobs[i].frame = frame_data[i];
    max_tiles = std::max(max_tiles, F->ref->G.n_tiles);
    max_nD = std::max(max_nD, F->ref->nD);
    most_items += (long long)F->ref->G.n_tiles * (vec4_all ? 2 : 1);
  }
  // host-made initial states went on every frame's stream: one wait per stream (the copies are done then)
  if (!peak_start)
    for (int i = 0; i < n; i++) FA_CU(cudaStreamSynchronize(frames[i]->stream));
  if (bc->cap < n) {
    FA_CU(cudaStreamSynchronize(s));
    batch_cache_release(ctx, bc);
    FA_TRY(dalloc_t(ctx, (size_t)n, &bc->jobs_dev, bc->allocs));
    FA_TRY(dalloc_t(ctx, 2, &bc->d_active, bc->allocs));  // [0] active frames, [1] rounds of the loop
    FA_TRY(dalloc_t(ctx, (size_t)n, &bc->d_list, bc->allocs));
    FA_TRY(dalloc_t(ctx, (size_t)n + 1, &bc->d_prefix, bc->allocs));
    if (cudaMallocHost(&bc->h_rounds, sizeof(int)) != cudaSuccess) {
      bc->h_rounds = nullptr;
      return fail(FA_ERR_OOM, "cudaMallocHost failed");
    }
    bc->cap = n;
  }
  // The job table goes up before any wait on the peaks (a copy from pageable memory may wait for the
  // stream); then the device-side start when the peaks are on the device, and the first active list
  // from the states.
  cudaError_t e = cudaMemcpyAsync(bc->jobs_dev, jobs.data(), n * sizeof(Job), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && peak_start) {
    e = cudaStreamWaitEvent(s, peak_start->ready, 0);
    if (e == cudaSuccess)
      e = fa::launch_activate_peaks(bc->jobs_dev, n, peak_start->peaks, peak_start->cnx, peak_start->cny,
                                    peak_start->cnz, peak_start->binning, max_iterations, vec4_all, s);
    g_launches += 1;
  }
  if (e == cudaSuccess)
    e = fa::launch_compact(bc->jobs_dev, n, bc->d_list, bc->d_active, bc->d_prefix, nullptr, nullptr, nullptr, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(bc->d_active + 1, 0, sizeof(int), s);
  g_launches += 1;
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("batch start: ") + cudaGetErrorString(e));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  constexpr int kGraphIters = 4;
  // each round runs kGraphIters iterations; the host loop this replaces stopped after max + 4 steps
  const int max_steps = (max_iterations > 0 ? max_iterations : 100) + 4;
  const int max_rounds = (max_steps + kGraphIters - 1) / kGraphIters;
  // the register budget tuned for launches of many frames, or of a few
  const int mb = n >= kManyFrames ? R0->host.tune_mb : R0->host.tune_mb_small;
  const long long key[7] = {n, most_items, max_nD, (vec4 ? 1 : 0) + 2 * frames[0]->kind, mb, 0, max_rounds};
  const bool reuse = bc->exec && bc->frames.size() == (size_t)n &&
                     std::equal(bc->frames.begin(), bc->frames.end(), frames) && std::equal(key, key + 7, bc->key);
  if (!reuse) {
    if (bc->exec) cudaGraphExecDestroy(bc->exec);
    bc->exec = nullptr;
    bc->frames.clear();
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphConditionalHandle loop{};
    e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = loop;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
      if (e == cudaSuccess) body = cp.conditional.phGraph_out[0];
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      for (int it = 0; it < kGraphIters && e == cudaSuccess; it++) {
        if (vec4)
          e = fa::launch_eval4_active(bc->jobs_dev, bc->d_list, bc->d_active, bc->d_prefix, most_items, R0->n_dim,
                                      frames[0]->kind, R0->prec == FA_PREC_MIXED, mb, mb * sms, s);
        else
          e = fa::launch_eval(bc->jobs_dev, n, max_tiles, R0->n_dim, frames[0]->kind, R0->prec == FA_PREC_MIXED, s,
                              false);
        if (e == cudaSuccess) e = fa::launch_solve(bc->jobs_dev, n, max_nD, R0->n_dim, s);
        if (e == cudaSuccess)
          e = fa::launch_compact(bc->jobs_dev, n, bc->d_list, bc->d_active, bc->d_prefix, nullptr, nullptr, nullptr, s);
      }
      if (e == cudaSuccess) e = fa::launch_loop_control(loop, bc->d_active, bc->d_active + 1, max_rounds, s);
      cudaGraph_t captured = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(s, &captured);
      if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&bc->exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      bc->exec = nullptr;
      return fail(FA_ERR_CUDA, std::string("batch graph: ") + cudaGetErrorString(e));
    }
    bc->frames.assign(frames, frames + n);
    std::copy(key, key + 7, bc->key);
  }
  e = cudaGraphLaunch(bc->exec, s);
  // the rounds that ran, for the launch count
  if (e == cudaSuccess) e = cudaMemcpyAsync(bc->h_rounds, bc->d_active + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("batch solve: ") + cudaGetErrorString(e));
  bc->per_round = 3 * kGraphIters + 1;
  // every frame's x and state in one batch of copies on the solve's stream
  for (int i = 0; i < n; i++) FA_TRY(finish_solve_enqueue(frames[i], s));
  return FA_OK;
}

// Waits for a batched solve queued with bc and writes D (and the statistics) of its frames.
fa_status align_batch_finish(fa_frame* const* frames, int n, const BatchCache* bc, double* D_out,
                             fa_align_stats* stats) {
  if (cudaStreamSynchronize(frames[0]->stream) != cudaSuccess) return fail(FA_ERR_CUDA, "batch solve failed");
  g_launches += (long long)*bc->h_rounds * bc->per_round;
  for (int i = 0; i < n; i++) {
    fa_frame* F = frames[i];
    finish_solve_read(F, D_out + (size_t)i * 3 * F->ref->nD, stats ? stats + i : nullptr);
    F->have_last = false;
  }
  return FA_OK;
}

// Synchronous batched solve under the frames' locks; cache (optional) keeps the buffers and the
// graph for the next call on the same frames.
fa_status align_batch_impl(fa_frame* const* frames, int n, const double* rigid_shifts, int max_iterations,
                           double* D_out, fa_align_stats* stats, const void* const* frame_data,
                           BatchCache* cache = nullptr) {
  if (!frames || n <= 0 || !D_out) return fail(FA_ERR_BAD_ARG, "bad arguments");
  for (int i = 0; i < n; i++)
    if (!frames[i]) return fail(FA_ERR_BAD_ARG, "NULL frame");
  std::vector<std::unique_lock<std::mutex>> locks;
  for (int i = 0; i < n; i++) locks.emplace_back(frames[i]->mu);
  BatchCache local;
  BatchCache* bc = cache ? cache : &local;
  fa_status r = align_batch_enqueue(frames, n, rigid_shifts, max_iterations, frame_data, bc, nullptr);
  if (r == FA_OK) r = align_batch_finish(frames, n, bc, D_out, stats);
  std::string keep = g_err;
  cudaSetDevice(frames[0]->ref->ctx->device);
  cudaStreamSynchronize(frames[0]->stream);
  if (bc == &local) batch_cache_release(frames[0]->ref->ctx, &local);
  g_err = keep;
  return r;
}

}  // namespace

namespace fa_rt {

void batch_cache_release(fa_context* ctx, BatchCache* c) {
  if (c->exec) cudaGraphExecDestroy(c->exec);
  c->exec = nullptr;
  c->frames.clear();
  if (c->h_rounds) cudaFreeHost(c->h_rounds);
  c->h_rounds = nullptr;
  dfree_all(ctx, c->allocs);
  c->jobs_dev = nullptr;
  c->d_active = c->d_list = c->d_prefix = nullptr;
  c->cap = 0;
}

}  // namespace fa_rt

extern "C" fa_status fa_align_batch(fa_frame* const* frames, int n, const double* rigid_shifts, int max_iterations,
                                    double* D_out, fa_align_stats* stats) {
  return align_batch_impl(frames, n, rigid_shifts, max_iterations, D_out, stats, nullptr);
}

// ================================================================== phase correlation =============

namespace fa_rt {

// Pointer staging for a batch of n inputs (pinned host + device arrays), grown on demand.
fa_status correlator_reserve(fa_correlator* C, int n) {
  if (n <= C->ptr_cap) return FA_OK;
  FA_CU(cudaStreamSynchronize(C->stream));
  dfree_all(C->ctx, C->ptr_allocs);
  if (C->h_ptrs) cudaFreeHost(C->h_ptrs);
  if (C->h_idx) cudaFreeHost(C->h_idx);
  C->h_ptrs = nullptr;
  C->h_idx = nullptr;
  C->ptr_cap = 0;
  FA_TRY(dalloc_t(C->ctx, 2 * (size_t)n, &C->d_ptrs, C->ptr_allocs));
  FA_TRY(dalloc_t(C->ctx, (size_t)n, &C->d_idx, C->ptr_allocs));
  if (cudaMallocHost(&C->h_ptrs, 2 * (size_t)n * sizeof(void*)) != cudaSuccess ||
      cudaMallocHost(&C->h_idx, (size_t)n * sizeof(long long)) != cudaSuccess)
    return fail(FA_ERR_OOM, "cudaMallocHost failed");
  C->ptr_cap = n;
  return FA_OK;
}

// Window, forward DFT, cross-power normalisation, inverse DFT and first-maximum argmax for n volumes
// (device pointers, FP32 or raw uint16) in batches of C->cap; peak indices to C->d_idx[first ..].
fa_status correlator_enqueue(fa_correlator* C, const void* const* vols, int in_kind, int n, double* surface,
                             bool planes, int first, void* const* slots, int slot_kind, int slot_pitch,
                             long long slot_plane, bool* slots_written) {
  if (slots_written) *slots_written = false;
  if (first > 0 && first + n > C->ptr_cap) return fail(FA_ERR_STATE, "correlator slots not reserved");
  FA_TRY(correlator_reserve(C, first + n));
  // the fused passes stage frames in 16-byte chunks: 16-byte aligned frames only
  for (int i = 0; i < n; i++) {
    C->h_ptrs[first + i] = vols[i];
    if (reinterpret_cast<uintptr_t>(vols[i]) % 16) planes = false;
  }
  planes = planes && C->planes;
  FA_CU(cudaMemcpyAsync(C->d_ptrs + first, C->h_ptrs + first, (size_t)n * sizeof(void*), cudaMemcpyHostToDevice,
                        C->stream));
  const void* const* d_ptrs = C->d_ptrs + first;
  // slots filled by the first pass: 16-byte aligned rows, and a raw uint16 slot only from uint16 frames
  const size_t slot_esz = slot_kind == fa::kFrameF32 ? 4 : 2;
  const bool fill = planes && slots && (slot_kind != fa::kFrameRawU16 || in_kind == FA_U16) &&
                    ((size_t)slot_pitch * slot_esz) % 16 == 0 && ((size_t)slot_plane * slot_esz) % 16 == 0 &&
                    C->nx % 8 == 0;
  bool fill_ok = fill;
  if (fill) {
    for (int i = 0; i < n; i++) {
      C->h_ptrs[C->ptr_cap + first + i] = slots[i];
      if (reinterpret_cast<uintptr_t>(slots[i]) % 16) fill_ok = false;
    }
  }
  fa::SlotOut slot_out{};
  if (fill_ok) {
    FA_CU(cudaMemcpyAsync(C->d_ptrs + C->ptr_cap + first, C->h_ptrs + C->ptr_cap + first, (size_t)n * sizeof(void*),
                          cudaMemcpyHostToDevice, C->stream));
    slot_out = fa::SlotOut{C->d_ptrs + C->ptr_cap + first, slot_kind, slot_pitch, slot_plane};
  }
  long long* d_idx = C->d_idx + first;
  if (!planes && C->planes && !C->ref_conj_rows) {  // a plane-path correlator falling back to cuFFT
    FA_CU(cudaStreamSynchronize(C->stream));
    FA_TRY(dalloc_t(C->ctx, (size_t)C->n_el * C->cap, &C->real, C->allocs));
    FA_TRY(dalloc_t(C->ctx, (size_t)C->n_complex, &C->ref_conj_rows, C->allocs));
    FA_CU(fa::launch_plane_to_rows(C->pd, C->ref_conj, C->ref_conj_rows, C->stream));
  }
  const double2* ref_rows = C->planes ? C->ref_conj_rows : C->ref_conj;
  for (int c0 = 0; c0 < n;) {
    int m = C->cap;  // the largest power-of-two batch that fits the rest
    while (m > n - c0) m >>= 1;
    double* surf = surface ? surface + (size_t)c0 * C->n_el : nullptr;
    if (planes) {
      const int nb = fa::plane_blocks_per_frame(C->pd);
      fa::SlotOut so = slot_out;
      if (fill_ok) so.ptrs += c0;
      FA_CU(fa::launch_plane_rows_fwd(C->pd, d_ptrs + c0, in_kind, m, C->wy, C->wx, C->tw_x, C->spec, C->stream,
                                      fill_ok ? &so : nullptr));
      if (C->pd.split)
        FA_CU(fa::launch_plane_yz_split(C->pd, C->spec, C->ref_conj, C->tw_y, C->tw_z, m, false, C->stream));
      else
        FA_CU(fa::launch_plane_yz(C->pd, C->spec, C->spec, C->ref_conj, C->tw_y, m, false, C->stream));
      FA_CU(fa::launch_plane_rows_inv_argmax(C->pd, C->spec, m, C->tw_x, C->bval, C->bidx, surf, C->stream));
      FA_CU(fa::launch_phase_argmax_final(C->bval, C->bidx, nb, m, d_idx + c0, C->stream));
      g_launches += C->pd.split ? 6 : 4;
    } else {
      cufftHandle fwd, inv;
      FA_TRY(correlator_plans(C, m, &fwd, &inv));
      FA_CU(fa::launch_phase_window(d_ptrs + c0, in_kind, C->wy, C->wx, C->ny, C->nx, C->n_el, m, C->real,
                                    C->stream));
      if (cufftExecD2Z(fwd, C->real, reinterpret_cast<cufftDoubleComplex*>(C->spec)) != CUFFT_SUCCESS)
        return fail(FA_ERR_CUDA, "cufftExecD2Z failed");
      FA_CU(fa::launch_phase_normalise(C->spec, ref_rows, C->n_complex, m, C->stream));
      if (cufftExecZ2D(inv, reinterpret_cast<cufftDoubleComplex*>(C->spec), C->real) != CUFFT_SUCCESS)
        return fail(FA_ERR_CUDA, "cufftExecZ2D failed");
      FA_CU(fa::launch_phase_argmax(C->real, C->n_el, m, C->bval, C->bidx, C->n_blocks, d_idx + c0, C->stream));
      if (surf)
        FA_CU(cudaMemcpyAsync(surf, C->real, (size_t)m * C->n_el * sizeof(double), cudaMemcpyDeviceToDevice,
                              C->stream));
      g_launches += 4;  // window, normalise, two argmax stages (the FFTs are cuFFT's)
    }
    c0 += m;
  }
  if (slots_written) *slots_written = fill_ok;
  return FA_OK;
}

}  // namespace fa_rt

namespace fa_rt {

// Peak index -> signed integer shift (VolumePhaseCorrelator.cpp:94-103).
void unravel_shift(const fa_correlator* C, long long idx, double* shift) {
  long long x = idx % C->nx;
  long long y = (idx / C->nx) % C->ny;
  long long z = idx / ((long long)C->nx * C->ny);
  if (x > C->nx / 2) x -= C->nx;
  if (y > C->ny / 2) y -= C->ny;
  if (z > C->nz / 2) z -= C->nz;
  shift[0] = (double)x;
  shift[1] = (double)y;
  shift[2] = (double)z;
}

}  // namespace fa_rt

namespace {

fa_status correlator_read(fa_correlator* C, int n, double* shifts) {
  FA_CU(cudaMemcpyAsync(C->h_idx, C->d_idx, (size_t)n * sizeof(long long), cudaMemcpyDeviceToHost, C->stream));
  FA_CU(cudaStreamSynchronize(C->stream));
  for (int i = 0; i < n; i++) unravel_shift(C, C->h_idx[i], shifts + 3 * i);
  return FA_OK;
}

}  // namespace

namespace fa_rt {

fa_status correlator_plans(fa_correlator* C, int batch, cufftHandle* fwd, cufftHandle* inv) {
  auto it = C->plans.find(batch);
  if (it != C->plans.end()) {
    *fwd = it->second.first;
    *inv = it->second.second;
    return FA_OK;
  }
  int dims[3] = {C->nz, C->ny, C->nx};
  int rank = 3;
  int* d = dims;
  if (C->nz == 1) {
    rank = 2;
    d = dims + 1;
    if (C->ny == 1) {
      rank = 1;
      d = dims + 2;
    }
  }
  // Basic layout: batches contiguous, n_el reals apart on the real side, n_complex on the complex side.
  cufftHandle f = 0, v = 0;
  size_t wf = 0, wv = 0;
  if (cufftCreate(&f) != CUFFT_SUCCESS || cufftCreate(&v) != CUFFT_SUCCESS || cufftSetAutoAllocation(f, 0) ||
      cufftSetAutoAllocation(v, 0) ||
      cufftMakePlanMany(f, rank, d, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, batch, &wf) != CUFFT_SUCCESS ||
      cufftMakePlanMany(v, rank, d, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, batch, &wv) != CUFFT_SUCCESS) {
    if (f) cufftDestroy(f);
    if (v) cufftDestroy(v);
    return fail(FA_ERR_CUDA, "cufftMakePlanMany failed");
  }
  C->plans[batch] = {f, v};
  const size_t need = std::max(wf, wv);
  if (need > C->work_bytes) {  // a larger shared work area, given to every plan
    FA_CU(cudaStreamSynchronize(C->stream));
    dfree_all(C->ctx, C->work_allocs);
    C->work = nullptr;
    C->work_bytes = 0;
    FA_TRY(dalloc(C->ctx, need, &C->work, C->work_allocs));
    C->work_bytes = need;
    for (auto& pl : C->plans)
      if (cufftSetWorkArea(pl.second.first, C->work) != CUFFT_SUCCESS ||
          cufftSetWorkArea(pl.second.second, C->work) != CUFFT_SUCCESS)
        return fail(FA_ERR_CUDA, "cufftSetWorkArea failed");
  } else if (cufftSetWorkArea(f, C->work) != CUFFT_SUCCESS || cufftSetWorkArea(v, C->work) != CUFFT_SUCCESS) {
    return fail(FA_ERR_CUDA, "cufftSetWorkArea failed");
  }
  cufftSetStream(f, C->stream);
  cufftSetStream(v, C->stream);
  *fwd = f;
  *inv = v;
  return FA_OK;
}

}  // namespace fa_rt

namespace {

fa_status correlator_create_impl(fa_context* ctx, const void* reference, bool ref_device, int nz, int ny, int nx,
                                 int cap, fa_correlator** out) {
  if (!ctx || !reference || !out || nz < 1 || ny < 1 || nx < 1) return fail(FA_ERR_BAD_ARG, "bad arguments");
  FA_CU(cudaSetDevice(ctx->device));
  fa_correlator* C = new fa_correlator;
  C->ctx = ctx;
  C->nz = nz;
  C->ny = ny;
  C->nx = nx;
  C->n_el = (long long)nz * ny * nx;
  C->n_complex = (long long)nz * ny * (nx / 2 + 1);
  // batch cap: a power of two, at most the requested cap and what 4 GiB of FP64 buffers hold
  {
    const long long per = C->n_el * 8 + C->n_complex * 16;
    const long long fit = std::max<long long>(1, (4LL << 30) / per);
    int c = 1;
    while (c * 2 <= cap && c * 2 <= fit) c *= 2;
    C->cap = c;
  }
  auto cleanup = [&](fa_status st) {
    std::string keep = g_err;
    fa_correlator_destroy(C);
    g_err = keep;
    return st;
  };
  if (cudaStreamCreateWithFlags(&C->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "stream"));
  fa_status st;
  if ((st = dalloc_t(ctx, (size_t)ny, &C->wy, C->allocs)) != FA_OK) return cleanup(st);
  if ((st = dalloc_t(ctx, (size_t)nx, &C->wx, C->allocs)) != FA_OK) return cleanup(st);
  C->planes = fa::plane_dims(nz, ny, nx, &C->pd);
  if (!C->planes)
    if ((st = dalloc_t(ctx, (size_t)C->n_el * C->cap, &C->real, C->allocs)) != FA_OK) return cleanup(st);
  if ((st = dalloc_t(ctx, (size_t)C->n_complex * C->cap, &C->spec, C->allocs)) != FA_OK) return cleanup(st);
  if ((st = dalloc_t(ctx, (size_t)C->n_complex, &C->ref_conj, C->allocs)) != FA_OK) return cleanup(st);
  if ((st = dalloc_t(ctx, (size_t)C->n_el, &C->vol, C->allocs)) != FA_OK) return cleanup(st);
  C->n_blocks = (int)std::min<long long>(std::max(1, 148 * 4 / C->cap), (C->n_el + 255) / 256);
  {
    const int nb = std::max(C->n_blocks, C->planes ? fa::plane_blocks_per_frame(C->pd) : 0);
    if ((st = dalloc_t(ctx, (size_t)nb * C->cap, &C->bval, C->allocs)) != FA_OK) return cleanup(st);
    if ((st = dalloc_t(ctx, (size_t)nb * C->cap, &C->bidx, C->allocs)) != FA_OK) return cleanup(st);
  }
  // Square-root Hann window in x and y, 1 along z (VolumePhaseCorrelator.cpp:141-166).
  auto hann = [](int n) {
    std::vector<double> w(n, 1.0);
    if (n > 1) {
      const double PI = 3.14159265358979323846;
      double f = 2.0 * PI / (n - 1);
      for (int i = 0; i < n; i++) w[i] = std::sqrt(0.5 * (1 - std::cos(f * i)));
    }
    return w;
  };
  std::vector<double> wy = hann(ny), wx = hann(nx);
  if (cudaMemcpy(C->wy, wy.data(), wy.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(C->wx, wx.data(), wx.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "window upload"));
  if (cudaMemcpyAsync(C->vol, reference, (size_t)C->n_el * sizeof(float),
                      ref_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "reference upload"));
  if ((st = correlator_reserve(C, 1)) != FA_OK) return cleanup(st);
  C->h_ptrs[0] = C->vol;
  if (cudaMemcpyAsync(C->d_ptrs, C->h_ptrs, sizeof(void*), cudaMemcpyHostToDevice, C->stream) != cudaSuccess)
    return cleanup(fail(FA_ERR_CUDA, "pointer upload"));
  if (C->planes) {
    std::vector<double2> tx, ty, tz;
    fa::plane_twiddles(C->pd, &tx, &ty, &tz);
    if ((st = dalloc_t(ctx, tx.size(), &C->tw_x, C->allocs)) != FA_OK) return cleanup(st);
    if ((st = dalloc_t(ctx, ty.size(), &C->tw_y, C->allocs)) != FA_OK) return cleanup(st);
    if ((st = dalloc_t(ctx, std::max<size_t>(tz.size(), 1), &C->tw_z, C->allocs)) != FA_OK) return cleanup(st);
    if (cudaMemcpy(C->tw_x, tx.data(), tx.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(C->tw_y, ty.data(), ty.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess ||
        (!tz.empty() &&
         cudaMemcpy(C->tw_z, tz.data(), tz.size() * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess))
      return cleanup(fail(FA_ERR_CUDA, "twiddle upload"));
    const cudaError_t e_fwd =
        fa::launch_plane_rows_fwd(C->pd, C->d_ptrs, FA_F32, 1, C->wy, C->wx, C->tw_x, C->spec, C->stream);
    const cudaError_t e_yz =
        e_fwd != cudaSuccess ? e_fwd
        : C->pd.split
            ? fa::launch_plane_yz_split(C->pd, C->spec, C->ref_conj, C->tw_y, C->tw_z, 1, true, C->stream)
            : fa::launch_plane_yz(C->pd, C->spec, C->ref_conj, nullptr, C->tw_y, 1, true, C->stream);
    if (e_yz != cudaSuccess) return cleanup(fail(FA_ERR_CUDA, "reference spectrum"));
  } else {
    cufftHandle fwd1, inv1;
    if ((st = correlator_plans(C, 1, &fwd1, &inv1)) != FA_OK) return cleanup(st);
    if (fa::launch_phase_window(C->d_ptrs, FA_F32, C->wy, C->wx, ny, nx, C->n_el, 1, C->real, C->stream) !=
        cudaSuccess)
      return cleanup(fail(FA_ERR_CUDA, "window kernel"));
    if (cufftExecD2Z(fwd1, C->real, reinterpret_cast<cufftDoubleComplex*>(C->spec)) != CUFFT_SUCCESS)
      return cleanup(fail(FA_ERR_CUDA, "cufftExecD2Z failed"));
    if (fa::launch_phase_conj(C->spec, C->ref_conj, C->n_complex, C->stream) != cudaSuccess)
      return cleanup(fail(FA_ERR_CUDA, "conj kernel"));
  }
  {
    const cudaError_t e = cudaStreamSynchronize(C->stream);
    if (e != cudaSuccess)
      return cleanup(fail(FA_ERR_CUDA, std::string("correlator set-up: ") + cudaGetErrorString(e)));
  }
  *out = C;
  return FA_OK;
}

}  // namespace

extern "C" fa_status fa_correlator_create(fa_context* ctx, const float* reference, int nz, int ny, int nx,
                                          fa_correlator** out) {
  return correlator_create_impl(ctx, reference, false, nz, ny, nx, 1, out);
}

extern "C" fa_status fa_correlator_destroy(fa_correlator* C) {
  if (!C) return fail(FA_ERR_BAD_ARG, "NULL correlator");
  cudaSetDevice(C->ctx->device);
  if (C->stream) cudaStreamSynchronize(C->stream);
  for (auto& pl : C->plans) {
    cufftDestroy(pl.second.first);
    cufftDestroy(pl.second.second);
  }
  C->plans.clear();
  dfree_all(C->ctx, C->work_allocs);
  if (C->h_ptrs) cudaFreeHost(C->h_ptrs);
  if (C->h_idx) cudaFreeHost(C->h_idx);
  if (C->stream) cudaStreamDestroy(C->stream);
  dfree_all(C->ctx, C->ptr_allocs);
  dfree_all(C->ctx, C->allocs);
  delete C;
  return FA_OK;
}

extern "C" fa_status fa_correlator_shift(fa_correlator* C, const float* volume, double* shift) {
  if (!C || !volume || !shift) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(C->mu);
  FA_CU(cudaSetDevice(C->ctx->device));
  FA_CU(cudaMemcpyAsync(C->vol, volume, (size_t)C->n_el * sizeof(float), cudaMemcpyHostToDevice, C->stream));
  const void* v = C->vol;
  FA_TRY(correlator_enqueue(C, &v, FA_F32, 1));
  return correlator_read(C, 1, shift);
}

extern "C" fa_status fa_correlator_shift_device(fa_correlator* C, const float* volume_device, double* shift) {
  if (!C || !volume_device || !shift) return fail(FA_ERR_BAD_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(C->mu);
  FA_CU(cudaSetDevice(C->ctx->device));
  const void* v = volume_device;
  FA_TRY(correlator_enqueue(C, &v, FA_F32, 1));
  return correlator_read(C, 1, shift);
}

// ================================================================== test hooks ====================

extern "C" fa_status fa_test_plane_tables(int nz, int ny, int nx, double* tw_x, int cap_x, int* n_x, int* x_post,
                                          double* tw_y, int cap_y, int* n_y, int* rows_per_cta, int* planes_per_cta) {
  if (!tw_x || !n_x || !x_post || !tw_y || !n_y || !rows_per_cta || !planes_per_cta)
    return fail(FA_ERR_BAD_ARG, "NULL argument");
  fa::PlaneDims d{};
  if (!fa::plane_dims(nz, ny, nx, &d)) return fail(FA_ERR_UNSUPPORTED, "dimensions outside the fused plane passes");
  std::vector<double2> tx, ty, tz;
  fa::plane_twiddles(d, &tx, &ty, &tz);
  if ((int)tx.size() != d.n_twx || (int)ty.size() != d.n_twy) return fail(FA_ERR_STATE, "twiddle table size");
  if ((int)tx.size() > cap_x || (int)ty.size() > cap_y) return fail(FA_ERR_BAD_ARG, "output arrays too small");
  for (size_t i = 0; i < tx.size(); i++) {
    tw_x[2 * i] = tx[i].x;
    tw_x[2 * i + 1] = tx[i].y;
  }
  for (size_t i = 0; i < ty.size(); i++) {
    tw_y[2 * i] = ty[i].x;
    tw_y[2 * i + 1] = ty[i].y;
  }
  *n_x = d.n_twx;
  *x_post = d.tw_x_post;
  *n_y = d.n_twy;
  *rows_per_cta = 1 << d.log2G;
  *planes_per_cta = d.PP;
  return FA_OK;
}

extern "C" fa_status fa_test_correlation_surface(fa_correlator* C, const float* volume, int use_planes,
                                                 double* surface) {
  if (!C || !volume || !surface) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (use_planes && !C->planes) return fail(FA_ERR_UNSUPPORTED, "dimensions outside the fused plane passes");
  std::lock_guard<std::mutex> lk(C->mu);
  FA_CU(cudaSetDevice(C->ctx->device));
  std::vector<Alloc> tmp;
  double* d_surf = nullptr;
  FA_TRY(dalloc_t(C->ctx, (size_t)C->n_el, &d_surf, tmp));
  auto done = [&](fa_status r) {
    cudaStreamSynchronize(C->stream);
    dfree_all(C->ctx, tmp);
    return r;
  };
  if (cudaMemcpyAsync(C->vol, volume, (size_t)C->n_el * sizeof(float), cudaMemcpyHostToDevice, C->stream) !=
      cudaSuccess)
    return done(fail(FA_ERR_CUDA, "volume upload"));
  const void* v = C->vol;
  fa_status st = correlator_enqueue(C, &v, FA_F32, 1, d_surf, use_planes != 0);
  if (st != FA_OK) return done(st);
  if (cudaMemcpyAsync(surface, d_surf, (size_t)C->n_el * sizeof(double), cudaMemcpyDeviceToHost, C->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(C->stream) != cudaSuccess)
    return done(fail(FA_ERR_CUDA, "surface read"));
  return done(FA_OK);
}

extern "C" fa_status fa_test_downsample(fa_context* ctx, const void* volume, fa_dtype dtype, int nz, int ny, int nx,
                                        int factor, float* out) {
  if (!ctx || !volume || !out || nz < 1 || ny < 1 || nx < 1 || factor < 1 || (dtype != FA_F32 && dtype != FA_U16))
    return fail(FA_ERR_BAD_ARG, "bad arguments");
  FA_CU(cudaSetDevice(ctx->device));
  const size_t n_in = (size_t)nz * ny * nx;
  const size_t n_out = (size_t)nz * ((ny + factor - 1) / factor) * ((nx + factor - 1) / factor);
  std::vector<Alloc> tmp;
  auto done = [&](fa_status st) {
    std::string keep = g_err;
    dfree_all(ctx, tmp);
    g_err = keep;
    return st;
  };
  void* d_in;
  float* d_out;
  fa_status st;
  if ((st = dalloc(ctx, n_in * dtype_size(dtype), &d_in, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, n_out, &d_out, tmp)) != FA_OK) return done(st);
  cudaError_t e = cudaMemcpy(d_in, volume, n_in * dtype_size(dtype), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = fa::launch_downsample(d_in, dtype, nz, ny, nx, factor, d_out, 0);
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, n_out * sizeof(float), cudaMemcpyDeviceToHost);
  g_launches += 1;
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("downsample: ") + cudaGetErrorString(e)));
  return done(FA_OK);
}

extern "C" fa_status fa_test_tr_subproblem(fa_context* ctx, int nD, int n_dim, const double* H, const double* g,
                                           double radius, double* p, int* on_boundary) {
  if (!ctx || !H || !g || !p || !on_boundary || nD < 1 || (n_dim != 2 && n_dim != 3))
    return fail(FA_ERR_BAD_ARG, "bad arguments");
  FA_CU(cudaSetDevice(ctx->device));
  const int P = nD * n_dim, nn = n_dim * n_dim;
  std::vector<double> hd((size_t)nD * nn, 0.0), hl((size_t)nD * nn, 0.0);
  for (int b = 0; b < nD; b++)
    for (int a = 0; a < n_dim; a++)
      for (int c = 0; c < n_dim; c++) {
        hd[(size_t)b * nn + a * n_dim + c] = H[(size_t)(b * n_dim + a) * P + b * n_dim + c];
        if (b > 0) hl[(size_t)b * nn + a * n_dim + c] = H[(size_t)(b * n_dim + a) * P + (b - 1) * n_dim + c];
      }
  std::vector<Alloc> tmp;
  double *dHd, *dHl, *dg, *dp, *work;
  int* db;
  auto done = [&](fa_status st) {
    std::string keep = g_err;
    dfree_all(ctx, tmp);
    g_err = keep;
    return st;
  };
  fa_status st;
  if ((st = dalloc_t(ctx, hd.size(), &dHd, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, hl.size(), &dHl, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, (size_t)P, &dg, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, (size_t)P, &dp, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, (size_t)P * (2 * n_dim) + 3 * (size_t)P, &work, tmp)) != FA_OK) return done(st);
  if ((st = dalloc_t(ctx, 1, &db, tmp)) != FA_OK) return done(st);
  cudaError_t e = cudaMemcpy(dHd, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dHl, hl.data(), hl.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dg, g, (size_t)P * sizeof(double), cudaMemcpyHostToDevice);
  double hinf, mindiag;
  fa::band_bounds(hd.data(), hl.data(), nD, n_dim, &hinf, &mindiag);
  if (e == cudaSuccess) e = fa::launch_test_subproblem(dHd, dHl, nD, n_dim, hinf, mindiag, dg, radius, dp, db, work, 0);
  if (e == cudaSuccess) e = cudaMemcpy(p, dp, (size_t)P * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(on_boundary, db, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return done(fail(FA_ERR_CUDA, std::string("subproblem: ") + cudaGetErrorString(e)));
  return done(FA_OK);
}

// ================================================================== aligner =======================

namespace {

void aligner_release_reference(fa_aligner* A) {
  aligner_release_results(A);
  for (auto& c : A->batch_cache) batch_cache_release(A->ctx, &c);
  dfree_all(A->ctx, A->smooth_allocs);
  A->smooth_kx = A->smooth_ky = A->smooth_tmp = A->smooth_out = nullptr;
  A->smooth_nkx = A->smooth_nky = 0;
  for (fa_frame* f : A->slots) fa_deregister_frame(f);
  A->slots.clear();
  A->slot_kind = -1;
  if (A->corr) fa_correlator_destroy(A->corr);
  A->corr = nullptr;
  if (A->ref) fa_reference_destroy(A->ref);
  A->ref = nullptr;
  dfree_all(A->ctx, A->ref_allocs);
}

}  // namespace

namespace fa_rt {

size_t dtype_size(fa_dtype t) { return t == FA_F32 ? 4 : 2; }

}  // namespace fa_rt

namespace fa_rt {

// Slot storage for a batch: raw uint16 counts (the kernels add the +1) when the input is uint16,
// unsmoothed and the reference is mixed precision; otherwise FP16 / FP32 values with the +1 applied.
int slot_kind_for(const fa_aligner* A, fa_dtype dtype) {
  if (A->prm.precision == FA_PREC_MIXED)
    return (dtype == FA_U16 && !(A->prm.smoothing > 0)) ? fa::kFrameRawU16 : fa::kFrameF16;
  return fa::kFrameF32;
}

}  // namespace fa_rt

namespace {

fa_status aligner_grow(fa_aligner* A, int n, int kind, size_t staging_need) {
  if (A->slot_kind != kind) {
    for (fa_frame* f : A->slots) fa_deregister_frame(f);
    A->slots.clear();
    A->slot_kind = kind;
  }
  while ((int)A->slots.size() < n) {
    fa_frame* F = nullptr;
    FA_TRY(frame_alloc(A->ref, kind, &F));
    A->slots.push_back(F);
  }
  const bool need_vols = A->prm.spatial_binning > 1;
  if (A->staging_bytes < staging_need || (need_vols && (int)A->vols_count < n)) {
    FA_CU(cudaStreamSynchronize(A->corr->stream));
    dfree_all(A->ctx, A->allocs);
    A->staging = nullptr;
    A->staging_bytes = 0;
    A->vols = nullptr;
    A->vols_count = 0;
    if (staging_need) {
      FA_TRY(dalloc(A->ctx, staging_need, &A->staging, A->allocs));
      A->staging_bytes = staging_need;
    }
    if (need_vols) {
      FA_TRY(dalloc_t(A->ctx, (size_t)n * A->dz * A->dy * A->dx, &A->vols, A->allocs));
      A->vols_count = (size_t)n;
    }
  }
  return FA_OK;
}

// Solve groups of one call, as frame boundaries {0, ..., n}: groups of `chunk` frames (a last
// remainder under chunk / 2 joins the group before it). Every group's solve is queued on its own
// stream behind its own peaks, so the solves of the first groups run while the later groups upload
// (host frames) and correlate, and the correlation kernels fill the SMs that the one-CTA-per-frame
// solve steps leave idle; the fused pass of one group still has chunk x tiles-per-frame work items
// (8 x 1024 for the 512 x 512 x 16 workload) to fill the GPU. Frames are independent, so the results
// do not depend on the grouping. (Measured on one B200, 50 frames of 512 x 512 x 16: one group
// 4959 frames/s with frames in HBM; two groups 5385; groups of 16 5555; groups of 8 5568, and from
// host memory 4088 / 4248 / 4400 for two groups / 16 / 8.)
std::vector<int> solve_groups(int n, int chunk) {
  std::vector<int> b;
  for (int i = 0; i == 0 || i + chunk / 2 < n; i += chunk) b.push_back(i);
  b.push_back(n);
  return b;
}

fa_status aligner_run(fa_aligner* A, const void* const* frames, fa_dtype dtype, int n, bool device_src,
                      double* D_out, fa_align_stats* stats) {
  if (!A->ref) return fail(FA_ERR_STATE, "Reference imaging not yet set");  // FrameWarpAligner.cpp:119
  if (!frames || n <= 0 || !D_out) return fail(FA_ERR_BAD_ARG, "bad arguments");
  if (dtype != FA_F32 && dtype != FA_U16) return fail(FA_ERR_BAD_ARG, "frames must be FA_F32 or FA_U16");
  for (int i = 0; i < n; i++)
    if (!frames[i]) return fail(FA_ERR_BAD_ARG, "NULL frame pointer");
  FA_CU(cudaSetDevice(A->ctx->device));
  const long long N = A->ref->N;
  const size_t raw_bytes = (size_t)N * dtype_size(dtype);
  const int kind = slot_kind_for(A, dtype);
  // Raw frames (host frames via a staging copy) go through the correlator as they are and into the
  // slots with the +1 offset (count + 1 for uint16 slots).
  FA_TRY(aligner_grow(A, n, kind, device_src ? 0 : (size_t)n * raw_bytes));
  cudaStream_t s = A->corr->stream;
  if (!A->ev0) {
    FA_CU(cudaEventCreate(&A->ev0));
    FA_CU(cudaEventCreate(&A->ev1));
    FA_CU(cudaEventCreate(&A->ev_corr));
  }
  FA_CU(cudaEventRecord(A->ev0, s));
  // Host frames upload on a copy stream in chunks of kChunk; each chunk's conversion and phase
  // correlation wait only for its own uploads, so they overlap the uploads of the chunks after it.
  constexpr int kChunk = 8;
  const int chunk = device_src ? n : kChunk;
  if (!device_src) {
    if (!A->copy_stream) FA_CU(cudaStreamCreateWithFlags(&A->copy_stream, cudaStreamNonBlocking));
    // one event per upload chunk: chunks never straddle a solve group, so a group adds at most one
    while ((int)A->copy_ev.size() < (n + chunk - 1) / chunk + (int)solve_groups(n, kChunk).size()) {
      cudaEvent_t e;
      FA_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      A->copy_ev.push_back(e);
    }
    // the copy stream starts after everything already queued on s (the previous call's readers of
    // the staging buffer)
    FA_CU(cudaEventRecord(A->ev1, s));
    FA_CU(cudaStreamWaitEvent(A->copy_stream, A->ev1, 0));
  }
  // Whatever the outcome, no upload from the caller's frames is left in flight when this returns
  // (after success they are complete already: the conversions waited for every one of them).
  struct DrainCopies {
    cudaStream_t cs;
    ~DrainCopies() {
      if (cs) cudaStreamSynchronize(cs);
    }
  } drain{device_src ? nullptr : A->copy_stream};
  FA_TRY(correlator_reserve(A->corr, n));
  const std::vector<int> gb = solve_groups(n, kChunk);  // group g: frames [gb[g], gb[g + 1])
  const int n_groups = (int)gb.size() - 1;
  while ((int)A->batch_cache.size() < n_groups) A->batch_cache.emplace_back();
  while ((int)A->group_ev.size() < n_groups) {
    cudaEvent_t e;
    FA_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    A->group_ev.push_back(e);
  }
  fa_correlator* C = A->corr;
  std::vector<const void*> raw((size_t)n), cin((size_t)n);
  std::vector<void*> slot_ptrs((size_t)n);
  int cin_kind = dtype;
  // Without smoothing or binning the correlator's first pass reads the raw frames anyway: it also
  // writes their slots (count + 1), in place of a separate conversion pass.
  const bool fuse_slots = A->prm.smoothing <= 0 && A->prm.spatial_binning <= 1;
  for (int c0 = 0, ci = 0, g = 0; c0 < n; ci++) {
    while (gb[g + 1] <= c0) g++;
    const int m = std::min(chunk, gb[g + 1] - c0);
    if (!device_src) {
      for (int i = c0; i < c0 + m; i++) {
        void* dst = static_cast<char*>(A->staging) + (size_t)i * raw_bytes;
        FA_CU(cudaMemcpyAsync(dst, frames[i], raw_bytes, cudaMemcpyHostToDevice, A->copy_stream));
      }
      FA_CU(cudaEventRecord(A->copy_ev[ci], A->copy_stream));
      FA_CU(cudaStreamWaitEvent(s, A->copy_ev[ci], 0));
    }
    for (int i = c0; i < c0 + m; i++) {
      fa_frame* F = A->slots[i];
      raw[i] = device_src ? frames[i] : static_cast<const char*>(A->staging) + (size_t)i * raw_bytes;
      if (A->prm.smoothing > 0) {  // smoothStack, then + 1 (FrameWarpAligner.cpp:139-142)
        FA_TRY(aligner_smooth(A, raw[i], dtype, s));
        FA_CU(fa::launch_to_slot(A->smooth_out, FA_F32, F->data, kind, A->nz, A->ny, A->nx, F->job.fpitch,
                                 F->job.fplane, true, s));
      } else if (!fuse_slots) {
        FA_CU(fa::launch_to_slot(raw[i], dtype, F->data, kind, A->nz, A->ny, A->nx, F->job.fpitch, F->job.fplane,
                                 true, s));
      }
      slot_ptrs[i] = F->data;
      if (!fuse_slots) g_launches += 1;
      // Phase correlation on the raw frames (FrameWarpAligner.cpp:181-190), downsampled when binning.
      if (A->prm.spatial_binning > 1) {
        float* vol = A->vols + (size_t)i * A->dz * A->dy * A->dx;
        FA_CU(fa::launch_downsample(raw[i], dtype, A->nz, A->ny, A->nx, A->prm.spatial_binning, vol, s));
        g_launches += 1;
        cin[i] = vol;
        cin_kind = FA_F32;
      } else {
        cin[i] = raw[i];
      }
    }
    bool written = false;
    FA_TRY(correlator_enqueue(C, cin.data() + c0, cin_kind, m, nullptr, true, c0, fuse_slots ? slot_ptrs.data() + c0 : nullptr,
                              kind, A->slots[c0]->job.fpitch, A->slots[c0]->job.fplane, &written));
    if (fuse_slots && !written) {  // the correlator took the cuFFT path: a separate conversion
      for (int i = c0; i < c0 + m; i++) {
        fa_frame* F = A->slots[i];
        FA_CU(fa::launch_to_slot(raw[i], dtype, F->data, kind, A->nz, A->ny, A->nx, F->job.fpitch, F->job.fplane,
                                 true, s));
        g_launches += 1;
      }
    }
    c0 += m;
    if (c0 == gb[g + 1]) FA_CU(cudaEventRecord(A->group_ev[g], s));  // a group's frames and peaks are ready
  }
  FA_CU(cudaEventRecord(A->ev_corr, s));
  // Every group's solve is queued at once, each on its first slot's stream behind its own frames and
  // peaks: the first group's solve runs while the later groups upload and correlate, and a later
  // group starts as soon as its peaks are there. The rigid starts are unravelled and scaled by the
  // binning on the device (FrameWarpAligner.cpp:181-190).
  std::vector<fa_frame*> batch(A->slots.begin(), A->slots.begin() + n);
  fa_status r = FA_OK;
  int queued = 0;
  for (int g = 0; g < n_groups && r == FA_OK; g++) {
    const int g0 = gb[g], g1 = gb[g + 1];
    const PeakStart ps{C->d_idx + g0, C->nx, C->ny, C->nz, A->prm.spatial_binning, A->group_ev[g]};
    r = align_batch_enqueue(batch.data() + g0, g1 - g0, nullptr, A->prm.max_iterations, nullptr, &A->batch_cache[g],
                            &ps);
    // the last group's stream also holds whatever its failed enqueue left queued
    queued = g + 1;
  }
  for (int g = 0; g < queued; g++) {
    const int g0 = gb[g], g1 = gb[g + 1];
    if (r != FA_OK) {  // drain without reading, keeping the first error
      std::string keep = g_err;
      cudaStreamSynchronize(batch[g0]->stream);
      g_err = keep;
      continue;
    }
    r = align_batch_finish(batch.data() + g0, g1 - g0, &A->batch_cache[g], D_out + (size_t)g0 * 3 * A->ref->nD,
                           stats ? stats + g0 : nullptr);
  }
  if (r != FA_OK) return r;
  // the end of the call: after every group's solve
  for (int g = 1; g < n_groups; g++) {
    FA_CU(cudaEventRecord(A->group_ev[g], batch[gb[g]]->stream));
    FA_CU(cudaStreamWaitEvent(batch[0]->stream, A->group_ev[g], 0));
  }
  FA_CU(cudaEventRecord(A->ev1, batch[0]->stream));
  FA_CU(cudaEventSynchronize(A->ev1));
  float ms = 0;
  FA_CU(cudaEventElapsedTime(&ms, A->ev0, A->ev1));
  A->last_ms = ms;
  FA_CU(cudaEventElapsedTime(&ms, A->ev0, A->ev_corr));
  A->last_corr_ms = ms;
  return FA_OK;
}

}  // namespace

namespace fa_rt {

std::vector<float> gaussian_kernel(double sigma) {
  // cv::getGaussianKernel for a float image: size cvRound(8 sigma + 1) | 1, weights exp(-x^2/(2 s^2))
  // rounded to float, summed in double, scaled by the reciprocal of the sum
  const int n = (int)std::nearbyint(sigma * 8 + 1) | 1;
  if (n > 257) return {};
  std::vector<float> k((size_t)n);
  const double scale2 = -0.5 / (sigma * sigma);
  double sum = 0;
  for (int i = 0; i < n; i++) {
    const double x = i - (n - 1) * 0.5;
    k[i] = (float)std::exp(scale2 * x * x);
    sum += k[i];
  }
  sum = 1.0 / sum;
  for (int i = 0; i < n; i++) k[i] = (float)(k[i] * sum);
  return k;
}

fa_status aligner_smooth(fa_aligner* A, const void* raw, fa_dtype dtype, cudaStream_t s) {
  if (!(A->prm.smoothing > 0)) return FA_OK;
  const size_t N = (size_t)A->nz * A->ny * A->nx;
  if (!A->smooth_kx) {
    const std::vector<float> kx = gaussian_kernel(A->prm.smoothing), ky = gaussian_kernel(1.0);
    FA_TRY(dalloc_t(A->ctx, kx.size(), &A->smooth_kx, A->smooth_allocs));
    FA_TRY(dalloc_t(A->ctx, ky.size(), &A->smooth_ky, A->smooth_allocs));
    FA_TRY(dalloc_t(A->ctx, N, &A->smooth_tmp, A->smooth_allocs));
    FA_TRY(dalloc_t(A->ctx, N, &A->smooth_out, A->smooth_allocs));
    FA_CU(cudaMemcpy(A->smooth_kx, kx.data(), kx.size() * sizeof(float), cudaMemcpyHostToDevice));
    FA_CU(cudaMemcpy(A->smooth_ky, ky.data(), ky.size() * sizeof(float), cudaMemcpyHostToDevice));
    A->smooth_nkx = (int)kx.size();
    A->smooth_nky = (int)ky.size();
  }
  FA_CU(fa::launch_smooth(raw, dtype, A->nz, A->ny, A->nx, A->smooth_kx, A->smooth_nkx, A->smooth_ky, A->smooth_nky,
                          A->smooth_tmp, A->smooth_out, s));
  g_launches += 2;
  return FA_OK;
}

}  // namespace fa_rt

extern "C" fa_status fa_aligner_create(fa_context* ctx, const fa_aligner_params* params, fa_aligner** out) {
  if (!ctx || !params || !out) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (!(params->smoothing >= 0.0) || (params->smoothing > 0.0 && gaussian_kernel(params->smoothing).empty()))
    return fail(FA_ERR_BAD_ARG, "smoothing must be >= 0 and at most 32 (a kernel of at most 257 taps)");
  if (params->spatial_binning < 1) return fail(FA_ERR_BAD_ARG, "spatial_binning must be >= 1");
  if (params->precision != FA_PREC_F32 && params->precision != FA_PREC_MIXED)
    return fail(FA_ERR_BAD_ARG, "unknown precision");
  fa_aligner* A = new fa_aligner;
  A->ctx = ctx;
  A->prm = *params;
  *out = A;
  return FA_OK;
}

extern "C" fa_status fa_aligner_destroy(fa_aligner* A) {
  if (!A) return fail(FA_ERR_BAD_ARG, "NULL aligner");
  cudaSetDevice(A->ctx->device);
  aligner_release_reference(A);
  dfree_all(A->ctx, A->allocs);
  if (A->stream) cudaStreamDestroy(A->stream);
  if (A->ev0) cudaEventDestroy(A->ev0);
  if (A->ev1) cudaEventDestroy(A->ev1);
  if (A->ev_corr) cudaEventDestroy(A->ev_corr);
  for (cudaEvent_t e : A->copy_ev) cudaEventDestroy(e);
  for (cudaEvent_t e : A->group_ev) cudaEventDestroy(e);
  if (A->copy_stream) cudaStreamDestroy(A->copy_stream);
  delete A;
  return FA_OK;
}

extern "C" fa_status fa_aligner_set_reference(fa_aligner* A, const void* reference, fa_dtype dtype, int nz, int ny,
                                              int nx, const fa_scan_params* scan) {
  if (!A || !reference || !scan) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (dtype != FA_F32 && dtype != FA_U16) return fail(FA_ERR_BAD_ARG, "reference must be FA_F32 or FA_U16");
  std::lock_guard<std::mutex> lk(A->mu);
  FA_CU(cudaSetDevice(A->ctx->device));
  aligner_release_reference(A);
  if (!A->stream) FA_CU(cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking));
  const long long N = (long long)nz * ny * nx;
  const int b = A->prm.spatial_binning;
  A->nz = nz;
  A->ny = ny;
  A->nx = nx;
  A->dz = nz;
  A->dy = (ny + b - 1) / b;
  A->dx = (nx + b - 1) / b;
  A->nD = A->prm.nD > 0 ? A->prm.nD : A->prm.n_resampling_points * nz + 1;  // FrameWarpAligner.cpp:100
  void *raw, *plus1, *down;
  FA_TRY(dalloc(A->ctx, (size_t)N * dtype_size(dtype), &raw, A->ref_allocs));
  FA_TRY(dalloc(A->ctx, (size_t)N * sizeof(float), &plus1, A->ref_allocs));
  FA_TRY(dalloc(A->ctx, (size_t)A->dz * A->dy * A->dx * sizeof(float), &down, A->ref_allocs));
  FA_CU(cudaMemcpyAsync(raw, reference, (size_t)N * dtype_size(dtype), cudaMemcpyHostToDevice, A->stream));
  // smoothed_reference = smoothStack(reference) + 1, FrameWarpAligner.cpp:86-90
  if (A->prm.smoothing > 0) {
    fa_status sst = aligner_smooth(A, raw, dtype, A->stream);
    if (sst != FA_OK) return sst;
    FA_CU(fa::launch_offset_convert(A->smooth_out, FA_F32, plus1, FA_F32, N, A->stream));
  } else {
    FA_CU(fa::launch_offset_convert(raw, dtype, plus1, FA_F32, N, A->stream));
  }
  FA_CU(fa::launch_downsample(raw, dtype, nz, ny, nx, b, static_cast<float*>(down), A->stream));
  FA_CU(cudaStreamSynchronize(A->stream));
  // Frames go through the correlator in batched cuFFT plans of up to 64 frames (less for large volumes).
  fa_status st = correlator_create_impl(A->ctx, down, true, A->dz, A->dy, A->dx, 64, &A->corr);
  if (st == FA_OK)
    st = fa_set_reference_device(A->ctx, static_cast<const float*>(plus1), nz, ny, nx, A->nD, scan, A->prm.precision,
                                 &A->ref);
  dfree_all(A->ctx, A->ref_allocs);
  if (st != FA_OK) {
    std::string keep = g_err;
    aligner_release_reference(A);
    g_err = keep;
  }
  return st;
}

extern "C" fa_status fa_aligner_reference(const fa_aligner* A, fa_reference** ref) {
  if (!A || !ref) return fail(FA_ERR_BAD_ARG, "NULL argument");
  if (!A->ref) return fail(FA_ERR_STATE, "Reference imaging not yet set");
  *ref = A->ref;
  return FA_OK;
}

extern "C" fa_status fa_aligner_info(const fa_aligner* A, int* nD, int* n_dim) {
  if (!A || !A->ref) return fail(FA_ERR_STATE, "Reference imaging not yet set");
  if (nD) *nD = A->ref->nD;
  if (n_dim) *n_dim = A->ref->n_dim;
  return FA_OK;
}

extern "C" fa_status fa_aligner_add_frames(fa_aligner* A, const void* const* frames, fa_dtype dtype, int n,
                                           double* D_out, fa_align_stats* stats) {
  if (!A) return fail(FA_ERR_BAD_ARG, "NULL aligner");
  std::lock_guard<std::mutex> lk(A->mu);
  return aligner_run(A, frames, dtype, n, false, D_out, stats);
}

extern "C" fa_status fa_aligner_add_frames_device(fa_aligner* A, const void* const* frames, fa_dtype dtype, int n,
                                                  double* D_out, fa_align_stats* stats) {
  if (!A) return fail(FA_ERR_BAD_ARG, "NULL aligner");
  std::lock_guard<std::mutex> lk(A->mu);
  return aligner_run(A, frames, dtype, n, true, D_out, stats);
}

// ================================================================== measurement ===================

extern "C" long long fa_kernel_launches(void) { return g_launches.load(); }

extern "C" fa_status fa_aligner_last_device_ms(const fa_aligner* A, double* ms) {
  if (!A || !ms) return fail(FA_ERR_BAD_ARG, "NULL argument");
  *ms = A->last_ms;
  return FA_OK;
}

extern "C" fa_status fa_aligner_last_phase_ms(const fa_aligner* A, double* correlate_ms, double* total_ms) {
  if (!A || !correlate_ms || !total_ms) return fail(FA_ERR_BAD_ARG, "NULL argument");
  *correlate_ms = A->last_corr_ms;
  *total_ms = A->last_ms;
  return FA_OK;
}

extern "C" fa_status fa_profile_eval(fa_frame* const* frames, int n, const double* D, int launches,
                                     double* ms_per_launch) {
  if (!frames || n <= 0 || !D || launches <= 0 || !ms_per_launch) return fail(FA_ERR_BAD_ARG, "bad arguments");
  fa_reference* R = frames[0]->ref;
  for (int i = 0; i < n; i++)
    if (!frames[i] || frames[i]->ref != R) return fail(FA_ERR_BAD_ARG, "frames must share one reference");
  FA_CU(cudaSetDevice(R->ctx->device));
  std::vector<float4> dp((size_t)R->nD * fa::kDParamF4);
  make_dparams(D, R->nD, R->n_dim, dp.data());
  std::vector<Job> jobs(n);
  for (int i = 0; i < n; i++) {
    FA_CU(cudaMemcpy(frames[i]->job.dparams, dp.data(), dp.size() * sizeof(float4), cudaMemcpyHostToDevice));
    jobs[i] = frames[i]->job;
    frames[i]->have_last = false;
  }
  std::vector<Alloc> tmp;
  Job* jd;
  FA_TRY(dalloc_t(R->ctx, (size_t)n, &jd, tmp));
  cudaStream_t s = frames[0]->stream;
  cudaEvent_t e0, e1;
  cudaError_t e = cudaMemcpyAsync(jd, jobs.data(), n * sizeof(Job), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  // one untimed launch, then the timed ones
  const bool v4 = R->nx % 4 == 0;
  const int mb = n >= kManyFrames ? R->host.tune_mb : R->host.tune_mb_small;
  if (e == cudaSuccess)
    e = fa::launch_eval(jd, n, R->G.n_tiles, R->n_dim, frames[0]->kind, R->prec == FA_PREC_MIXED, s, v4, mb);
  if (e == cudaSuccess) e = cudaEventRecord(e0, s);
  for (int l = 0; l < launches && e == cudaSuccess; l++)
    e = fa::launch_eval(jd, n, R->G.n_tiles, R->n_dim, frames[0]->kind, R->prec == FA_PREC_MIXED, s, v4, mb);
  if (e == cudaSuccess) e = cudaEventRecord(e1, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  float ms = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  g_launches += launches + 1;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dfree_all(R->ctx, tmp);
  if (e != cudaSuccess) return fail(FA_ERR_CUDA, std::string("profile: ") + cudaGetErrorString(e));
  *ms_per_launch = ms / launches;
  return FA_OK;
}

// ================================================================== static-scratch evaluation ======

namespace fa {

fa_status static_eval_prepare(const fa_reference* R, const double* D, const RefDev** dev, const RefDev** host, int* nD,
                              int* n_dim, bool* mixed, int* device) {
  if (!finite_all(D, (size_t)R->nD * 3)) return fail(FA_ERR_BAD_ARG, "D has non-finite entries");
  *device = R->ctx->device;
  *dev = R->dev;
  *host = &R->host;
  *nD = R->nD;
  *n_dim = R->n_dim;
  *mixed = R->prec == FA_PREC_MIXED;
  return FA_OK;
}

fa_status static_eval_fail(fa_status s, const char* msg) { return fail(s, msg); }

void static_eval_dparams(const double* D, int nD, int n_dim, float4* out) { make_dparams(D, nD, n_dim, out); }

void static_eval_count_launches(int n) { g_launches += n; }

}  // namespace fa
